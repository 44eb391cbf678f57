// Learned dispatcher: a 16 -> 64 -> 64 -> 3 MLP over row-block features that
// predicts, for each counting variant, log2 of the time the variant spends on
// the row block; dispatch picks the smallest. It changes scheduling only:
// every variant counts exactly, so the count never depends on the model.
//
// Weights are used in BF16 (rounded from FP32 master copies), activations and
// accumulation are FP32. Forward, backward and Adam are hand-written kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tb {

constexpr int kIn = 16, kH1 = 64, kH2 = 64, kOut = 3;
constexpr int kW1 = 0;                      // [kIn][kH1]
constexpr int kB1 = kW1 + kIn * kH1;        // [kH1]
constexpr int kW2 = kB1 + kH1;              // [kH1][kH2]
constexpr int kB2 = kW2 + kH1 * kH2;        // [kH2]
constexpr int kW3 = kB2 + kH2;              // [kH2][kOut]
constexpr int kB3 = kW3 + kH2 * kOut;       // [kOut]
constexpr int kNumParams = kB3 + kOut;      // 5443

// Device-resident model. `eff` holds the parameters as the kernels use them:
// weights rounded to BF16 (stored as float), biases in FP32.
struct DeviceModel {
  float* master = nullptr;  // kNumParams, FP32
  float* eff = nullptr;     // kNumParams
  float* m = nullptr;       // Adam first moment
  float* v = nullptr;       // Adam second moment
  float* grad = nullptr;    // kNumParams
  float* norm = nullptr;    // in_mean[16], in_std[16], out_mean[3], out_std[3]
  int steps = 0;
  bool loaded = false;
};

void model_alloc(DeviceModel& m, cudaStream_t st);
void model_free(DeviceModel& m);
void model_refresh_eff(DeviceModel& m, cudaStream_t st);

// variant_of[rb] = argmin over variants of the predicted time, for row blocks
// with work; features are nrb x kIn.
void model_dispatch(const DeviceModel& m, const float* features, uint32_t nrb, uint8_t* variant_of, cudaStream_t st);

}  // namespace tb
