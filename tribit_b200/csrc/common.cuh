// Shared helpers for the tribit_b200 CUDA sources.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <mutex>
#include <stdexcept>
#include <string>

#include "tribit.h"

namespace tb {

// A failed CUDA call inside the library. Converted to a tribit_status at the
// C-ABI boundary; never escapes an extern "C" function.
struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const char* what_) : std::runtime_error(what_), code(c) {}
};

struct StatusError : std::runtime_error {
  tribit_status status;
  StatusError(tribit_status s, const std::string& what_) : std::runtime_error(what_), status(s) {}
};

inline void cuda_check(cudaError_t e, const char* expr, const char* file, int line) {
  if (e != cudaSuccess) {
    char buf[512];
    std::snprintf(buf, sizeof buf, "%s failed at %s:%d: %s", expr, file, line, cudaGetErrorString(e));
    throw CudaError(e, buf);
  }
}

#define TB_CUDA(expr) ::tb::cuda_check((expr), #expr, __FILE__, __LINE__)
#define TB_LAUNCH_CHECK() ::tb::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

constexpr int kWarp = 32;

template <typename T>
__host__ __device__ __forceinline__ T ceil_div(T a, T b) {
  return (a + b - 1) / b;
}

inline int bits_for(uint64_t n) {  // smallest b with 2^b >= n (at least 1)
  int b = 1;
  while (b < 64 && (1ull << b) < n) ++b;
  return b;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

template <typename T>
__device__ __forceinline__ T warp_inclusive_sum(T v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) >= (unsigned)o) v += t;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T t = __shfl_xor_sync(0xffffffffu, v, o);
    v = t > v ? t : v;
  }
  return v;
}

// Runs fn() once per CUDA device (the current one when called), for settings
// such as cudaFuncSetAttribute that apply per device. Thread-safe; a call whose
// fn throws leaves the device unmarked, so a later call retries it.
template <int Tag, typename F>
void once_per_device(F&& fn) {
  constexpr int kMaxDevices = 64;
  static std::once_flag flags[kMaxDevices];
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice", __FILE__, __LINE__);
  if (dev < 0 || dev >= kMaxDevices) {
    fn();
    return;
  }
  std::call_once(flags[dev], fn);
}

// Device-side error flags shared by the preprocessing and counting kernels.
enum : uint32_t {
  kErrIdRange = 1u << 0,    // an entry named a vertex >= num_nodes
  kErrReserved = 1u << 1,   // never set (kept so the flag values stay those of the C-ABI)
  kErrTimeout = 1u << 2,    // a bounded wait gave up
  kErrInput = 1u << 3,      // streamed counts: host entries changed between their passes
};

}  // namespace tb
