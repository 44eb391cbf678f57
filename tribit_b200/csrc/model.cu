// Learned dispatcher: MLP kernels (forward, backward, Adam, dispatch) and the
// C-ABI around them and around the per-row-block data they learn from.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "context.h"
#include "gen.h"

namespace tb {
namespace {

constexpr uint32_t kFull = 0xffffffffu;
constexpr int kNorm = 2 * kIn + 2 * kOut;  // in_mean, in_std, out_mean, out_std
constexpr int kModelThreads = 256;
constexpr char kMagic[8] = {'T', 'B', 'M', 'L', 'P', '0', '0', '1'};

__host__ __device__ __forceinline__ bool is_weight(int p) {
  return p < kB1 || (p >= kW2 && p < kB2) || (p >= kW3 && p < kB3);
}

// Shared-memory image of a model: parameters, W2 transposed (so the backward
// reads of W2 run across lanes without bank conflicts) and normalisation.
struct SmemModel {
  float p[kNumParams];
  float w2t[kH1 * kH2];
  float norm[kNorm];
};

__device__ void load_model(SmemModel& s, const float* __restrict__ eff, const float* __restrict__ norm) {
  for (int i = threadIdx.x; i < kNumParams; i += blockDim.x) s.p[i] = eff[i];
  for (int i = threadIdx.x; i < kH1 * kH2; i += blockDim.x) {
    const int k = i / kH2, j = i % kH2;
    s.w2t[j * kH1 + k] = eff[kW2 + i];
  }
  for (int i = threadIdx.x; i < kNorm; i += blockDim.x) s.norm[i] = norm[i];
  __syncthreads();
}

struct Acts {  // per-row activations kept for the weight gradients
  float* xn;   // B x kIn
  float* h1;   // B x kH1
  float* dz1;  // B x kH1
  float* h2;   // B x kH2
  float* dz2;  // B x kH2
  float* dy;   // B x kOut
};

// One warp per row; lane l owns hidden units l and l + 32 of both layers.
// Computes the normalised prediction; with Train also the backward pass for
// the MSE loss on normalised targets (scaled by inv_count), storing what the
// weight-gradient kernel needs.
template <bool Train>
__device__ __forceinline__ void row_pass(const SmemModel& s, const float* __restrict__ x, const float* __restrict__ y,
                                         float inv_count, float out[kOut], const Acts* acts, uint32_t slot,
                                         float* loss) {
  const int lane = threadIdx.x & 31;
  float xn[kIn];
#pragma unroll
  for (int q = 0; q < kIn; ++q) xn[q] = (x[q] - s.norm[q]) / s.norm[kIn + q];
  float z1a = s.p[kB1 + lane], z1b = s.p[kB1 + lane + 32];
#pragma unroll
  for (int q = 0; q < kIn; ++q) {
    z1a = fmaf(xn[q], s.p[kW1 + q * kH1 + lane], z1a);
    z1b = fmaf(xn[q], s.p[kW1 + q * kH1 + lane + 32], z1b);
  }
  const float h1a = fmaxf(z1a, 0.f), h1b = fmaxf(z1b, 0.f);
  float z2a = s.p[kB2 + lane], z2b = s.p[kB2 + lane + 32];
#pragma unroll 8
  for (int k = 0; k < 32; ++k) {
    const float hk = __shfl_sync(kFull, h1a, k);
    z2a = fmaf(hk, s.p[kW2 + k * kH2 + lane], z2a);
    z2b = fmaf(hk, s.p[kW2 + k * kH2 + lane + 32], z2b);
  }
#pragma unroll 8
  for (int k = 0; k < 32; ++k) {
    const float hk = __shfl_sync(kFull, h1b, k);
    z2a = fmaf(hk, s.p[kW2 + (k + 32) * kH2 + lane], z2a);
    z2b = fmaf(hk, s.p[kW2 + (k + 32) * kH2 + lane + 32], z2b);
  }
  const float h2a = fmaxf(z2a, 0.f), h2b = fmaxf(z2b, 0.f);
#pragma unroll
  for (int o = 0; o < kOut; ++o)
    out[o] = s.p[kB3 + o] + warp_sum(h2a * s.p[kW3 + lane * kOut + o] + h2b * s.p[kW3 + (lane + 32) * kOut + o]);
  if (!Train) return;
  float dy[kOut];
  float sq = 0.f;
#pragma unroll
  for (int o = 0; o < kOut; ++o) {
    const float t = (y[o] - s.norm[2 * kIn + o]) / s.norm[2 * kIn + kOut + o];
    const float e = out[o] - t;
    sq += e * e;
    dy[o] = 2.f * e * inv_count;
  }
  float dh2a = 0.f, dh2b = 0.f;
#pragma unroll
  for (int o = 0; o < kOut; ++o) {
    dh2a = fmaf(s.p[kW3 + lane * kOut + o], dy[o], dh2a);
    dh2b = fmaf(s.p[kW3 + (lane + 32) * kOut + o], dy[o], dh2b);
  }
  const float dz2a = z2a > 0.f ? dh2a : 0.f, dz2b = z2b > 0.f ? dh2b : 0.f;
  float dh1a = 0.f, dh1b = 0.f;
#pragma unroll 8
  for (int j = 0; j < 32; ++j) {
    const float dj = __shfl_sync(kFull, dz2a, j);
    dh1a = fmaf(s.w2t[j * kH1 + lane], dj, dh1a);
    dh1b = fmaf(s.w2t[j * kH1 + lane + 32], dj, dh1b);
  }
#pragma unroll 8
  for (int j = 0; j < 32; ++j) {
    const float dj = __shfl_sync(kFull, dz2b, j);
    dh1a = fmaf(s.w2t[(j + 32) * kH1 + lane], dj, dh1a);
    dh1b = fmaf(s.w2t[(j + 32) * kH1 + lane + 32], dj, dh1b);
  }
  const float dz1a = z1a > 0.f ? dh1a : 0.f, dz1b = z1b > 0.f ? dh1b : 0.f;
  const size_t r64 = (size_t)slot * 64;
  if (lane < kIn) acts->xn[(size_t)slot * kIn + lane] = (x[lane] - s.norm[lane]) / s.norm[kIn + lane];
  acts->h1[r64 + lane] = h1a;
  acts->h1[r64 + lane + 32] = h1b;
  acts->dz1[r64 + lane] = dz1a;
  acts->dz1[r64 + lane + 32] = dz1b;
  acts->h2[r64 + lane] = h2a;
  acts->h2[r64 + lane + 32] = h2b;
  acts->dz2[r64 + lane] = dz2a;
  acts->dz2[r64 + lane + 32] = dz2b;
  if (lane < kOut) acts->dy[(size_t)slot * kOut + lane] = dy[lane];
  if (lane == 0) atomicAdd(loss, sq);
}

// Forward + backward over rows idx[r0 .. r0 + B) (idx null: identity).
__global__ void __launch_bounds__(kModelThreads) k_fwd_bwd(const float* __restrict__ X, const float* __restrict__ Y,
                                                            const uint32_t* __restrict__ idx, uint32_t r0, uint32_t B,
                                                            const float* __restrict__ eff,
                                                            const float* __restrict__ norm, float inv_count, Acts acts,
                                                            float* loss) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SmemModel& s = *reinterpret_cast<SmemModel*>(smem_raw);
  load_model(s, eff, norm);
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = warp; i < B; i += nw) {
    const uint32_t row = idx ? idx[r0 + i] : r0 + i;
    float out[kOut];
    row_pass<true>(s, X + (size_t)row * kIn, Y + (size_t)row * kOut, inv_count, out, &acts, i, loss);
  }
}

// grad[p] = sum over the B rows of the batch, in row order (deterministic).
__global__ void k_wgrad(Acts a, uint32_t B, float* __restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNumParams) return;
  float g = 0.f;
  if (p < kB1) {
    const int i = p / kH1, j = p % kH1;
    for (uint32_t r = 0; r < B; ++r) g = fmaf(a.xn[(size_t)r * kIn + i], a.dz1[(size_t)r * kH1 + j], g);
  } else if (p < kW2) {
    const int j = p - kB1;
    for (uint32_t r = 0; r < B; ++r) g += a.dz1[(size_t)r * kH1 + j];
  } else if (p < kB2) {
    const int k = (p - kW2) / kH2, j = (p - kW2) % kH2;
    for (uint32_t r = 0; r < B; ++r) g = fmaf(a.h1[(size_t)r * kH1 + k], a.dz2[(size_t)r * kH2 + j], g);
  } else if (p < kW3) {
    const int j = p - kB2;
    for (uint32_t r = 0; r < B; ++r) g += a.dz2[(size_t)r * kH2 + j];
  } else if (p < kB3) {
    const int k = (p - kW3) / kOut, o = (p - kW3) % kOut;
    for (uint32_t r = 0; r < B; ++r) g = fmaf(a.h2[(size_t)r * kH2 + k], a.dy[(size_t)r * kOut + o], g);
  } else {
    const int o = p - kB3;
    for (uint32_t r = 0; r < B; ++r) g += a.dy[(size_t)r * kOut + o];
  }
  grad[p] = g;
}

__device__ __forceinline__ float to_eff(int p, float w) {
  return is_weight(p) ? __bfloat162float(__float2bfloat16_rn(w)) : w;
}

__global__ void k_adam(float* __restrict__ master, float* __restrict__ eff, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ grad, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNumParams) return;
  const float g = grad[p];
  const float mm = b1 * m[p] + (1.f - b1) * g;
  const float vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  const float w = master[p] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  master[p] = w;
  eff[p] = to_eff(p, w);
}

__global__ void k_refresh(const float* __restrict__ master, float* __restrict__ eff) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kNumParams) eff[p] = to_eff(p, master[p]);
}

// Denormalised predictions (log2 time per variant) for rows of X.
__global__ void __launch_bounds__(kModelThreads) k_predict(const float* __restrict__ X, uint32_t rows,
                                                            const float* __restrict__ eff,
                                                            const float* __restrict__ norm, float* __restrict__ Y) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SmemModel& s = *reinterpret_cast<SmemModel*>(smem_raw);
  load_model(s, eff, norm);
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t r = warp; r < rows; r += nw) {
    float out[kOut];
    row_pass<false>(s, X + (size_t)r * kIn, nullptr, 0.f, out, nullptr, 0, nullptr);
    if ((threadIdx.x & 31) < kOut) {
      const int o = threadIdx.x & 31;
      Y[(size_t)r * kOut + o] = out[o] * s.norm[2 * kIn + kOut + o] + s.norm[2 * kIn + o];
    }
  }
}

// variant_of[rb] = argmin of the predicted (normalised-back) time.
__global__ void __launch_bounds__(kModelThreads) k_dispatch(const float* __restrict__ feat, uint32_t nrb,
                                                             const float* __restrict__ eff,
                                                             const float* __restrict__ norm,
                                                             uint8_t* __restrict__ variant_of) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SmemModel& s = *reinterpret_cast<SmemModel*>(smem_raw);
  load_model(s, eff, norm);
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t rb = warp; rb < nrb; rb += nw) {
    float out[kOut];
    row_pass<false>(s, feat + (size_t)rb * kIn, nullptr, 0.f, out, nullptr, 0, nullptr);
    if ((threadIdx.x & 31) == 0) {
      // Bit tiles only where the block fits one tile (span of 1..kTileMaxK
      // column blocks); elsewhere the tile kernel would sweep the block's rows
      // one at a time on a single warp.
      const float span = feat[(size_t)rb * kIn + kFeatSpan];
      const bool tile_ok = span > 0.f && span <= log2f(1.f + (float)kTileMaxK) + 1e-4f;
      int best = -1;
      float bt = 0.f;
      for (int o = 0; o < kOut; ++o) {
        if (o == TRIBIT_VARIANT_MMA && !tile_ok) continue;
        const float t = out[o] * s.norm[2 * kIn + kOut + o] + s.norm[2 * kIn + o];
        if (best < 0 || t < bt) bt = t, best = o;
      }
      variant_of[rb] = (uint8_t)best;
    }
  }
}

constexpr size_t kModelSmem = sizeof(SmemModel);

void set_smem_attrs() {
  once_per_device<1>([] {
    TB_CUDA(cudaFuncSetAttribute(k_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kModelSmem));
    TB_CUDA(cudaFuncSetAttribute(k_predict, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kModelSmem));
    TB_CUDA(cudaFuncSetAttribute(k_dispatch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kModelSmem));
  });
}

unsigned grid_warps(uint64_t rows) {
  const uint64_t g = ceil_div<uint64_t>(rows, kModelThreads / 32);
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 8));
}

struct TrainBuffers {
  float* X = nullptr;
  float* Y = nullptr;
  uint32_t* idx = nullptr;
  float* loss = nullptr;
  Acts acts{};
};

TrainBuffers layout_train(Arena& ar, uint64_t rows, uint32_t B) {
  TrainBuffers t;
  t.X = ar.take<float>(rows * kIn + 1);
  t.Y = ar.take<float>(rows * kOut + 1);
  t.idx = ar.take<uint32_t>(rows + 1);
  t.loss = ar.take<float>(1);
  t.acts.xn = ar.take<float>((uint64_t)B * kIn);
  t.acts.h1 = ar.take<float>((uint64_t)B * kH1);
  t.acts.dz1 = ar.take<float>((uint64_t)B * kH1);
  t.acts.h2 = ar.take<float>((uint64_t)B * kH2);
  t.acts.dz2 = ar.take<float>((uint64_t)B * kH2);
  t.acts.dy = ar.take<float>((uint64_t)B * kOut);
  return t;
}

TrainBuffers stage_training(tribit_context* c, const float* X, const float* Y, uint64_t rows, uint32_t B) {
  Arena& ar = c->train_arena;
  ar.begin(true);
  layout_train(ar, rows, B);
  ar.reserve(ar.used());
  ar.begin(false);
  TrainBuffers t = layout_train(ar, rows, B);
  TB_CUDA(cudaMemcpyAsync(t.X, X, rows * kIn * sizeof(float), cudaMemcpyHostToDevice, c->st));
  if (Y) TB_CUDA(cudaMemcpyAsync(t.Y, Y, rows * kOut * sizeof(float), cudaMemcpyHostToDevice, c->st));
  return t;
}

void require_model(tribit_context* c) {
  if (!c->model.loaded) throw StatusError(TRIBIT_ERR_NO_MODEL, "no dispatcher model: load or initialise one first");
}

}  // namespace

void model_alloc(DeviceModel& m, cudaStream_t st) {
  if (m.master) return;
  float* base = nullptr;
  const size_t n = 5 * (size_t)kNumParams + kNorm;
  TB_CUDA(cudaMalloc(&base, n * sizeof(float)));
  // On the caller's stream: the uploads that follow are ordered after it.
  TB_CUDA(cudaMemsetAsync(base, 0, n * sizeof(float), st));
  m.master = base;
  m.eff = base + kNumParams;
  m.m = base + 2 * kNumParams;
  m.v = base + 3 * kNumParams;
  m.grad = base + 4 * kNumParams;
  m.norm = base + 5 * kNumParams;
}

void model_free(DeviceModel& m) {
  if (m.master) cudaFree(m.master);
  m = DeviceModel{};
}

void model_refresh_eff(DeviceModel& m, cudaStream_t st) {
  k_refresh<<<(kNumParams + 255) / 256, 256, 0, st>>>(m.master, m.eff);
  TB_LAUNCH_CHECK();
}

void model_dispatch(const DeviceModel& m, const float* features, uint32_t nrb, uint8_t* variant_of, cudaStream_t st) {
  if (nrb == 0) return;
  set_smem_attrs();
  k_dispatch<<<grid_warps(nrb), kModelThreads, kModelSmem, st>>>(features, nrb, m.eff, m.norm, variant_of);
  TB_LAUNCH_CHECK();
}

void apply_dispatch(tribit_context* c, cudaStream_t st) {
  const int mode = c->opts.dispatch;
  c->sched.piece_width = c->piece_width;
  c->sched.tile_min_nnz = c->tile_min_nnz;
  c->sched.merge_ratio = c->merge_ratio;
  c->sched.tile_engine = c->tile_engine;
  // Only merge blocks use the hub lists; the plain rule picks merge blocks
  // from the neighbour-side features, so it reads the full set too.
  c->sched.hubs = mode == TRIBIT_DISPATCH_LEARNED || mode == TRIBIT_DISPATCH_MERGE || mode == TRIBIT_DISPATCH_PLAIN;
  drop_graph(c);
  if (mode == TRIBIT_DISPATCH_LEARNED) {
    require_model(c);
    compute_features(c->prep.view, c->sched, TRIBIT_DISPATCH_PLAIN, true, st);
    model_dispatch(c->model, c->sched.features, c->sched.num_row_blocks, c->sched.variant_of, st);
  } else {
    compute_features(c->prep.view, c->sched, mode, mode == TRIBIT_DISPATCH_PLAIN, st);
  }
  // Both rules choose merge for the hub pass; a schedule taken without hub
  // lists (the rows tier under a small device budget) sweeps those blocks as
  // bitmaps instead (RMAT-24: 132 ms all-bitmap against 168 ms merge without
  // the hub pass).
  if (!c->sched.eflag && (mode == TRIBIT_DISPATCH_LEARNED || mode == TRIBIT_DISPATCH_PLAIN))
    merge_blocks_to_bitmap(c->sched, st);
  build_pieces(c->prep.view, c->sched, st);
}

}  // namespace tb

using tb::DeviceGuard;
using tb::guarded;
using tb::StatusError;

extern "C" {

uint32_t tribit_model_num_params(void) { return (uint32_t)tb::kNumParams; }

tribit_status tribit_model_init(tribit_context* c, uint64_t seed, const float* norm) {
  if (!c || !norm) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    DeviceGuard dg(c->device);
    tb::model_alloc(c->model, c->st);
    std::vector<float> p(tb::kNumParams, 0.f);
    auto fill = [&](int off, int fan_in, int count) {
      const double lim = std::sqrt(6.0 / fan_in);
      for (int i = 0; i < count; ++i) p[off + i] = (float)((2.0 * tb_unit(tb_rand(seed, off + i)) - 1.0) * lim);
    };
    fill(tb::kW1, tb::kIn, tb::kIn * tb::kH1);
    fill(tb::kW2, tb::kH1, tb::kH1 * tb::kH2);
    fill(tb::kW3, tb::kH2, tb::kH2 * tb::kOut);
    TB_CUDA(cudaMemcpyAsync(c->model.master, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice, c->st));
    TB_CUDA(cudaMemsetAsync(c->model.m, 0, 2 * tb::kNumParams * sizeof(float), c->st));
    TB_CUDA(cudaMemcpyAsync(c->model.norm, norm, tb::kNorm * sizeof(float), cudaMemcpyHostToDevice, c->st));
    tb::model_refresh_eff(c->model, c->st);
    TB_CUDA(cudaStreamSynchronize(c->st));
    c->model.steps = 0;
    c->model.loaded = true;
  });
}

tribit_status tribit_model_get_params(tribit_context* c, float* out, int effective) {
  if (!c || !out) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    tb::require_model(c);
    DeviceGuard dg(c->device);
    TB_CUDA(cudaMemcpyAsync(out, effective ? c->model.eff : c->model.master, tb::kNumParams * sizeof(float),
                            cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaStreamSynchronize(c->st));
  });
}

tribit_status tribit_model_set_params(tribit_context* c, const float* in) {
  if (!c || !in) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    tb::require_model(c);
    DeviceGuard dg(c->device);
    TB_CUDA(cudaMemcpyAsync(c->model.master, in, tb::kNumParams * sizeof(float), cudaMemcpyHostToDevice, c->st));
    tb::model_refresh_eff(c->model, c->st);
    TB_CUDA(cudaStreamSynchronize(c->st));
  });
}

tribit_status tribit_model_predict(tribit_context* c, const float* x, uint64_t rows, float* y) {
  if (!c || (!x && rows) || (!y && rows)) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    tb::require_model(c);
    DeviceGuard dg(c->device);
    if (rows == 0) return;
    tb::set_smem_attrs();
    tb::TrainBuffers t = tb::stage_training(c, x, nullptr, rows, 1);
    tb::k_predict<<<tb::grid_warps(rows), tb::kModelThreads, tb::kModelSmem, c->st>>>(t.X, (uint32_t)rows,
                                                                                     c->model.eff, c->model.norm, t.Y);
    TB_LAUNCH_CHECK();
    TB_CUDA(cudaMemcpyAsync(y, t.Y, rows * tb::kOut * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaStreamSynchronize(c->st));
  });
}

tribit_status tribit_model_gradients(tribit_context* c, const float* x, const float* y, uint64_t rows, float* grad,
                                     float* loss_out) {
  if (!c || !x || !y || !grad || rows == 0 || rows > 0xffffffffull) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    tb::require_model(c);
    DeviceGuard dg(c->device);
    tb::set_smem_attrs();
    tb::TrainBuffers t = tb::stage_training(c, x, y, rows, (uint32_t)rows);
    TB_CUDA(cudaMemsetAsync(t.loss, 0, sizeof(float), c->st));
    const float inv = 1.f / (float)(tb::kOut * rows);
    tb::k_fwd_bwd<<<tb::grid_warps(rows), tb::kModelThreads, tb::kModelSmem, c->st>>>(
        t.X, t.Y, nullptr, 0, (uint32_t)rows, c->model.eff, c->model.norm, inv, t.acts, t.loss);
    TB_LAUNCH_CHECK();
    tb::k_wgrad<<<(tb::kNumParams + 255) / 256, 256, 0, c->st>>>(t.acts, (uint32_t)rows, c->model.grad);
    TB_LAUNCH_CHECK();
    float loss = 0.f;
    TB_CUDA(cudaMemcpyAsync(grad, c->model.grad, tb::kNumParams * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaMemcpyAsync(&loss, t.loss, sizeof(float), cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaStreamSynchronize(c->st));
    if (loss_out) *loss_out = loss / (float)(tb::kOut * rows);
  });
}

tribit_status tribit_model_train(tribit_context* c, const float* x, const float* y, uint64_t rows, uint32_t epochs,
                                 uint32_t batch, float lr, uint64_t seed, float* loss_out) {
  if (!c || !x || !y || rows == 0 || rows > 0xffffffffull || batch == 0 || epochs == 0) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    tb::require_model(c);
    DeviceGuard dg(c->device);
    tb::set_smem_attrs();
    const uint32_t B = (uint32_t)std::min<uint64_t>(batch, rows);
    tb::TrainBuffers t = tb::stage_training(c, x, y, rows, B);
    std::vector<uint32_t> order(rows);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float last = 0.f;
    for (uint32_t ep = 0; ep < epochs; ++ep) {
      for (uint64_t i = 0; i < rows; ++i) order[i] = (uint32_t)i;
      for (uint64_t i = rows - 1; i > 0; --i) std::swap(order[i], order[tb_rand(seed + ep, i) % (i + 1)]);
      TB_CUDA(cudaMemcpyAsync(t.idx, order.data(), rows * sizeof(uint32_t), cudaMemcpyHostToDevice, c->st));
      TB_CUDA(cudaMemsetAsync(t.loss, 0, sizeof(float), c->st));
      for (uint64_t r0 = 0; r0 < rows; r0 += B) {
        const uint32_t nb = (uint32_t)std::min<uint64_t>(B, rows - r0);
        const float inv = 1.f / (float)(tb::kOut * nb);
        tb::k_fwd_bwd<<<tb::grid_warps(nb), tb::kModelThreads, tb::kModelSmem, c->st>>>(
            t.X, t.Y, t.idx, (uint32_t)r0, nb, c->model.eff, c->model.norm, inv, t.acts, t.loss);
        TB_LAUNCH_CHECK();
        tb::k_wgrad<<<(tb::kNumParams + 255) / 256, 256, 0, c->st>>>(t.acts, nb, c->model.grad);
        TB_LAUNCH_CHECK();
        const int step = ++c->model.steps;
        tb::k_adam<<<(tb::kNumParams + 255) / 256, 256, 0, c->st>>>(
            c->model.master, c->model.eff, c->model.m, c->model.v, c->model.grad, lr, b1, b2, eps,
            1.f - std::pow(b1, (float)step), 1.f - std::pow(b2, (float)step));
        TB_LAUNCH_CHECK();
      }
      TB_CUDA(cudaMemcpyAsync(&last, t.loss, sizeof(float), cudaMemcpyDeviceToHost, c->st));
      TB_CUDA(cudaStreamSynchronize(c->st));
    }
    if (loss_out) *loss_out = last / (float)(tb::kOut * rows);
  });
}

tribit_status tribit_block_features(tribit_context* c, float* out, uint64_t cap, uint64_t* num_row_blocks) {
  if (!c || !num_row_blocks) return TRIBIT_ERR_INVALID_ARGUMENT;
  if (!c->prepared) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    DeviceGuard dg(c->device);
    const uint64_t nrb = c->sched.num_row_blocks;
    *num_row_blocks = nrb;
    if (!out) return;
    if (cap < nrb * tb::kIn) throw StatusError(TRIBIT_ERR_INVALID_ARGUMENT, "feature buffer too small");
    tb::compute_features(c->prep.view, c->sched, TRIBIT_DISPATCH_PLAIN, true, c->st);
    TB_CUDA(cudaMemcpyAsync(out, c->sched.features, nrb * tb::kIn * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    tb::apply_dispatch(c, c->st);
    TB_CUDA(cudaStreamSynchronize(c->st));
  });
}

tribit_status tribit_block_times(tribit_context* c, int variant, float* cycles_out, uint64_t cap,
                                 uint64_t* triangles_out, float* variant_ms) {
  if (!c || !c->prepared || variant < 0 || variant >= TRIBIT_NUM_VARIANTS) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    DeviceGuard dg(c->device);
    const uint64_t nrb = c->sched.num_row_blocks;
    if (cycles_out && cap < nrb) throw StatusError(TRIBIT_ERR_INVALID_ARGUMENT, "timing buffer too small");
    // Per-block times, and the in-list rows the hub pieces charge their
    // cycles to (a one-piece schedule keeps no rows).
    tb::Arena& ar = c->timing_arena;
    const bool hub_rows = variant == TRIBIT_VARIANT_MERGE && c->sched.inl;
    ar.begin(true);
    ar.take<unsigned long long>(nrb + 1);
    if (hub_rows) ar.take<uint32_t>(c->sched.inl_cap);
    ar.reserve(ar.used());
    ar.begin(false);
    unsigned long long* ns = ar.take<unsigned long long>(nrb + 1);
    c->sched.inrow = hub_rows ? ar.take<uint32_t>(c->sched.inl_cap) : nullptr;
    TB_CUDA(cudaMemsetAsync(ns, 0, (nrb + 1) * sizeof(unsigned long long), c->st));
    if (nrb) TB_CUDA(cudaMemsetAsync(c->sched.variant_of, variant, nrb, c->st));
    c->sched.hubs = variant == TRIBIT_VARIANT_MERGE;
    c->sched.hub_rows = hub_rows;  // the hub pieces charge their cycles to their rows' blocks
    tb::build_pieces(c->prep.view, c->sched, c->st);
    c->sched.hub_rows = false;
    tb::CountConfig cfg = tb::count_config(c);
    cfg.block_ns = ns;
    cfg.variant_start = c->ev[0];
    cfg.variant_stop = c->ev[1];
    tb::launch_count(c->prep.view, c->sched, c->prep.stats, c->per_graph, cfg, c->st);
    std::vector<unsigned long long> h(nrb + 1);
    TB_CUDA(cudaMemcpyAsync(h.data(), ns, nrb * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaMemcpyAsync(c->h_stats, c->prep.stats, sizeof(tb::DeviceStats), cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaStreamSynchronize(c->st));
    if (triangles_out) *triangles_out = c->h_stats->triangles;
    if (variant_ms) TB_CUDA(cudaEventElapsedTime(variant_ms, c->ev[0], c->ev[1]));
    if (cycles_out)
      for (uint64_t i = 0; i < nrb; ++i) cycles_out[i] = (float)h[i];
    c->sched.inrow = nullptr;
    tb::apply_dispatch(c, c->st);
    TB_CUDA(cudaStreamSynchronize(c->st));
  });
}

tribit_status tribit_model_save(tribit_context* c, const char* path) {
  if (!c || !path) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    tb::require_model(c);
    DeviceGuard dg(c->device);
    std::vector<float> p(tb::kNumParams), nrm(tb::kNorm);
    TB_CUDA(cudaMemcpyAsync(p.data(), c->model.master, p.size() * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaMemcpyAsync(nrm.data(), c->model.norm, nrm.size() * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaStreamSynchronize(c->st));
    FILE* f = std::fopen(path, "wb");
    if (!f) throw StatusError(TRIBIT_ERR_IO, "cannot write model file");
    const uint32_t dims[4] = {tb::kIn, tb::kH1, tb::kH2, tb::kOut};
    bool ok = std::fwrite(tb::kMagic, 1, 8, f) == 8 && std::fwrite(dims, 4, 4, f) == 4 &&
              std::fwrite(nrm.data(), 4, nrm.size(), f) == nrm.size() && std::fwrite(p.data(), 4, p.size(), f) == p.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) throw StatusError(TRIBIT_ERR_IO, "cannot write model file");
  });
}

tribit_status tribit_model_load(tribit_context* c, const char* path) {
  if (!c || !path) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    FILE* f = std::fopen(path, "rb");
    if (!f) throw StatusError(TRIBIT_ERR_IO, "cannot open model file");
    char magic[8];
    uint32_t dims[4];
    std::vector<float> p(tb::kNumParams), nrm(tb::kNorm);
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, tb::kMagic, 8) == 0 &&
              std::fread(dims, 4, 4, f) == 4 && dims[0] == (uint32_t)tb::kIn && dims[1] == (uint32_t)tb::kH1 &&
              dims[2] == (uint32_t)tb::kH2 && dims[3] == (uint32_t)tb::kOut &&
              std::fread(nrm.data(), 4, nrm.size(), f) == nrm.size() &&
              std::fread(p.data(), 4, p.size(), f) == p.size();
    std::fclose(f);
    if (!ok) throw StatusError(TRIBIT_ERR_FORMAT, "not a tribit dispatcher model file");
    DeviceGuard dg(c->device);
    tb::model_alloc(c->model, c->st);
    TB_CUDA(cudaMemcpyAsync(c->model.master, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice, c->st));
    TB_CUDA(cudaMemcpyAsync(c->model.norm, nrm.data(), nrm.size() * sizeof(float), cudaMemcpyHostToDevice, c->st));
    TB_CUDA(cudaMemsetAsync(c->model.m, 0, 2 * tb::kNumParams * sizeof(float), c->st));
    tb::model_refresh_eff(c->model, c->st);
    TB_CUDA(cudaStreamSynchronize(c->st));
    c->model.steps = 0;
    c->model.loaded = true;
  });
}

}  // extern "C"
