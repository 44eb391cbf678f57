// Device-wide scans (sum / min / max) and the LSD radix sort built on them.
//
// These replace the CUB calls of the reference (DeviceScan tribit.cu:116-153,
// DeviceRadixSort tribit.cu:358-397, DeviceSelect::Unique tribit.cu:335-356).
// Both are "reduce, then scan": per-tile partials, a scan of the partials
// (recursive), then a per-tile pass that applies the carry. No kernel waits on
// another CTA, so nothing here can spin.
//
// Scratch is taken from an Arena by the take_* helpers in a fixed order, so a
// caller can size one reservation for a whole pipeline; the launch functions
// themselves only launch.
#pragma once
#include "arena.h"
#include "common.cuh"

namespace tb {

struct OpSum {
  template <typename T>
  __device__ __forceinline__ T operator()(T a, T b) const {
    return a + b;
  }
};
struct OpMin {
  template <typename T>
  __device__ __forceinline__ T operator()(T a, T b) const {
    return b < a ? b : a;
  }
};
struct OpMax {
  template <typename T>
  __device__ __forceinline__ T operator()(T a, T b) const {
    return a < b ? b : a;
  }
};

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of one value per thread (256 threads). Returns the
// thread's exclusive prefix; *total receives the block aggregate.
template <typename T, typename Op>
__device__ __forceinline__ T block_exclusive_scan(T v, Op op, T id, T* total) {
  __shared__ T warp_tot[kScanThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc = op(inc, t);
  }
  if (lane == 31) warp_tot[w] = inc;
  __syncthreads();
  T wpre = id, all = id;
#pragma unroll
  for (int k = 0; k < kScanThreads / 32; ++k) {
    if (k < w) wpre = op(wpre, warp_tot[k]);
    all = op(all, warp_tot[k]);
  }
  T ex = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) ex = id;
  __syncthreads();  // warp_tot may be reused by the next call
  *total = all;
  return op(wpre, ex);
}

template <bool Rev>
__device__ __forceinline__ uint64_t scan_index(uint64_t i, uint64_t n) {
  return Rev ? n - 1 - i : i;
}

template <typename T, typename Op, bool Rev>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const T* in, uint64_t n,
                                                               T* __restrict__ partial, Op op, T id) {
  uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  T acc = id;
#pragma unroll 4
  for (int j = 0; j < kScanItems; ++j) {
    uint64_t i = base + (uint64_t)j * kScanThreads + threadIdx.x;
    if (i < n) acc = op(acc, in[scan_index<Rev>(i, n)]);
  }
  T tot;
  block_exclusive_scan(acc, op, id, &tot);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

// Scans one tile. carry (may be null) holds the exclusive prefix of each tile.
template <typename T, typename Op, bool Rev>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const T* in, T* out, uint64_t n,
                                                              const T* __restrict__ carry, Op op, T id,
                                                              bool exclusive) {
  constexpr int kPad = kScanTile + kScanTile / 32;
  __shared__ T s[kPad];
  uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  for (int j = 0; j < kScanItems; ++j) {
    int p = j * kScanThreads + threadIdx.x;
    uint64_t i = base + p;
    s[p + p / 32] = i < n ? in[scan_index<Rev>(i, n)] : id;
  }
  __syncthreads();
  T v[kScanItems];
  T acc = id;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int p = threadIdx.x * kScanItems + k;
    v[k] = s[p + p / 32];
    acc = op(acc, v[k]);
  }
  T tot;
  T pre = block_exclusive_scan(acc, op, id, &tot);
  if (carry) pre = op(carry[blockIdx.x], pre);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int p = threadIdx.x * kScanItems + k;
    T nxt = op(pre, v[k]);
    s[p + p / 32] = exclusive ? pre : nxt;
    pre = nxt;
  }
  __syncthreads();
  for (int j = 0; j < kScanItems; ++j) {
    int p = j * kScanThreads + threadIdx.x;
    uint64_t i = base + p;
    if (i < n) out[scan_index<Rev>(i, n)] = s[p + p / 32];
  }
}

// Elements of scratch a scan of n elements needs (partials of every level).
inline uint64_t scan_temp_elems(uint64_t n) {
  uint64_t tiles = ceil_div<uint64_t>(n, kScanTile);
  return tiles <= 1 ? 0 : tiles + scan_temp_elems(tiles);
}

// out[i] = op-scan of in (exclusive or inclusive); Rev scans from the end.
// in and out may alias. temp holds scan_temp_elems(n) elements. Launches only.
template <typename T, typename Op, bool Rev = false>
void device_scan(const T* in, T* out, uint64_t n, bool exclusive, Op op, T id, T* temp, cudaStream_t st) {
  if (n == 0) return;
  uint64_t tiles = ceil_div<uint64_t>(n, kScanTile);
  if (tiles == 1) {
    k_scan_apply<T, Op, Rev><<<1, kScanThreads, 0, st>>>(in, out, n, nullptr, op, id, exclusive);
    TB_LAUNCH_CHECK();
    return;
  }
  T* partial = temp;
  k_scan_reduce<T, Op, Rev><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, partial, op, id);
  TB_LAUNCH_CHECK();
  device_scan<T, Op, false>(partial, partial, tiles, true, op, id, temp + tiles, st);
  k_scan_apply<T, Op, Rev><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, n, partial, op, id, exclusive);
  TB_LAUNCH_CHECK();
}

// Takes scratch for a scan of n elements from the arena.
template <typename T>
T* take_scan_temp(Arena& ar, uint64_t n) {
  return ar.take<T>(scan_temp_elems(n) + 1);
}

// ------------------------------------------------------------------------
// LSD radix sort, 8-bit digits, stable. A pass is: per-tile digit counts
// (digit-major so one exclusive scan yields every tile's global offsets),
// the scan, and a scatter that ranks keys inside the tile with warp-level
// multisplit (__match_any_sync), stages the tile in shared memory in digit
// order and writes each digit run contiguously.
// ------------------------------------------------------------------------

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortKeysPerThread = 16;
constexpr int kSortTile = kSortThreads * kSortKeysPerThread;

template <typename K>
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const K* __restrict__ keys, uint64_t n, int shift,
                                                              uint32_t tiles, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll 4
  for (int j = 0; j < kSortKeysPerThread; ++j) {
    uint64_t i = base + (uint64_t)j * kSortThreads + threadIdx.x;
    uint32_t d = i < n ? (uint32_t)((keys[i] >> shift) & 255) : 256u;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    if (d < 256 && (threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicAdd(&h[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

struct NoVal {};

template <typename K, typename V, bool HasVals>
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const K* __restrict__ kin, K* __restrict__ kout,
                                                                 const V* __restrict__ vin, V* __restrict__ vout,
                                                                 uint64_t n, int shift, uint32_t tiles,
                                                                 const uint32_t* __restrict__ offs) {
  __shared__ K skeys[kSortTile];
  __shared__ V svals[HasVals ? kSortTile : 1];
  __shared__ uint32_t wcnt[kSortWarps][256];
  __shared__ uint32_t dstart[256];
  __shared__ uint32_t gbase[256];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int d = threadIdx.x; d < kSortWarps * 256; d += kSortThreads) (&wcnt[0][0])[d] = 0;
  __syncthreads();
  const uint64_t tbase = (uint64_t)blockIdx.x * kSortTile;
  const uint64_t wbase = tbase + (uint64_t)w * (kSortKeysPerThread * 32);
  const uint32_t lt = (1u << lane) - 1u;
  K key[kSortKeysPerThread];
  V val[HasVals ? kSortKeysPerThread : 1];
  uint32_t pos[kSortKeysPerThread];
#pragma unroll
  for (int k = 0; k < kSortKeysPerThread; ++k) {
    uint64_t i = wbase + (uint64_t)k * 32 + lane;
    bool valid = i < n;
    key[k] = valid ? kin[i] : K(0);
    if constexpr (HasVals) val[k] = valid ? vin[i] : V();
    uint32_t d = valid ? (uint32_t)((key[k] >> shift) & 255) : 256u;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    int leader = __ffs(peers) - 1;
    uint32_t b = 0;
    if (valid && lane == leader) {
      b = wcnt[w][d];
      wcnt[w][d] = b + __popc(peers);
    }
    b = __shfl_sync(0xffffffffu, b, leader);
    pos[k] = b + __popc(peers & lt);
  }
  __syncthreads();
  {
    const int d = threadIdx.x;
    uint32_t s = 0;
#pragma unroll
    for (int ww = 0; ww < kSortWarps; ++ww) {
      uint32_t c = wcnt[ww][d];
      wcnt[ww][d] = s;
      s += c;
    }
    uint32_t tot;
    uint32_t ex = block_exclusive_scan<uint32_t>(s, OpSum{}, 0u, &tot);
    dstart[d] = ex;
    gbase[d] = offs[(uint64_t)d * tiles + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kSortKeysPerThread; ++k) {
    uint64_t i = wbase + (uint64_t)k * 32 + lane;
    if (i < n) {
      uint32_t d = (uint32_t)((key[k] >> shift) & 255);
      uint32_t p = dstart[d] + wcnt[w][d] + pos[k];
      skeys[p] = key[k];
      if constexpr (HasVals) svals[p] = val[k];
    }
  }
  __syncthreads();
  uint64_t rem = n - tbase;
  uint32_t cnt = rem < (uint64_t)kSortTile ? (uint32_t)rem : (uint32_t)kSortTile;
  for (uint32_t p = threadIdx.x; p < cnt; p += kSortThreads) {
    K kk = skeys[p];
    uint32_t d = (uint32_t)((kk >> shift) & 255);
    uint64_t o = (uint64_t)gbase[d] + (p - dstart[d]);
    kout[o] = kk;
    if constexpr (HasVals) vout[o] = svals[p];
  }
}

struct RadixTemp {
  uint32_t* hist = nullptr;
  uint32_t* scan = nullptr;
};

// Takes the scratch a radix sort of n keys needs.
inline RadixTemp take_radix_temp(Arena& ar, uint64_t n) {
  uint64_t tiles = ceil_div<uint64_t>(n, kSortTile);
  RadixTemp t;
  t.hist = ar.take<uint32_t>(tiles * 256 + 1);
  t.scan = take_scan_temp<uint32_t>(ar, tiles * 256);
  return t;
}

// Sorts keys[0, n) on bits [begin_bit, end_bit) (stable). keys_alt (and
// vals_alt) are scratch of the same size. Returns the buffer that holds the
// sorted keys (keys or keys_alt); *vals_sorted receives the matching values
// buffer. first_hist_ready: tmp.hist already holds the first pass's per-tile
// digit counts (digit-major, k_radix_hist's layout), counted by the kernel that
// wrote the keys. Launches only.
template <typename K, typename V, bool HasVals>
K* radix_sort(K* keys, K* keys_alt, V* vals, V* vals_alt, uint64_t n, int end_bit, const RadixTemp& tmp,
              cudaStream_t st, V** vals_sorted, int begin_bit = 0, bool first_hist_ready = false) {
  static_assert(sizeof(K) * kSortTile + (HasVals ? sizeof(V) * kSortTile : 0) + 4 * (kSortWarps * 256 + 512) <= 48 * 1024,
                "radix scatter tile exceeds static shared memory");
  uint64_t tiles = ceil_div<uint64_t>(n, kSortTile);
  K* src = keys;
  K* dst = keys_alt;
  V* vsrc = vals;
  V* vdst = vals_alt;
  for (int shift = begin_bit; n > 0 && shift < end_bit; shift += 8) {
    if (!(first_hist_ready && shift == begin_bit)) {
      k_radix_hist<K><<<(unsigned)tiles, kSortThreads, 0, st>>>(src, n, shift, (uint32_t)tiles, tmp.hist);
      TB_LAUNCH_CHECK();
    }
    device_scan<uint32_t, OpSum>(tmp.hist, tmp.hist, tiles * 256, true, OpSum{}, 0u, tmp.scan, st);
    k_radix_scatter<K, V, HasVals><<<(unsigned)tiles, kSortThreads, 0, st>>>(src, dst, vsrc, vdst, n, shift,
                                                                             (uint32_t)tiles, tmp.hist);
    TB_LAUNCH_CHECK();
    K* t = src;
    src = dst;
    dst = t;
    V* tv = vsrc;
    vsrc = vdst;
    vdst = tv;
  }
  if (vals_sorted) *vals_sorted = vsrc;
  return src;
}

}  // namespace tb
