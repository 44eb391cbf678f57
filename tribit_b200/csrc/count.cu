// Counting kernels; see count.cuh.
//
// Work unit: a 32-row block of the oriented graph (ranks 32*rb .. 32*rb+31).
// Each variant kernel is persistent (grid = SMs x CTAs/SM) and pulls row
// blocks of its own list, highest rank first, from a device cursor. A row that
// does not fit a warp's shared-memory slice is deferred to a CTA-wide pass,
// and a row too large for that to a global-memory pass, so every row of every
// list is counted exactly once whatever its size.
#include "count.cuh"
#include "scan.cuh"

namespace tb {
namespace {

constexpr uint32_t kFull = 0xffffffffu;
constexpr int kWarpsPerCta = 8;
constexpr int kWarpSlots = 512;                        // 8-byte words of shared memory per warp
constexpr uint32_t kWarpMaxBlocks = kWarpSlots / 2;    // bitmap rows up to this many bit blocks
constexpr uint32_t kWarpMaxList = kWarpSlots * 2;      // merge rows up to this many neighbours
constexpr int kCtaThreads = 512;
constexpr int kCtaLogSlots = 14;                       // 16384 slots = 128 KiB
constexpr uint32_t kCtaMaxBlocks = (1u << kCtaLogSlots) / 2;
constexpr uint64_t kEmptySlot = 0xFFFFFFFF00000000ull;

enum { kCurVariant0 = 0, kCurCta = 4, kCurGlobal = 5 };
enum { kOvfCta = 0, kOvfGlobal = 1 };

__device__ __forceinline__ int log2_ceil(uint32_t x) {  // smallest b with 2^b >= x
  return x <= 1 ? 0 : 32 - __clz(x - 1);
}

__device__ __forceinline__ uint32_t hash_slot(uint32_t blk, int logsz) { return (blk * 0x9E3779B1u) >> (32 - logsz); }

// Open-addressing table of one row's bit blocks: slot = (block << 32) | mask,
// linear probing, at most half full, so every probe sequence ends.
__device__ __forceinline__ void table_clear(uint64_t* tbl, int logsz, int tid, int nthreads) {
  for (int s = tid; s < (1 << logsz); s += nthreads) tbl[s] = kEmptySlot;
}

__device__ __forceinline__ void table_insert(uint64_t* tbl, int logsz, const uint64_t* __restrict__ bent, uint32_t bs,
                                             uint32_t be, int tid, int nthreads) {
  const uint32_t m = (1u << logsz) - 1u;
  for (uint32_t k = bs + tid; k < be; k += nthreads) {
    uint64_t e = bent[k];
    uint32_t h = hash_slot((uint32_t)(e >> 32), logsz);
    while (atomicCAS(reinterpret_cast<unsigned long long*>(tbl + h), kEmptySlot, e) != kEmptySlot) h = (h + 1) & m;
  }
}

__device__ __forceinline__ uint32_t table_find(const uint64_t* tbl, int logsz, uint32_t blk) {
  const uint32_t m = (1u << logsz) - 1u;
  uint32_t h = hash_slot(blk, logsz);
  for (;;) {
    uint64_t x = tbl[h];
    uint32_t k = (uint32_t)(x >> 32);
    if (k == blk) return (uint32_t)x;
    if (k == 0xFFFFFFFFu) return 0u;
    h = (h + 1) & m;
  }
}

// Visits, for the neighbours N+(u)[c] with c in [rs, re) taken in chunks of 32
// (chunk0, chunk0 + step, ...), every item of each neighbour's list -- its bit
// blocks (Blocks) or its neighbour ids -- spreading the flattened items of a
// chunk over the warp's lanes. probe(item_index, neighbour_slot) returns the
// matches it found. Must be called by all 32 lanes.
template <bool Blocks, class Probe>
__device__ __forceinline__ uint64_t sweep(const GraphView& g, uint32_t rs, uint32_t re, uint32_t chunk0,
                                          uint32_t step, Probe&& probe) {
  const uint32_t lane = threadIdx.x & 31;
  uint64_t acc = 0;
  for (uint32_t c = rs + chunk0 * 32; c < re; c += step * 32) {
    uint32_t j = c + lane;
    uint32_t ib = 0, il = 0;
    if (j < re) {
      uint32_t v = g.col[j];
      uint64_t a = g.rp[v], b = g.rp[v + 1];
      if (Blocks) {
        ib = rp_blk(a);
        il = rp_blk(b) - ib;
      } else {
        ib = rp_row(a);
        il = rp_row(b) - ib;
      }
    }
    uint32_t incl = warp_inclusive_sum(il);
    uint32_t total = __shfl_sync(kFull, incl, 31);
    uint32_t excl = incl - il;
    for (uint32_t base = 0; base < total; base += 32) {
      uint32_t t = base + lane;
      uint32_t s = 0;
#pragma unroll
      for (uint32_t st = 16; st >= 1; st >>= 1) {
        uint32_t x = __shfl_sync(kFull, incl, s + st - 1);
        if (x <= t) s += st;
      }
      uint32_t sb = __shfl_sync(kFull, ib, s);
      uint32_t se = __shfl_sync(kFull, excl, s);
      if (t < total) acc += probe(sb + (t - se), c + s);
    }
  }
  return acc;
}

__device__ __forceinline__ void push_row(DeviceStats* stats, int which, uint32_t* list, uint32_t u) {
  uint32_t i = atomicAdd(&stats->overflow[which], 1u);
  list[i] = u;
}

// ---- warp-per-row kernels (bitmap and merge variants) --------------------

template <int V>
__global__ void __launch_bounds__(kWarpsPerCta * 32) k_rows_warp(GraphView g, const uint32_t* __restrict__ list,
                                                                  const uint32_t* __restrict__ list_len,
                                                                  DeviceStats* stats, uint32_t* __restrict__ ovf_cta,
                                                                  unsigned long long* per_graph) {
  __shared__ __align__(16) uint64_t smem[kWarpsPerCta][kWarpSlots];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint64_t* tbl = smem[w];
  uint32_t* lst = reinterpret_cast<uint32_t*>(smem[w]);
  const uint32_t len = list_len[V];
  uint64_t acc = 0;
  for (;;) {
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(&stats->cursor[kCurVariant0 + V], 1u);
    t = __shfl_sync(kFull, t, 0);
    if (t >= len) break;
    const uint32_t rb = list[len - 1 - t];
    const uint32_t u0 = rb * 32, u1 = min(u0 + 32, g.n);
    for (uint32_t u = u0; u < u1; ++u) {
      const uint64_t a = g.rp[u], b = g.rp[u + 1];
      const uint32_t rs = rp_row(a), re = rp_row(b);
      if (re - rs < 2) continue;
      uint64_t racc = 0;
      if (V == TRIBIT_VARIANT_MERGE) {
        const uint32_t d = re - rs;
        if (d > kWarpMaxList) {
          if (lane == 0) push_row(stats, kOvfCta, ovf_cta, u);
          continue;
        }
        for (uint32_t k = lane; k < d; k += 32) lst[k] = g.col[rs + k];
        __syncwarp();
        const uint32_t last = lst[d - 1];
        racc = sweep<false>(g, rs, re, 0, 1, [&](uint32_t k, uint32_t c) -> uint32_t {
          uint32_t x = g.col[k];
          if (x > last) return 0u;
          uint32_t lo = c - rs + 1, hi = d;
          while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (lst[mid] < x)
              lo = mid + 1;
            else
              hi = mid;
          }
          return (lo < d && lst[lo] == x) ? 1u : 0u;
        });
        __syncwarp();
      } else {
        const uint32_t bs = rp_blk(a), be = rp_blk(b), nbu = be - bs;
        if (nbu > kWarpMaxBlocks) {
          if (lane == 0) push_row(stats, kOvfCta, ovf_cta, u);
          continue;
        }
        const int logsz = max(5, log2_ceil(2 * nbu));
        table_clear(tbl, logsz, lane, 32);
        __syncwarp();
        table_insert(tbl, logsz, g.bent, bs, be, lane, 32);
        __syncwarp();
        const uint32_t bmin = (uint32_t)(g.bent[bs] >> 32), bmax = (uint32_t)(g.bent[be - 1] >> 32);
        racc = sweep<true>(g, rs, re, 0, 1, [&](uint32_t k, uint32_t) -> uint32_t {
          uint64_t e = g.bent[k];
          uint32_t blk = (uint32_t)(e >> 32);
          if (blk < bmin || blk > bmax) return 0u;
          return (uint32_t)__popc((uint32_t)e & table_find(tbl, logsz, blk));
        });
        __syncwarp();
      }
      if (per_graph) {
        uint64_t s = warp_sum(racc);
        if (lane == 0 && s) atomicAdd(&per_graph[g.graph_of_rank[u]], (unsigned long long)s);
      }
      acc += racc;
    }
  }
  acc = warp_sum(acc);
  if (lane == 0 && acc) atomicAdd(&stats->triangles, (unsigned long long)acc);
}

// ---- CTA-per-row pass for rows deferred by the warp kernels --------------

__device__ __forceinline__ uint64_t block_sum_u64(uint64_t v) {
  __shared__ unsigned long long part[kCtaThreads / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
  __syncthreads();
  uint64_t s = 0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0ull;
    s = warp_sum(s);
  }
  __syncthreads();
  return s;  // valid in thread 0
}

__global__ void __launch_bounds__(kCtaThreads) k_rows_cta(GraphView g, const uint32_t* __restrict__ rows,
                                                           DeviceStats* stats, uint32_t* __restrict__ ovf_global,
                                                           unsigned long long* per_graph) {
  extern __shared__ __align__(16) uint64_t tbl[];
  __shared__ uint32_t s_t;
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t len = stats->overflow[kOvfCta];
  uint64_t acc = 0;
  for (;;) {
    if (threadIdx.x == 0) s_t = atomicAdd(&stats->cursor[kCurCta], 1u);
    __syncthreads();
    const uint32_t t = s_t;
    __syncthreads();
    if (t >= len) break;
    const uint32_t u = rows[t];
    const uint64_t a = g.rp[u], b = g.rp[u + 1];
    const uint32_t rs = rp_row(a), re = rp_row(b), bs = rp_blk(a), be = rp_blk(b), nbu = be - bs;
    if (nbu > kCtaMaxBlocks) {
      if (threadIdx.x == 0) push_row(stats, kOvfGlobal, ovf_global, u);
      continue;
    }
    const int logsz = max(5, log2_ceil(2 * nbu));
    table_clear(tbl, logsz, threadIdx.x, blockDim.x);
    __syncthreads();
    table_insert(tbl, logsz, g.bent, bs, be, threadIdx.x, blockDim.x);
    __syncthreads();
    const uint32_t bmin = (uint32_t)(g.bent[bs] >> 32), bmax = (uint32_t)(g.bent[be - 1] >> 32);
    uint64_t racc = sweep<true>(g, rs, re, w, nw, [&](uint32_t k, uint32_t) -> uint32_t {
      uint64_t e = g.bent[k];
      uint32_t blk = (uint32_t)(e >> 32);
      if (blk < bmin || blk > bmax) return 0u;
      return (uint32_t)__popc((uint32_t)e & table_find(tbl, logsz, blk));
    });
    if (per_graph) {
      uint64_t s = block_sum_u64(racc);
      if (threadIdx.x == 0 && s) atomicAdd(&per_graph[g.graph_of_rank[u]], (unsigned long long)s);
    } else {
      __syncthreads();  // the table is rebuilt for the next row
    }
    acc += racc;
  }
  (void)lane;
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(&stats->triangles, (unsigned long long)acc);
}

// ---- global-memory pass: any row size, merge by binary search in global ---

__global__ void __launch_bounds__(kCtaThreads) k_rows_global(GraphView g, const uint32_t* __restrict__ rows,
                                                              DeviceStats* stats, unsigned long long* per_graph) {
  __shared__ uint32_t s_t;
  const uint32_t w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t len = stats->overflow[kOvfGlobal];
  uint64_t acc = 0;
  for (;;) {
    if (threadIdx.x == 0) s_t = atomicAdd(&stats->cursor[kCurGlobal], 1u);
    __syncthreads();
    const uint32_t t = s_t;
    __syncthreads();
    if (t >= len) break;
    const uint32_t u = rows[t];
    const uint32_t rs = rp_row(g.rp[u]), re = rp_row(g.rp[u + 1]);
    const uint32_t last = g.col[re - 1];
    uint64_t racc = sweep<false>(g, rs, re, w, nw, [&](uint32_t k, uint32_t c) -> uint32_t {
      uint32_t x = g.col[k];
      if (x > last) return 0u;
      uint32_t lo = c + 1, hi = re;
      while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (g.col[mid] < x)
          lo = mid + 1;
        else
          hi = mid;
      }
      return (lo < re && g.col[lo] == x) ? 1u : 0u;
    });
    if (per_graph) {
      uint64_t s = block_sum_u64(racc);
      if (threadIdx.x == 0 && s) atomicAdd(&per_graph[g.graph_of_rank[u]], (unsigned long long)s);
    }
    acc += racc;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(&stats->triangles, (unsigned long long)acc);
}

// ---- schedule ------------------------------------------------------------

// Row-block features (one warp per row block) and the plain dispatcher's
// choice. Features are log-scaled so the learned dispatcher sees O(1) inputs.
__global__ void k_features(GraphView g, uint32_t nrb, int mode, float* __restrict__ feat,
                           uint8_t* __restrict__ variant_of, int full) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t rb = warp; rb < nrb; rb += nwarps) {
    uint32_t u = rb * 32 + lane;
    uint32_t d = 0, nbu = 0;
    if (u < g.n) {
      uint64_t a = g.rp[u], b = g.rp[u + 1];
      d = rp_row(b) - rp_row(a);
      nbu = rp_blk(b) - rp_blk(a);
    }
    uint32_t active = d >= 2 ? 1u : 0u;
    float fd = (float)d;
    float rows = (float)warp_sum(active);
    float nnz = (float)warp_sum(d);
    float nb = (float)warp_sum(nbu);
    float sq = warp_sum(fd * fd);
    uint32_t dmax = d;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = max(dmax, __shfl_xor_sync(kFull, dmax, o));
    // Neighbour-side work: bit blocks and ids the sweeps will read.
    float wb = 0.f, wm = 0.f, vmax = 0.f, top = 0.f;
    if (full) {
      for (uint32_t r = 0; r < 32; ++r) {
        uint32_t ur = rb * 32 + r;
        if (ur >= g.n) break;
        uint64_t a = g.rp[ur], b = g.rp[ur + 1];
        uint32_t rs = rp_row(a), re = rp_row(b);
        if (re - rs < 2) continue;
        for (uint32_t k = rs + lane; k < re; k += 32) {
          uint32_t v = g.col[k];
          uint64_t va = g.rp[v], vb = g.rp[v + 1];
          float dv = (float)(rp_row(vb) - rp_row(va));
          wb += (float)(rp_blk(vb) - rp_blk(va));
          wm += dv;
          vmax = fmaxf(vmax, dv);
          top += v + 4096u >= g.n ? 1.f : 0.f;
        }
      }
      wb = warp_sum(wb);
      wm = warp_sum(wm);
      top = warp_sum(top);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(kFull, vmax, o));
    }
    if (lane == 0) {
      float* f = feat + (size_t)rb * kNumFeatures;
      float mean = rows > 0 ? nnz / fmaxf(rows, 1.f) : 0.f;
      f[0] = rows / 32.f;
      f[1] = log2f(1.f + nnz);
      f[2] = log2f(1.f + nb);
      f[3] = nb > 0 ? nnz / (32.f * nb) : 0.f;
      f[4] = log2f(1.f + mean);
      f[5] = log2f(1.f + (float)dmax);
      f[6] = log2f(1.f + sqrtf(fmaxf(sq / 32.f - (nnz / 32.f) * (nnz / 32.f), 0.f)));
      f[7] = log2f(1.f + wb);
      f[8] = log2f(1.f + wm);
      f[9] = wb > 0 ? log2f(wm / wb) : 0.f;
      f[10] = log2f(1.f + vmax);
      f[11] = nnz > 0 ? top / nnz : 0.f;
      f[12] = (float)rb * 32.f / fmaxf((float)g.n, 1.f);
      f[13] = log2f(1.f + (float)g.n) / 32.f;
      f[14] = nnz > 0 ? log2f(1.f + wb / nnz) : 0.f;
      f[15] = log2f(1.f + sq);
      uint8_t var;
      if (mode == TRIBIT_DISPATCH_MERGE)
        var = TRIBIT_VARIANT_MERGE;
      else if (mode == TRIBIT_DISPATCH_BITMAP || mode == TRIBIT_DISPATCH_MMA)
        var = TRIBIT_VARIANT_BITMAP;
      else
        var = TRIBIT_VARIANT_BITMAP;
      if (rows == 0.f) var = TRIBIT_VARIANT_MERGE;  // nothing to count; cheapest skip
      variant_of[rb] = var;
    }
  }
}

// Packs (is MMA << 32) | is BITMAP for a scan; merge positions follow.
__global__ void k_variant_flags(const uint8_t* __restrict__ variant_of, uint32_t nrb, uint64_t* __restrict__ flags) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > nrb) return;
  uint64_t f = 0;
  if (i < nrb) {
    uint8_t v = variant_of[i];
    f = (v == TRIBIT_VARIANT_MMA ? (1ull << 32) : 0ull) | (v == TRIBIT_VARIANT_BITMAP ? 1ull : 0ull);
  }
  flags[i] = f;
}

__global__ void k_variant_lists(const uint8_t* __restrict__ variant_of, uint32_t nrb, const uint64_t* __restrict__ pos,
                                uint32_t* l_mma, uint32_t* l_bitmap, uint32_t* l_merge, uint32_t* list_len) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nrb) {
    uint64_t p = pos[i];
    uint32_t pm = (uint32_t)(p >> 32), pb = (uint32_t)p;
    uint8_t v = variant_of[i];
    if (v == TRIBIT_VARIANT_MMA)
      l_mma[pm] = i;
    else if (v == TRIBIT_VARIANT_BITMAP)
      l_bitmap[pb] = i;
    else
      l_merge[i - pm - pb] = i;
  }
  if (i == nrb) {
    uint64_t p = pos[nrb];
    list_len[TRIBIT_VARIANT_MMA] = (uint32_t)(p >> 32);
    list_len[TRIBIT_VARIANT_BITMAP] = (uint32_t)p;
    list_len[TRIBIT_VARIANT_MERGE] = nrb - (uint32_t)(p >> 32) - (uint32_t)p;
  }
}

}  // namespace

Schedule take_schedule(Arena& ar, uint64_t n) {
  Schedule s;
  uint32_t nrb = (uint32_t)ceil_div<uint64_t>(n, 32);
  s.num_row_blocks = nrb;
  s.variant_of = ar.take<uint8_t>(nrb + 1);
  for (int v = 0; v < TRIBIT_NUM_VARIANTS; ++v) s.list[v] = ar.take<uint32_t>(nrb + 1);
  s.list_len = ar.take<uint32_t>(TRIBIT_NUM_VARIANTS);
  s.overflow_cap = (uint32_t)(n + 1);
  s.overflow = ar.take<uint32_t>(2 * (n + 1));
  s.features = ar.take<float>((uint64_t)nrb * kNumFeatures + 1);
  s.flags = reinterpret_cast<uint32_t*>(ar.take<uint64_t>(nrb + 1));
  s.scan_tmp = reinterpret_cast<uint32_t*>(take_scan_temp<uint64_t>(ar, nrb + 1));
  return s;
}

void build_schedule(const GraphView& g, Schedule& s, int mode, const void* /*mlp*/, cudaStream_t st) {
  const uint32_t nrb = s.num_row_blocks;
  if (nrb > 0) {
    unsigned blocks = (unsigned)std::min<uint64_t>(ceil_div<uint64_t>(nrb, 8), 148ull * 16);
    k_features<<<blocks, 256, 0, st>>>(g, nrb, mode, s.features, s.variant_of, 0);
    TB_LAUNCH_CHECK();
  }
  uint64_t* flags = reinterpret_cast<uint64_t*>(s.flags);
  k_variant_flags<<<(unsigned)ceil_div<uint64_t>(nrb + 1, 256), 256, 0, st>>>(s.variant_of, nrb, flags);
  TB_LAUNCH_CHECK();
  device_scan<uint64_t, OpSum>(flags, flags, nrb + 1, true, OpSum{}, 0ull, reinterpret_cast<uint64_t*>(s.scan_tmp), st);
  k_variant_lists<<<(unsigned)ceil_div<uint64_t>(nrb + 1, 256), 256, 0, st>>>(
      s.variant_of, nrb, flags, s.list[TRIBIT_VARIANT_MMA], s.list[TRIBIT_VARIANT_BITMAP], s.list[TRIBIT_VARIANT_MERGE],
      s.list_len);
  TB_LAUNCH_CHECK();
}

LaunchInfo launch_count(const GraphView& g, const Schedule& s, DeviceStats* stats, unsigned long long* per_graph,
                      const CountConfig& cfg, cudaStream_t st) {
  static bool attr_done = false;
  if (!attr_done) {
    TB_CUDA(cudaFuncSetAttribute(k_rows_cta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(uint64_t) << kCtaLogSlots)));
    attr_done = true;
  }
  const int sms = cfg.num_sms > 0 ? cfg.num_sms : 148;
  const int per_sm = cfg.ctas_per_sm > 0 ? cfg.ctas_per_sm : 6;
  const unsigned warp_grid = (unsigned)(sms * per_sm);
  LaunchInfo info;
  uint64_t& ctas = info.ctas;
  TB_CUDA(cudaMemsetAsync(stats->cursor, 0, sizeof(stats->cursor) + sizeof(stats->overflow), st));
  TB_CUDA(cudaMemsetAsync(&stats->triangles, 0, sizeof(stats->triangles), st));
  uint32_t* ovf_cta = s.overflow;
  uint32_t* ovf_global = s.overflow + s.overflow_cap;
  // The MMA list is counted by the bitmap kernel until the tile kernel lands.
  k_rows_warp<TRIBIT_VARIANT_BITMAP><<<warp_grid, kWarpsPerCta * 32, 0, st>>>(
      g, s.list[TRIBIT_VARIANT_BITMAP], s.list_len, stats, ovf_cta, per_graph);
  TB_LAUNCH_CHECK();
  ctas += warp_grid;
  k_rows_warp<TRIBIT_VARIANT_MMA><<<warp_grid, kWarpsPerCta * 32, 0, st>>>(g, s.list[TRIBIT_VARIANT_MMA], s.list_len,
                                                                           stats, ovf_cta, per_graph);
  TB_LAUNCH_CHECK();
  ctas += warp_grid;
  k_rows_warp<TRIBIT_VARIANT_MERGE><<<warp_grid, kWarpsPerCta * 32, 0, st>>>(
      g, s.list[TRIBIT_VARIANT_MERGE], s.list_len, stats, ovf_cta, per_graph);
  TB_LAUNCH_CHECK();
  ctas += warp_grid;
  k_rows_cta<<<(unsigned)sms, kCtaThreads, sizeof(uint64_t) << kCtaLogSlots, st>>>(g, ovf_cta, stats, ovf_global,
                                                                                   per_graph);
  TB_LAUNCH_CHECK();
  ctas += sms;
  k_rows_global<<<(unsigned)sms, kCtaThreads, 0, st>>>(g, ovf_global, stats, per_graph);
  TB_LAUNCH_CHECK();
  ctas += sms;
  info.kernels = 5;
  return info;
}

}  // namespace tb
