// GPU preprocessing pipeline; see prep.cuh.
#include "prep.cuh"
#include "scan.cuh"

namespace tb {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kFull = 0xffffffffu;

inline unsigned grid_for(uint64_t n, int per_thread = 1) {
  uint64_t g = ceil_div<uint64_t>(n, (uint64_t)kThreads * per_thread);
  return (unsigned)(g == 0 ? 1 : g);
}

// Graph of entry i in batch mode: largest g with eoff[g] <= i.
__device__ __forceinline__ uint32_t graph_of_entry(const uint64_t* eoff, uint32_t G, uint64_t i) {
  uint32_t lo = 0, hi = G;  // answer in [0, G)
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (eoff[mid] <= i)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Decodes entry i into global vertex ids. Returns false for an entry naming a
// vertex outside its graph (flagged) and for a self-loop (silently dropped,
// as read_mtx does at tribit.cu:261-267).
__device__ __forceinline__ bool load_entry(const PrepInput& in, uint64_t i, uint32_t& a, uint32_t& b,
                                           unsigned int* err) {
  uint64_t e = in.entries[i];
  uint64_t x = e >> 32, y = e & 0xffffffffull;
  uint64_t base = 0, lim = in.n;
  if (in.G) {
    uint32_t g = graph_of_entry(in.eoff, in.G, i);
    base = in.voff[g];
    lim = in.voff[g + 1] - base;
  }
  if (x >= lim || y >= lim) {
    atomicOr(err, kErrIdRange);
    return false;
  }
  a = (uint32_t)(x + base);
  b = (uint32_t)(y + base);
  return a != b;
}

// The degree order only has to be a good order (any total order counts every
// triangle once): degrees may be counted over every kDegreeSample-th entry
// (a strided sample, which a sorted input does not bias). Every entry is still
// checked for range when it is oriented (k_row_count).
#ifndef TB_DEGREE_SAMPLE
#define TB_DEGREE_SAMPLE 1
#endif
constexpr uint64_t kDegreeSample = TB_DEGREE_SAMPLE;

// Degrees (with duplicates) over the sampled entries of [i0, i1).
__global__ void k_degree(PrepInput in, uint64_t i0, uint64_t i1, uint32_t* __restrict__ deg, unsigned int* err) {
  const uint64_t first = (i0 + kDegreeSample - 1) / kDegreeSample, last = (i1 + kDegreeSample - 1) / kDegreeSample;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = first + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < last; s += stride) {
    uint32_t a, b;
    if (load_entry(in, s * kDegreeSample, a, b, err)) {
      atomicAdd(&deg[a], 1u);
      atomicAdd(&deg[b], 1u);
    }
  }
}

__device__ __forceinline__ uint32_t graph_of_vertex(const uint64_t* voff, uint32_t G, uint64_t v) {
  uint32_t lo = 0, hi = G;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (voff[mid] <= v)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Sort key of vertex v: (graph << dbits) | min(degree, 2^dbits - 1). A stable
// sort of these keys over ids 0..n-1 gives the (graph, degree, id) order.
__global__ void k_vertex_keys(const uint32_t* __restrict__ deg, uint64_t n, const uint64_t* voff, uint32_t G,
                              int dbits, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  uint32_t cap = dbits >= 32 ? 0xffffffffu : ((1u << dbits) - 1u);
  uint32_t d = deg[v] < cap ? deg[v] : cap;
  uint32_t g = G ? graph_of_vertex(voff, G, v) : 0u;
  keys[v] = dbits >= 32 ? d : ((g << dbits) | d);
  vals[v] = (uint32_t)v;
}

__global__ void k_rank_scatter(const uint32_t* __restrict__ sorted_ids, uint64_t n, uint32_t* __restrict__ rank,
                               const uint64_t* voff, uint32_t G, uint32_t* __restrict__ graph_of_rank) {
  uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  uint32_t v = sorted_ids[r];
  rank[v] = (uint32_t)r;
  if (graph_of_rank) graph_of_rank[r] = graph_of_vertex(voff, G, v);
}

__global__ void k_identity_graph_of(uint64_t n, const uint64_t* voff, uint32_t G, uint32_t* __restrict__ graph_of_rank) {
  uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) graph_of_rank[r] = graph_of_vertex(voff, G, r);
}

// ---- phase 2: rows in rank space --------------------------------------------
// Every entry is oriented from its lower-ranked endpoint lo to the higher hi.
// A counting sort by lo (the histogram is the oriented out-degree) places the
// hi's of each row together; each row is then sorted and deduplicated on its
// own (rows are short: with degree order no row exceeds sqrt(2m) entries), and
// one scan of the per-row (distinct neighbours, distinct 32-column blocks)
// pairs gives the CSR and bit-row offsets. The 48-bit global radix sort of
// (lo, hi) keys that this replaces took six passes over all entries.

// Oriented (lo, hi) of entry i in rank space; false for dropped entries.
__device__ __forceinline__ bool orient_entry(const PrepInput& in, const uint32_t* __restrict__ rank, uint64_t i,
                                             uint32_t& lo, uint32_t& hi, unsigned int* err) {
  uint32_t a, b;
  if (!load_entry(in, i, a, b, err)) return false;
  const uint32_t ra = rank ? rank[a] : a, rb = rank ? rank[b] : b;
  lo = ra < rb ? ra : rb;
  hi = ra < rb ? rb : ra;
  return true;
}

// keys[i] = (lo << 32) | hi of entry i (kDropped for a dropped entry), and
// cnt[lo] += 1.
constexpr uint64_t kDropped = ~0ull;
__global__ void k_row_count(PrepInput in, const uint32_t* __restrict__ rank, uint32_t* __restrict__ cnt,
                            uint64_t* __restrict__ keys, unsigned int* err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < in.E; i += stride) {
    uint32_t lo, hi;
    uint64_t key = kDropped;
    if (orient_entry(in, rank, i, lo, hi, err)) {
      atomicAdd(&cnt[lo], 1u);
      key = ((uint64_t)lo << 32) | hi;
    }
    keys[i] = key;
  }
}

// nbr[cur[lo]++] = hi (cur starts as the row offsets): the only random
// accesses are the cursors, which stay in L2.
__global__ void k_row_fill(const uint64_t* __restrict__ keys, uint64_t E, uint32_t* __restrict__ cur,
                           uint32_t* __restrict__ nbr) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += stride) {
    const uint64_t key = keys[i];
    if (key != kDropped) nbr[atomicAdd(&cur[key >> 32], 1u)] = (uint32_t)key;
  }
}

// Slot path (inputs that take the presort, under degree order): row r is
// given a slot of deg(v) entries, v the vertex of rank r (every entry oriented
// from v is one of the deg(v) entries that touch v), so no pass counts the
// rows: cap[r] = deg(v), cap[n] = 0, scanned to the slot starts.
__global__ void k_slot_sizes(const uint32_t* __restrict__ deg, const uint32_t* __restrict__ rank, uint64_t n,
                             uint32_t* __restrict__ cap) {
  const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) cap[rank[v]] = deg[v];
  if (v == n) cap[n] = 0;
}

// Slot path: keys[i] = (lo << 32) | hi of entry i (kDropped for a dropped
// entry), over the presort's radix tiles, each tile also counting its keys'
// presort digits (key >> shift) & 255 into hist (digit-major, as k_radix_hist
// leaves them): the keys and the presort's histogram in one pass.
__global__ void __launch_bounds__(kSortThreads) k_row_keys_hist(PrepInput in, const uint32_t* __restrict__ rank,
                                                                 uint64_t* __restrict__ keys, int shift,
                                                                 uint32_t tiles, uint32_t* __restrict__ hist,
                                                                 unsigned int* err) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll 4
  for (int j = 0; j < kSortKeysPerThread; ++j) {
    const uint64_t i = base + (uint64_t)j * kSortThreads + threadIdx.x;
    uint32_t d = 256u;
    if (i < in.E) {
      uint32_t lo, hi;
      uint64_t key = kDropped;
      if (orient_entry(in, rank, i, lo, hi, err)) key = ((uint64_t)lo << 32) | hi;
      keys[i] = key;
      d = (uint32_t)((key >> shift) & 255);
    }
    const uint32_t peers = __match_any_sync(kFull, d);
    if (d < 256 && (threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&h[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

#ifndef TB_PRESORT_MIN
#define TB_PRESORT_MIN (1ull << 27)
#endif
// Smaller inputs fill straight from the keys: their rows (under 512 MB) keep
// enough of the fill in L2 that the extra pass costs more than it saves
// (measured: RMAT-22 13.3 ms without, 13.6-14.1 with; RMAT-24 50.8 -> 48.6).
constexpr uint64_t kPresortMinEntries = TB_PRESORT_MIN;
constexpr uint32_t kPad = 0xFFFFFFFFu;  // sorts last; no vertex has this rank (n < 2^32)
constexpr uint32_t kWarpSortMax = 1024;  // longer rows are sorted by a CTA
constexpr uint32_t kCtaSortThreads = 1024;
constexpr uint32_t kCtaSortSmem = 8192;  // longer rows are sorted in global scratch

// Bitonic sort of the warp's 32 K values, value r * 32 + lane in x[r] of
// lane lane, ascending.
template <int K>
__device__ __forceinline__ void warp_bitonic(uint32_t (&x)[K]) {
  const uint32_t lane = threadIdx.x & 31;
#pragma unroll
  for (uint32_t k = 2; k <= 32u * K; k <<= 1) {
#pragma unroll
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
        const uint32_t jr = j >> 5;
#pragma unroll
        for (int r = 0; r < K; ++r) {
          if ((r & jr) == 0) {
            const int p = r | (int)jr;
            const bool up = ((r * 32u + lane) & k) == 0;
            const uint32_t a = x[r], b = x[p];
            const bool sw = up ? a > b : a < b;
            x[r] = sw ? b : a;
            x[p] = sw ? a : b;
          }
        }
      } else {
#pragma unroll
        for (int r = 0; r < K; ++r) {
          const uint32_t y = __shfl_xor_sync(kFull, x[r], j);
          const bool up = ((r * 32u + lane) & k) == 0;
          const bool take_min = ((lane & j) == 0) == up;
          x[r] = take_min ? min(x[r], y) : max(x[r], y);
        }
      }
    }
  }
}

// Sorts row a[0, L) (L <= 32 K) with the warp, writes its distinct values
// back to a[0, u) and returns (u << 32) | distinct 32-column blocks.
template <int K>
__device__ __forceinline__ uint64_t warp_sort_row(uint32_t* __restrict__ a, uint32_t L) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t x[K];
#pragma unroll
  for (int r = 0; r < K; ++r) {
    const uint32_t i = r * 32u + lane;
    x[r] = i < L ? a[i] : kPad;
  }
  warp_bitonic<K>(x);
  uint32_t nu = 0, nbk = 0;
  uint32_t last = kPad;  // value 32 r - 1, from the previous register row
#pragma unroll
  for (int r = 0; r < K; ++r) {
    uint32_t prev = __shfl_up_sync(kFull, x[r], 1);
    if (lane == 0) prev = last;
    last = __shfl_sync(kFull, x[r], 31);
    const bool first = r == 0 && lane == 0;
    const bool is_new = x[r] != kPad && (first || x[r] != prev);
    const bool new_blk = is_new && (first || (x[r] >> 5) != (prev >> 5));
    const uint32_t nb = __ballot_sync(kFull, is_new);
    if (is_new) a[nu + __popc(nb & ((1u << lane) - 1u))] = x[r];
    nu += __popc(nb);
    nbk += __popc(__ballot_sync(kFull, new_blk));
  }
  return ((uint64_t)nu << 32) | nbk;
}

// Rows of at most G entries (G = 8, 16 or 32), 32 / G at a time: lane group
// g (lanes [g G, g G + G)) sorts the g-th row of the pass with a bitonic
// network inside the group, then writes the row's distinct values and
// rows[u] = (distinct << 32) | blocks. pending: the warp lanes whose rows
// belong here; lane l's row starts at s_l with L_l entries; u = ubase + l.
template <uint32_t G>
__device__ __forceinline__ void sort_short_rows(uint32_t pending, uint32_t s_l, uint32_t L_l, uint32_t ubase,
                                                uint32_t* __restrict__ nbr, uint64_t* __restrict__ rows) {
  constexpr uint32_t R = 32 / G;
  const uint32_t lane = threadIdx.x & 31, grp = lane / G, gl = lane % G;
  const uint32_t gmask = G == 32 ? kFull : ((1u << G) - 1u) << (grp * G);
  while (pending) {
    int mine = -1;  // the warp lane whose row this group sorts in this pass
#pragma unroll
    for (uint32_t r = 0; r < R; ++r) {
      const int lr = pending ? __ffs(pending) - 1 : -1;
      if (r == grp) mine = lr;
      pending &= pending - 1;
    }
    const uint32_t src = mine >= 0 ? (uint32_t)mine : 0u;
    const uint32_t s = __shfl_sync(kFull, s_l, src), L = __shfl_sync(kFull, L_l, src);
    uint32_t x = mine >= 0 && gl < L ? nbr[s + gl] : kPad;
#pragma unroll
    for (uint32_t k = 2; k <= G; k <<= 1) {
#pragma unroll
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        const uint32_t y = __shfl_xor_sync(kFull, x, j);
        const bool up = (gl & k) == 0;
        x = (((lane & j) == 0) == up) ? min(x, y) : max(x, y);
      }
    }
    const uint32_t prev = __shfl_up_sync(kFull, x, 1);
    const bool first = gl == 0;
    const bool is_new = x != kPad && (first || x != prev);
    const bool new_blk = is_new && (first || (x >> 5) != (prev >> 5));
    const uint32_t nb = __ballot_sync(kFull, is_new) & gmask;
    const uint32_t nbk = __popc(__ballot_sync(kFull, new_blk) & gmask);
    if (is_new) nbr[s + __popc(nb & ((1u << lane) - 1u))] = x;
    if (first && mine >= 0) rows[ubase + mine] = ((uint64_t)__popc(nb) << 32) | nbk;
  }
}

// One warp per 32-row block: rows of up to 8 and 16 entries are sorted four
// and two at a time in lane groups, rows of up to kWarpSortMax one at a time
// in registers; longer rows go to big[] for k_sort_big_rows. Row u holds
// nbr[start[u], end[u]). rows[u] = (distinct << 32) | blocks, rows[n] = 0.
// (Four CTAs of 256 per SM: 64 registers, no spills.)
__global__ void __launch_bounds__(256, 4)
    k_sort_rows(const uint32_t* __restrict__ start, const uint32_t* __restrict__ end, uint32_t n,
                uint32_t* __restrict__ nbr, uint64_t* __restrict__ rows, uint32_t* __restrict__ big,
                uint32_t* __restrict__ nbig) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  if (warp == 0 && lane == 0) rows[n] = 0;
  for (uint32_t ubase = warp * 32; ubase < n; ubase += nwarps * 32) {
    const uint32_t u = ubase + lane;
    const bool here = u < n;
    const uint32_t s_l = here ? start[u] : 0u, L_l = here ? end[u] - s_l : 0u;
    if (here && L_l == 0) rows[u] = 0;
    sort_short_rows<8>(__ballot_sync(kFull, L_l >= 1 && L_l <= 8), s_l, L_l, ubase, nbr, rows);
    sort_short_rows<16>(__ballot_sync(kFull, L_l > 8 && L_l <= 16), s_l, L_l, ubase, nbr, rows);
    sort_short_rows<32>(__ballot_sync(kFull, L_l > 16 && L_l <= 32), s_l, L_l, ubase, nbr, rows);
    uint32_t longer = __ballot_sync(kFull, L_l > 32);
    while (longer) {
      const uint32_t r = __ffs(longer) - 1;
      longer &= longer - 1;
      const uint32_t s = __shfl_sync(kFull, s_l, r), L = __shfl_sync(kFull, L_l, r);
      uint32_t* a = nbr + s;
      uint64_t res;
      if (L <= 64) {
        res = warp_sort_row<2>(a, L);
      } else if (L <= 128) {
        res = warp_sort_row<4>(a, L);
      } else if (L <= 256) {
        res = warp_sort_row<8>(a, L);
      } else if (L <= 512) {
        res = warp_sort_row<16>(a, L);
      } else if (L <= kWarpSortMax) {
        res = warp_sort_row<32>(a, L);
      } else {
        if (lane == 0) big[atomicAdd(nbig, 1u)] = ubase + r;
        continue;
      }
      if (lane == 0) rows[ubase + r] = res;
    }
  }
}

// Rows longer than kWarpSortMax, one CTA per row: a bitonic sort of the row
// padded to a power of two P, in shared memory (P <= kCtaSortSmem) or in the
// row's slice [2 s, 2 s + P) of scratch (P <= 2 L; scratch holds twice the
// entries nbr's row slots hold), then the distinct values written back to the
// front of the row.
__global__ void __launch_bounds__(kCtaSortThreads) k_sort_big_rows(const uint32_t* __restrict__ start,
                                                                   const uint32_t* __restrict__ end,
                                                                   uint32_t* __restrict__ nbr,
                                                                   uint32_t* __restrict__ scratch,
                                                                   uint64_t* __restrict__ rows,
                                                                   const uint32_t* __restrict__ big,
                                                                   const uint32_t* __restrict__ nbig) {
  __shared__ uint32_t sm[kCtaSortSmem];
  __shared__ uint32_t wsum[2][kCtaSortThreads / 32];
  const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t count = *nbig;
  for (uint32_t bi = blockIdx.x; bi < count; bi += gridDim.x) {
    const uint32_t u = big[bi];
    const uint32_t s = start[u], L = end[u] - s;
    uint32_t P = 1;
    while (P < L) P <<= 1;
    uint32_t* a = P <= kCtaSortSmem ? sm : scratch + 2ull * s;
    for (uint32_t i = tid; i < P; i += blockDim.x) a[i] = i < L ? nbr[s + i] : kPad;
    __syncthreads();
    for (uint32_t k = 2; k <= P; k <<= 1) {
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        for (uint32_t t = tid; t < P / 2; t += blockDim.x) {
          const uint32_t i = ((t & ~(j - 1)) << 1) | (t & (j - 1));  // pairs (i, i + j); j is a power of 2
          const bool up = (i & k) == 0;
          const uint32_t x = a[i], y = a[i + j];
          if (up ? x > y : x < y) {
            a[i] = y;
            a[i + j] = x;
          }
        }
        __syncthreads();
      }
    }
    // Distinct values in order: per tile of blockDim values, a block-wide
    // count of the new ones places them.
    uint32_t nu = 0, nbk = 0;
    for (uint32_t base = 0; base < L; base += blockDim.x) {
      const uint32_t i = base + tid;
      const uint32_t x = i < L ? a[i] : kPad;
      const uint32_t p = i > 0 && i < L ? a[i - 1] : kPad;
      const bool is_new = x != kPad && (i == 0 || x != p);
      const bool new_blk = is_new && (i == 0 || (x >> 5) != (p >> 5));
      const uint32_t bn = __ballot_sync(kFull, is_new), bb = __ballot_sync(kFull, new_blk);
      if (lane == 0) {
        wsum[0][w] = __popc(bn);
        wsum[1][w] = __popc(bb);
      }
      __syncthreads();
      uint32_t before = 0, tile_u = 0, tile_b = 0;
      for (uint32_t q = 0; q < blockDim.x / 32; ++q) {
        if (q < w) before += wsum[0][q];
        tile_u += wsum[0][q];
        tile_b += wsum[1][q];
      }
      if (is_new) nbr[s + nu + before + __popc(bn & ((1u << lane) - 1u))] = x;
      nu += tile_u;
      nbk += tile_b;
      __syncthreads();  // a[] reads of this tile and wsum before the next tile
    }
    if (tid == 0) rows[u] = ((uint64_t)nu << 32) | nbk;
    __syncthreads();
  }
}

// The row's distinct sorted values (front of its nbr slice, from off[u]) to col, and its
// bit-row entries (block << 32 | mask) to bent, each written once. One warp
// per 32 rows: a row of at most kLaneEmit values is written by its own lane;
// a longer one by the whole warp, where the mask of a block is a segmented OR
// over the lanes holding its values (a block cut by a chunk boundary carries
// its partial mask over). Most rows of a power-law graph hold 0 or 1 values.
constexpr uint32_t kLaneEmit = 8;
__global__ void k_emit_rows(const uint32_t* __restrict__ off, const uint32_t* __restrict__ nbr,
                            const uint64_t* __restrict__ rp, uint32_t n, uint32_t* __restrict__ col,
                            uint64_t* __restrict__ bent) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t ubase = warp * 32; ubase < n; ubase += nwarps * 32) {
    const uint32_t mu = ubase + lane;
    const bool here = mu < n;
    uint32_t mslot = 0, mnu = 0, mb0 = 0, moff = 0;
    if (here) {
      const uint64_t r0 = rp[mu], r1 = rp[mu + 1];
      mslot = (uint32_t)(r0 >> 32);
      mnu = (uint32_t)(r1 >> 32) - mslot;
      mb0 = (uint32_t)r0;
      moff = mnu ? off[mu] : 0u;
    }
    if (here && mnu <= kLaneEmit && mnu > 0) {
      const uint32_t* a = nbr + moff;
      uint32_t nblk = 0, cur = a[0] >> 5, m = 0;
      for (uint32_t i = 0; i < mnu; ++i) {
        const uint32_t x = a[i];
        col[mslot + i] = x;
        if ((x >> 5) != cur) {
          bent[mb0 + nblk++] = ((uint64_t)cur << 32) | m;
          cur = x >> 5;
          m = 0;
        }
        m |= 1u << (x & 31);
      }
      bent[mb0 + nblk] = ((uint64_t)cur << 32) | m;
    }
    uint32_t longer = __ballot_sync(kFull, here && mnu > kLaneEmit);
    while (longer) {
      const uint32_t r = __ffs(longer) - 1;
      longer &= longer - 1;
      const uint32_t slot = __shfl_sync(kFull, mslot, r), nu = __shfl_sync(kFull, mnu, r),
                     b0 = __shfl_sync(kFull, mb0, r);
      const uint32_t* a = nbr + __shfl_sync(kFull, moff, r);
      // Blocks written so far; the previous chunk's last value and the partial
      // mask of its last block.
      uint32_t nblk = 0, last = kPad, carry = 0;
      for (uint32_t c = 0; c < nu; c += 32) {
        const uint32_t i = c + lane;
        const bool in = i < nu;
        const uint32_t x = in ? a[i] : kPad;
        const uint32_t blk = x >> 5;
        uint32_t prev = __shfl_up_sync(kFull, x, 1);
        if (lane == 0) prev = last;
        uint32_t next = __shfl_down_sync(kFull, x, 1);
        if (lane == 31) next = c + 32 < nu ? a[c + 32] : kPad;
        const bool new_blk = in && (i == 0 || blk != (prev >> 5));
        const bool end_blk = in && (i + 1 == nu || blk != (next >> 5));
        // Segmented OR of the block's bits from its first lane in this chunk.
        uint32_t m = in ? 1u << (x & 31) : 0u;
  #pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(kFull, m, o);
          const uint32_t yb = __shfl_up_sync(kFull, blk, o);
          if (lane >= o && yb == blk) m |= y;
        }
        if (i > 0 && c > 0 && blk == (last >> 5)) m |= carry;  // the block began in the previous chunk
        const uint32_t incl = warp_inclusive_sum(new_blk ? 1u : 0u);
        if (in) col[slot + i] = x;
        if (end_blk) bent[b0 + nblk + incl - 1] = ((uint64_t)blk << 32) | m;
        carry = __shfl_sync(kFull, m, 31);
        last = __shfl_sync(kFull, x, 31);
        nblk += __shfl_sync(kFull, incl, 31);
      }
    }
  }
}

__global__ void k_finalize(const uint64_t* __restrict__ rp, uint64_t n, DeviceStats* stats) {
  const uint64_t tot = rp[n];
  stats->edges = tot >> 32;
  stats->blocks = tot & 0xffffffffull;
}

// Range-relative row starts of rows [s, s + z]: off[k] = cursor[k] =
// row_start[s + k] - row_start[s].
__global__ void k_range_starts(const uint64_t* __restrict__ row_start, uint32_t s, uint32_t z,
                               uint32_t* __restrict__ off, uint32_t* __restrict__ cursor) {
  const uint64_t base = row_start[s];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= z; k += gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)(row_start[s + k] - base);
    off[k] = v;
    cursor[k] = v;
  }
}

// The range's keys into their rows' slots (any order within a row).
__global__ void k_range_fill(const uint64_t* __restrict__ keys, uint64_t cnt, uint32_t s, uint32_t z,
                             const uint32_t* __restrict__ off, uint32_t* __restrict__ cursor,
                             uint32_t* __restrict__ nbr, unsigned int* err) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t key = keys[i];
    const uint32_t r = (uint32_t)(key >> 32) - s;
    if (r >= z) {
      atomicOr(err, kErrInput);
      continue;
    }
    const uint32_t pos = atomicAdd(&cursor[r], 1u);
    if (pos >= off[r + 1]) {
      atomicOr(err, kErrInput);
      continue;
    }
    nbr[pos] = (uint32_t)key;
  }
}

// Every row of the range got exactly its counted entries (a row short of them
// would hold stale slots: the entries changed between passes).
__global__ void k_range_check(const uint32_t* __restrict__ off, const uint32_t* __restrict__ cursor, uint32_t z,
                              unsigned int* err) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < z; k += gridDim.x * blockDim.x)
    if (cursor[k] != off[k + 1]) atomicOr(err, kErrInput);
}

// rp[k] += *carry, k < count: the range's prefix continues the ranges before.
__global__ void k_range_carry(uint64_t* __restrict__ rp, uint32_t count, const uint64_t* __restrict__ carry) {
  const uint64_t c = *carry;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) rp[k] += c;
}

void run_rows(Arena& ar, const PrepInput& in, const uint32_t* rank, const uint32_t* deg, cudaStream_t st,
              Prepared* out, DeviceStats* stats, uint64_t* rp) {
  const uint64_t E = in.E, n = in.n;
  const bool presort = E >= kPresortMinEntries && n > 256;
  // Slot path: with full degrees, rows take degree-sized slots (2E entries
  // in all, u32 offsets) and the keys' presort histogram is counted while they
  // are written: no per-row atomics, no separate histogram pass (RMAT-24:
  // row counts 2.9 ms and the histogram 1.0 ms, for 1 GB more of nbr).
  // (Decided from the order, not from deg: the arena's measuring pass hands
  // out null buffers and must plan the same layout.)
  const bool slots =
      presort && in.order == TRIBIT_ORDER_DEGREE && kDegreeSample == 1 && 2 * E < 0xFFFFFFFFull;
  const uint64_t cap = slots ? 2 * E : E;  // nbr entries
  uint32_t* cnt = ar.take<uint32_t>(n + 1);  // row lengths or slot sizes, then the fill cursors: the row ends
  uint32_t* off = ar.take<uint32_t>(n + 1);  // row starts
  uint32_t* otmp = take_scan_temp<uint32_t>(ar, n + 1);
  uint64_t* rtmp = take_scan_temp<uint64_t>(ar, n + 1);
  uint32_t* big = ar.take<uint32_t>(n + 1);
  uint32_t* nbig = ar.take<uint32_t>(1);
  uint32_t* nbr = ar.take<uint32_t>(cap ? cap : 1);
  // The oriented keys (on the slot path both presort buffers), then long
  // rows' sort space (twice nbr).
  uint32_t* scratch = ar.take<uint32_t>(2 * cap + 2);
  uint64_t* keys_alt = nullptr;
  if (slots)
    keys_alt = reinterpret_cast<uint64_t*>(scratch + 2 * E + 2);
  else if (presort)
    keys_alt = ar.take<uint64_t>(E);
  RadixTemp ktmp;
  if (presort) ktmp = take_radix_temp(ar, E);
  uint32_t* col = ar.take<uint32_t>(E + 4);   // + 4: 16-byte quad loads may read three ids past the end
  uint64_t* bent = ar.take<uint64_t>(E + 2);  // + 2: 16-byte pair loads may read one entry past the end
  out->view.col = col;
  out->view.bent = bent;
  if (ar.measuring()) return;

  const unsigned wgrid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div<uint64_t>(n, 8), 148ull * 32));
  uint64_t* keys = reinterpret_cast<uint64_t*>(scratch);
  const int top = 32 + bits_for(n) - 8;  // the presort digit: the top 8 bits of lo
  TB_CUDA(cudaMemsetAsync(nbig, 0, sizeof(uint32_t), st));
  if (slots) {
    k_slot_sizes<<<grid_for(n + 1), kThreads, 0, st>>>(deg, rank, n, cnt);
    TB_LAUNCH_CHECK();
    device_scan<uint32_t, OpSum>(cnt, off, n + 1, true, OpSum{}, 0u, otmp, st);
    const uint64_t tiles = ceil_div<uint64_t>(E, kSortTile);
    k_row_keys_hist<<<(unsigned)tiles, kSortThreads, 0, st>>>(in, rank, keys, top, (uint32_t)tiles, ktmp.hist,
                                                               &stats->err);
    TB_LAUNCH_CHECK();
  } else {
    TB_CUDA(cudaMemsetAsync(cnt, 0, (n + 1) * sizeof(uint32_t), st));
    if (E > 0) {
      k_row_count<<<grid_for(E, 8), kThreads, 0, st>>>(in, rank, cnt, keys, &stats->err);
      TB_LAUNCH_CHECK();
    }
    device_scan<uint32_t, OpSum>(cnt, off, n + 1, true, OpSum{}, 0u, otmp, st);
  }
  if (E > 0) {
    // One radix pass on the top 8 bits of lo groups the keys into 256 ranges
    // of rows, so the fill's cursors and stores at any time stay in one
    // range's few MB of L2 instead of scattering over all rows.
    const uint64_t* fill_keys = keys;
    if (presort)
      fill_keys = radix_sort<uint64_t, NoVal, false>(keys, keys_alt, nullptr, nullptr, E, top + 8, ktmp, st, nullptr,
                                                     top, slots);
    TB_CUDA(cudaMemcpyAsync(cnt, off, (n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    k_row_fill<<<grid_for(E, 8), kThreads, 0, st>>>(fill_keys, E, cnt, nbr);
    TB_LAUNCH_CHECK();
  }
  // Row u: nbr[off[u], cnt[u]) (with no entries every row is empty: 0, 0).
  k_sort_rows<<<wgrid, kThreads, 0, st>>>(off, cnt, (uint32_t)n, nbr, rp, big, nbig);
  TB_LAUNCH_CHECK();
  if (E > kWarpSortMax) {
    k_sort_big_rows<<<148 * 2, kCtaSortThreads, 0, st>>>(off, cnt, nbr, scratch, rp, big, nbig);
    TB_LAUNCH_CHECK();
  }
  device_scan<uint64_t, OpSum>(rp, rp, n + 1, true, OpSum{}, 0ull, rtmp, st);
  k_emit_rows<<<wgrid, kThreads, 0, st>>>(off, nbr, rp, (uint32_t)n, col, bent);
  TB_LAUNCH_CHECK();
  k_finalize<<<1, 1, 0, st>>>(rp, n, stats);
  TB_LAUNCH_CHECK();
}

}  // namespace

RowRangeBuffers take_row_range_buffers(Arena& ar, uint64_t n, uint64_t cap) {
  RowRangeBuffers b;
  b.keys = ar.take<uint64_t>(cap + 1);
  b.scratch = reinterpret_cast<uint32_t*>(b.keys);
  b.nbr = ar.take<uint32_t>(cap ? cap : 1);
  b.off = ar.take<uint32_t>(n + 1);
  b.cursor = ar.take<uint32_t>(n + 1);
  b.big = ar.take<uint32_t>(n + 1);
  b.nbig = ar.take<uint32_t>(1);
  b.carry = ar.take<uint64_t>(1);
  b.scan_tmp = take_scan_temp<uint64_t>(ar, n + 1);
  return b;
}

void begin_row_range(const RowRangeBuffers& b, const uint64_t* row_start, uint32_t s, uint32_t z, uint64_t* rp,
                     cudaStream_t st) {
  if (z == 0) return;
  // The ranges before this one left rp[s] = the prefix at row s, which the
  // row sort overwrites.
  if (s == 0)
    TB_CUDA(cudaMemsetAsync(b.carry, 0, sizeof(uint64_t), st));
  else
    TB_CUDA(cudaMemcpyAsync(b.carry, rp + s, sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
  TB_CUDA(cudaMemsetAsync(b.nbig, 0, sizeof(uint32_t), st));
  k_range_starts<<<grid_for((uint64_t)z + 1), kThreads, 0, st>>>(row_start, s, z, b.off, b.cursor);
  TB_LAUNCH_CHECK();
}

void finish_row_range(const RowRangeBuffers& b, uint32_t s, uint32_t z, uint64_t cnt, uint64_t* rp, uint32_t* col,
                      uint64_t* bent, unsigned int* err, cudaStream_t st) {
  if (z == 0) return;
  k_range_check<<<grid_for(z), kThreads, 0, st>>>(b.off, b.cursor, z, err);
  TB_LAUNCH_CHECK();
  const unsigned wgrid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div<uint64_t>(z, 8), 148ull * 32));
  k_sort_rows<<<wgrid, kThreads, 0, st>>>(b.off, b.off + 1, z, b.nbr, rp + s, b.big, b.nbig);
  TB_LAUNCH_CHECK();
  if (cnt > kWarpSortMax) {
    k_sort_big_rows<<<148 * 2, kCtaSortThreads, 0, st>>>(b.off, b.off + 1, b.nbr, b.scratch, rp + s, b.big,
                                                         b.nbig);
    TB_LAUNCH_CHECK();
  }
  device_scan<uint64_t, OpSum>(rp + s, rp + s, (uint64_t)z + 1, true, OpSum{}, 0ull, b.scan_tmp, st);
  k_range_carry<<<grid_for((uint64_t)z + 1), kThreads, 0, st>>>(rp + s, z + 1, b.carry);
  TB_LAUNCH_CHECK();
  k_emit_rows<<<wgrid, kThreads, 0, st>>>(b.off, b.nbr, rp + s, z, col, bent);
  TB_LAUNCH_CHECK();
}

void build_row_range(const RowRangeBuffers& b, const uint64_t* row_start, uint32_t s, uint32_t z, uint64_t cnt,
                     uint64_t* rp, uint32_t* col, uint64_t* bent, unsigned int* err, cudaStream_t st) {
  if (z == 0) return;
  begin_row_range(b, row_start, s, z, rp, st);
  if (cnt > 0) {
    k_range_fill<<<grid_for(cnt, 8), kThreads, 0, st>>>(b.keys, cnt, s, z, b.off, b.cursor, b.nbr, err);
    TB_LAUNCH_CHECK();
  }
  finish_row_range(b, s, z, cnt, rp, col, bent, err, st);
}

void finalize_rows(const uint64_t* rp, uint64_t n, DeviceStats* stats, cudaStream_t st) {
  k_finalize<<<1, 1, 0, st>>>(rp, n, stats);
  TB_LAUNCH_CHECK();
}

RankBuffers take_rank_buffers(Arena& ar, uint64_t n) {
  RankBuffers b;
  b.vk = ar.take<uint32_t>(n ? n : 1);
  b.vk2 = ar.take<uint32_t>(n ? n : 1);
  b.vv = ar.take<uint32_t>(n ? n : 1);
  b.vv2 = ar.take<uint32_t>(n ? n : 1);
  b.tmp = take_radix_temp(ar, n);
  return b;
}

void rank_vertices(const uint32_t* deg, uint64_t n, uint64_t E, const RankBuffers& b, uint32_t* rank, cudaStream_t st) {
  if (n == 0) return;
  int dbits = bits_for(2 * E + 2);
  if (dbits > 32) dbits = 32;
  k_vertex_keys<<<grid_for(n), kThreads, 0, st>>>(deg, n, nullptr, 0, 32, b.vk, b.vv);
  TB_LAUNCH_CHECK();
  uint32_t* sorted_ids = nullptr;
  radix_sort<uint32_t, uint32_t, true>(b.vk, b.vk2, b.vv, b.vv2, n, dbits, b.tmp, st, &sorted_ids);
  k_rank_scatter<<<grid_for(n), kThreads, 0, st>>>(sorted_ids, n, rank, nullptr, 0, nullptr);
  TB_LAUNCH_CHECK();
}

void prepare_graph(Arena& ar, const PrepInput& in, cudaStream_t st, Prepared* out) {
  const uint64_t n = in.n, E = in.E;
  if (n > 0xffffffffull || E > 0xfffffffeull)
    throw StatusError(TRIBIT_ERR_TOO_LARGE, "graphs are limited to 2^32-1 vertices and 2^32-2 entries");
  DeviceStats* stats = ar.take<DeviceStats>(1);
  uint64_t* rp = ar.take<uint64_t>(n + 1);
  uint32_t* rank = nullptr;
  uint32_t* graph_of_rank = in.G ? ar.take<uint32_t>(n ? n : 1) : nullptr;
  uint32_t *deg = nullptr, *vk = nullptr, *vk2 = nullptr, *vv = nullptr, *vv2 = nullptr;
  RadixTemp vtmp;
  const bool by_degree = in.order == TRIBIT_ORDER_DEGREE;
  if (by_degree) {
    rank = ar.take<uint32_t>(n ? n : 1);
    deg = ar.take<uint32_t>(n ? n : 1);
    vk = ar.take<uint32_t>(n ? n : 1);
    vk2 = ar.take<uint32_t>(n ? n : 1);
    vv = ar.take<uint32_t>(n ? n : 1);
    vv2 = ar.take<uint32_t>(n ? n : 1);
    vtmp = take_radix_temp(ar, n);
  }
  out->n = n;
  out->E = E;
  out->stats = stats;
  out->rank = rank;
  out->view.n = (uint32_t)n;
  out->view.rp = rp;
  out->view.graph_of_rank = graph_of_rank;
  out->view.eflag = nullptr;

  // Phase 1 (launch only when not measuring): the upload of host entries,
  // degrees and the rank order.
  if (!ar.measuring()) {
    TB_CUDA(cudaMemsetAsync(stats, 0, sizeof(DeviceStats), st));
    const HostUpload& up = in.upload;
    uint64_t* dst = const_cast<uint64_t*>(in.entries);
    const bool upload = up.host && E > 0;
    const bool overlap = upload && by_degree && n > 0;
    auto copy = [&](uint64_t* to, const uint64_t* from, uint64_t words, cudaStream_t s) {
      if (up.stage)
        up.stage(up.stage_ctx, to, from, words * sizeof(uint64_t), s);
      else
        TB_CUDA(cudaMemcpyAsync(to, from, words * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    };
    if (upload && !overlap) copy(dst, up.host, E, st);
    if (upload && !overlap && up.uploaded) TB_CUDA(cudaEventRecord(up.uploaded, st));
    if (by_degree && n > 0) {
      TB_CUDA(cudaMemsetAsync(deg, 0, n * sizeof(uint32_t), st));
      if (overlap) {
        // The copies wait for the stream's earlier work (which may still read
        // the staging buffer); piece k's degree pass waits for piece k.
        TB_CUDA(cudaEventRecord(up.events[0], st));
        TB_CUDA(cudaStreamWaitEvent(up.copy_stream, up.events[0], 0));
        const uint64_t piece = ceil_div<uint64_t>(E, kUploadChunks);
        for (int k = 0; k < kUploadChunks; ++k) {
          const uint64_t i0 = k * piece, i1 = std::min<uint64_t>(E, i0 + piece);
          if (i0 >= i1) break;
          copy(dst + i0, up.host + i0, i1 - i0, up.copy_stream);
          TB_CUDA(cudaEventRecord(up.events[k + 1], up.copy_stream));
          TB_CUDA(cudaStreamWaitEvent(st, up.events[k + 1], 0));
          if (i1 == E && up.uploaded) TB_CUDA(cudaEventRecord(up.uploaded, st));
          k_degree<<<grid_for(i1 - i0, 8), kThreads, 0, st>>>(in, i0, i1, deg, &stats->err);
          TB_LAUNCH_CHECK();
        }
      } else if (E > 0) {
        k_degree<<<grid_for(E, 8), kThreads, 0, st>>>(in, 0, E, deg, &stats->err);
        TB_LAUNCH_CHECK();
      }
      int gbits = in.G ? bits_for((uint64_t)in.G) : 0;
      int dbits = bits_for(2 * E + 2);
      if (dbits > 32 - gbits) dbits = 32 - gbits;
      k_vertex_keys<<<grid_for(n), kThreads, 0, st>>>(deg, n, in.voff, in.G, in.G ? dbits : 32, vk, vv);
      TB_LAUNCH_CHECK();
      uint32_t* sorted_ids = nullptr;
      radix_sort<uint32_t, uint32_t, true>(vk, vk2, vv, vv2, n, in.G ? gbits + dbits : dbits, vtmp, st, &sorted_ids);
      k_rank_scatter<<<grid_for(n), kThreads, 0, st>>>(sorted_ids, n, rank, in.voff, in.G, graph_of_rank);
      TB_LAUNCH_CHECK();
    } else if (in.G && n > 0) {
      k_identity_graph_of<<<grid_for(n), kThreads, 0, st>>>(n, in.voff, in.G, graph_of_rank);
      TB_LAUNCH_CHECK();
    }
  }
  // Phase 2: orient, rows, sort + dedup per row, CSR + bit rows.
  run_rows(ar, in, rank, deg, st, out, stats, rp);
}

}  // namespace tb
