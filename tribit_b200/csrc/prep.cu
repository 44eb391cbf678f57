// GPU preprocessing pipeline; see prep.cuh.
#include "prep.cuh"
#include "scan.cuh"

namespace tb {
namespace {

constexpr int kThreads = 256;

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

__global__ void k_degree(PrepInput in, uint32_t* __restrict__ deg, unsigned int* err) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (; i < in.E; i += stride) {
    uint32_t a, b;
    if (load_entry(in, i, a, b, err)) {
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

// Oriented key (lo << B) | hi in rank space; invalid entries and self-loops
// become the all-ones sentinel, which sorts last and is dropped.
template <typename K>
__global__ void k_orient(PrepInput in, const uint32_t* __restrict__ rank, int B, K* __restrict__ keys,
                         unsigned int* err) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const K sentinel = (K)(((unsigned __int128)1 << (2 * B)) - 1);
  for (; i < in.E; i += stride) {
    uint32_t a, b;
    K key = sentinel;
    if (load_entry(in, i, a, b, err)) {
      uint32_t ra = rank ? rank[a] : a, rb = rank ? rank[b] : b;
      uint32_t lo = ra < rb ? ra : rb, hi = ra < rb ? rb : ra;
      key = ((K)lo << B) | (K)hi;
    }
    keys[i] = key;
  }
}

// flags[i] = (first of a distinct key << 32) | (first of a distinct
// (row, 32-column block)), flags[E] = 0; an exclusive scan then gives every
// distinct edge its CSR slot and every bit-row entry its slot.
template <typename K>
__global__ void k_unique_flags(const K* __restrict__ keys, uint64_t E, int B, uint64_t* __restrict__ flags) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > E) return;
  if (i == E) {
    flags[E] = 0;
    return;
  }
  const K sentinel = (K)(((unsigned __int128)1 << (2 * B)) - 1);
  K k = keys[i];
  uint64_t f = 0;
  if (k != sentinel) {
    K p = i ? keys[i - 1] : sentinel;
    bool is_new = (i == 0) || p != k;
    if (is_new) {
      const K mask = ((K)1 << B) - 1;
      bool new_blk = (i == 0) || (p >> B) != (k >> B) || ((p & mask) >> 5) != ((k & mask) >> 5);
      f = (1ull << 32) | (new_blk ? 1ull : 0ull);
    }
  }
  flags[i] = f;
}

template <typename K>
__global__ void k_unique_scatter(const K* __restrict__ keys, uint64_t E, int B, const uint64_t* __restrict__ pos,
                                 uint32_t* __restrict__ col, uint64_t* __restrict__ bent, uint64_t* __restrict__ rp) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= E) return;
  uint64_t p0 = pos[i], p1 = pos[i + 1];
  uint32_t is_new = (uint32_t)((p1 >> 32) - (p0 >> 32));
  if (!is_new) return;
  uint32_t new_blk = (uint32_t)(p1 - p0) & 1u;  // low halves never carry
  const K mask = ((K)1 << B) - 1;
  K k = keys[i];
  uint32_t row = (uint32_t)(k >> B), hi = (uint32_t)(k & mask);
  uint32_t slot = (uint32_t)(p0 >> 32);
  uint32_t bidx = (uint32_t)p0 + new_blk - 1u;
  col[slot] = hi;
  uint32_t* bw = reinterpret_cast<uint32_t*>(bent + bidx);
  if (new_blk) bw[1] = hi >> 5;
  atomicOr(&bw[0], 1u << (hi & 31));
  bool row_first = (i == 0) || (uint32_t)(keys[i - 1] >> B) != row;
  if (row_first) rp[row] = ((uint64_t)slot << 32) | bidx;
}

__global__ void k_finalize(const uint64_t* __restrict__ pos, uint64_t E, uint64_t n, uint64_t* __restrict__ rp,
                           DeviceStats* stats) {
  uint64_t tot = pos[E];
  rp[n] = tot;
  stats->edges = tot >> 32;
  stats->blocks = tot & 0xffffffffull;
}

template <typename K>
void run_edges(Arena& ar, const PrepInput& in, const uint32_t* rank, int B, cudaStream_t st, Prepared* out,
               DeviceStats* stats, uint64_t* rp) {
  const uint64_t E = in.E, n = in.n;
  K* keys = ar.take<K>(E ? E : 1);
  K* keys_alt = ar.take<K>(E ? E : 1);
  RadixTemp etmp = take_radix_temp(ar, E);
  uint64_t* pos = ar.take<uint64_t>(E + 1);
  uint64_t* ptmp = take_scan_temp<uint64_t>(ar, E + 1);
  uint32_t* col = ar.take<uint32_t>(E ? E : 1);
  uint64_t* bent = ar.take<uint64_t>(E + 2);  // + 2: 16-byte pair loads may read one entry past the end
  uint64_t* rtmp = take_scan_temp<uint64_t>(ar, n + 1);
  out->view.col = col;
  out->view.bent = bent;
  if (ar.measuring()) return;

  TB_CUDA(cudaMemsetAsync(rp, 0xff, (n + 1) * sizeof(uint64_t), st));
  if (E > 0) {
    TB_CUDA(cudaMemsetAsync(bent, 0, E * sizeof(uint64_t), st));
    k_orient<K><<<grid_for(E, 8), kThreads, 0, st>>>(in, rank, B, keys, &stats->err);
    TB_LAUNCH_CHECK();
    K* sorted = radix_sort<K, NoVal, false>(keys, keys_alt, nullptr, nullptr, E, 2 * B, etmp, st, nullptr);
    k_unique_flags<K><<<grid_for(E + 1), kThreads, 0, st>>>(sorted, E, B, pos);
    TB_LAUNCH_CHECK();
    device_scan<uint64_t, OpSum>(pos, pos, E + 1, true, OpSum{}, 0ull, ptmp, st);
    k_unique_scatter<K><<<grid_for(E), kThreads, 0, st>>>(sorted, E, B, pos, col, bent, rp);
    TB_LAUNCH_CHECK();
  } else {
    TB_CUDA(cudaMemsetAsync(pos, 0, sizeof(uint64_t), st));
  }
  k_finalize<<<1, 1, 0, st>>>(pos, E, n, rp, stats);
  TB_LAUNCH_CHECK();
  // Rows without edges take the start of the next row that has one.
  device_scan<uint64_t, OpMin, true>(rp, rp, n + 1, false, OpMin{}, ~0ull, rtmp, st);
}

}  // namespace

void prepare_graph(Arena& ar, const PrepInput& in, cudaStream_t st, Prepared* out) {
  const uint64_t n = in.n, E = in.E;
  if (n > 0xffffffffull || E > 0xfffffffeull)
    throw StatusError(TRIBIT_ERR_TOO_LARGE, "graphs are limited to 2^32-1 vertices and 2^32-2 entries");
  const int B = bits_for(n ? n : 1);
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

  // Phase 1 (launch only when not measuring): degrees and the rank order.
  if (!ar.measuring()) {
    TB_CUDA(cudaMemsetAsync(stats, 0, sizeof(DeviceStats), st));
    if (by_degree && n > 0) {
      TB_CUDA(cudaMemsetAsync(deg, 0, n * sizeof(uint32_t), st));
      if (E > 0) {
        k_degree<<<grid_for(E, 8), kThreads, 0, st>>>(in, deg, &stats->err);
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
  // Phase 2: orient, sort, dedup, CSR + bit rows.
  if (2 * B <= 32)
    run_edges<uint32_t>(ar, in, rank, B, st, out, stats, rp);
  else
    run_edges<uint64_t>(ar, in, rank, B, st, out, stats, rp);
}

}  // namespace tb
