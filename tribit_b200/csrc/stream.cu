// Counting graphs whose buffers exceed the device's memory (or the context's
// device budget): tribit_count_edges on host entries, in rank ranges.
//
// The reference splits a graph too large for one GPU into partitions of
// block_size vertices and tasks of at most 1e9 entries
// (src/multi_gpu/src/main.rs:98-220), on several GPUs. Here the graph is
// counted on one GPU in pieces, and no triangle is counted twice:
//
//   T = sum over u of sum over v in N+(u) of |N+(u) & N+(v)|
//     = sum over i <= j of T(i, j), where u ranges over rank range R_i and
//       v over R_j (v > u, so j >= i).
//
// Phase 1 streams the host entries through the GPU three times in 32 MiB
// pieces, so it needs device memory per vertex only: degrees; each oriented
// entry's lower endpoint, counted per row; then each entry's oriented key
// (lo << 32 | hi, in rank space), sent back to a host bucket per rank range.
// The ranges are contiguous in rank and hold at most `cap` entries each.
//
// Phase 2 counts every pair i <= j as an ordinary graph in id order, on the
// device, with the same preprocessing and counting kernels as any count:
//   - i == j: bucket i with every id moved down by the start of R_i: T(i, i).
//   - i < j: three id spaces, in this order: A, a copy of every row u of R_i;
//     V, the rows of R_j; W, every vertex from the start of R_i on, with no
//     row. A copy lists its neighbours as W ids, and its neighbours in R_j
//     also as V ids; a row of R_j lists its neighbours as W ids. A W id has an
//     empty row, so only the (copy of u, V id of v) edges count, each
//     |N+(u) & N+(v)| over W ids: the count is T(i, j).
// Duplicated entries share their lower endpoint and so their bucket, where
// the task's own deduplication removes them; the undirected edge count is the
// sum of the diagonal tasks' edges.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "context.h"

namespace tb {
namespace {

constexpr int kThreads = 256;
constexpr uint64_t kPieceWords = (32u << 20) / sizeof(uint64_t);  // entries of one pinned buffer
constexpr uint32_t kMaxRanges = 1023;                              // one CTA computes the bounds
// Rows tier: up to this many ranges are each filled from one more pass over
// the host entries (pinned, copied as they are; pageable, through host
// copies to the staging buffers); more go through host buckets (one pass,
// keys back and up).
constexpr uint64_t kDirectRangesPinned = 4;
constexpr uint64_t kDirectRangesPageable = 2;
constexpr uint64_t kNoKey = ~0ull;
static_assert(kUploadChunks + 1 >= 5, "the piece streaming uses five upload events");

inline unsigned grid_for(uint64_t n) {
  const uint64_t g = ceil_div<uint64_t>(n, (uint64_t)kThreads * 8);
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 64));
}

// Entry e of a graph of n vertices: false for a self-loop, and for an id
// >= n (flagged).
__device__ __forceinline__ bool entry_ids(uint64_t e, uint64_t n, uint32_t& a, uint32_t& b, unsigned int* err) {
  const uint64_t x = e >> 32, y = e & 0xffffffffull;
  if (x >= n || y >= n) {
    atomicOr(err, kErrIdRange);
    return false;
  }
  a = (uint32_t)x;
  b = (uint32_t)y;
  return a != b;
}

__global__ void k_s_degree(const uint64_t* __restrict__ e, uint64_t cnt, uint64_t n, uint32_t* __restrict__ deg,
                           unsigned int* err) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a, b;
    if (entry_ids(e[i], n, a, b, err)) {
      atomicAdd(&deg[a], 1u);
      atomicAdd(&deg[b], 1u);
    }
  }
}

__global__ void k_s_rows(const uint64_t* __restrict__ e, uint64_t cnt, uint64_t n, const uint32_t* __restrict__ rank,
                         uint32_t* __restrict__ rows, unsigned int* err) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a, b;
    if (entry_ids(e[i], n, a, b, err)) atomicAdd(&rows[min(rank[a], rank[b])], 1u);
  }
}

// off[i] = rows[i] (widened for the prefix), max_row = the longest row.
__global__ void k_s_widen(const uint32_t* __restrict__ rows, uint64_t cnt, uint64_t* __restrict__ off,
                          unsigned int* max_row) {
  uint32_t m = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
    off[i] = rows[i];
    m = max(m, rows[i]);
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0 && m) atomicMax(max_row, m);
}

// off: exclusive prefix of the row entries (n + 1). bounds[k] = first row
// whose prefix reaches k * step (k < P; bounds[0] = 0), bounds[P] = n;
// size[k] = entries of range k. One CTA of at least P + 1 threads.
__global__ void k_s_bounds(const uint64_t* __restrict__ off, uint64_t n, uint64_t step, uint32_t P,
                           uint32_t* __restrict__ bounds, uint64_t* __restrict__ size) {
  const uint32_t k = threadIdx.x;
  if (k <= P) {
    uint64_t b = n;
    if (k == 0) {
      b = 0;
    } else if (k < P) {
      const uint64_t target = (uint64_t)k * step;
      uint64_t lo = 0, hi = n;
      while (lo < hi) {
        const uint64_t mid = lo + ((hi - lo) >> 1);
        if (off[mid] < target)
          lo = mid + 1;
        else
          hi = mid;
      }
      b = lo;
    }
    bounds[k] = (uint32_t)b;
  }
  __syncthreads();
  if (k < P) size[k] = off[bounds[k + 1]] - off[bounds[k]];
}

__device__ __forceinline__ uint32_t range_of(const uint32_t* bounds, uint32_t P, uint32_t lo) {
  uint32_t a = 0, b = P;  // last k < P with bounds[k] <= lo
  while (b - a > 1) {
    const uint32_t m = (a + b) >> 1;
    if (bounds[m] <= lo)
      a = m;
    else
      b = m;
  }
  return a;
}

// Oriented key and range of every entry of the piece; hist[range] += 1.
__global__ void k_s_keys(const uint64_t* __restrict__ e, uint64_t cnt, uint64_t n, const uint32_t* __restrict__ rank,
                         const uint32_t* __restrict__ bounds, uint32_t P, uint64_t* __restrict__ keys,
                         uint32_t* __restrict__ rng, uint32_t* __restrict__ hist, unsigned int* err) {
  extern __shared__ uint32_t sh[];  // bounds (P + 1), then the CTA's histogram (P)
  for (uint32_t k = threadIdx.x; k <= P; k += blockDim.x) sh[k] = bounds[k];
  for (uint32_t k = threadIdx.x; k < P; k += blockDim.x) sh[P + 1 + k] = 0u;
  __syncthreads();
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a, b;
    uint64_t key = kNoKey;
    uint32_t r = 0;
    if (entry_ids(e[i], n, a, b, err)) {
      const uint32_t ra = rank[a], rb = rank[b];
      const uint32_t lo = min(ra, rb), hi = max(ra, rb);
      key = ((uint64_t)lo << 32) | hi;
      r = range_of(sh, P, lo);
      atomicAdd(&sh[P + 1 + r], 1u);
    }
    keys[i] = key;
    rng[i] = r;
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < P; k += blockDim.x)
    if (sh[P + 1 + k]) atomicAdd(&hist[k], sh[P + 1 + k]);
}

// Groups the piece's keys by range: cursor[r] starts at range r's first slot.
__global__ void k_s_scatter(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ rng, uint64_t cnt,
                            uint32_t* __restrict__ cursor, uint64_t* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t key = keys[i];
    if (key != kNoKey) out[atomicAdd(&cursor[rng[i]], 1u)] = key;
  }
}

// Rows tier, direct fill of rank range [s, s + z): every entry of the piece
// whose lower endpoint's rank falls in the range goes to a slot of its row
// (the range's keys never exist as such).
__global__ void k_s_fill(const uint64_t* __restrict__ e, uint64_t cnt, uint64_t n, const uint32_t* __restrict__ rank,
                         uint32_t s, uint32_t z, const uint32_t* __restrict__ off, uint32_t* __restrict__ cursor,
                         uint32_t* __restrict__ nbr, unsigned int* err) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a, b;
    if (!entry_ids(e[i], n, a, b, err)) continue;
    const uint32_t ra = rank[a], rb = rank[b];
    const uint32_t r = min(ra, rb) - s;
    if (r >= z) continue;
    const uint32_t pos = atomicAdd(&cursor[r], 1u);
    if (pos < off[r + 1])
      nbr[pos] = max(ra, rb);
    else
      atomicOr(err, kErrInput);
  }
}

// Diagonal task: every rank r >= s becomes r - s.
__global__ void k_s_diag(uint64_t* __restrict__ w, uint64_t cnt, uint32_t s) {
  const uint64_t d = ((uint64_t)s << 32) | s;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += (uint64_t)gridDim.x * blockDim.x)
    w[k] -= d;
}

// Off-diagonal task (i < j) in place over w = [bucket i (ci) | bucket j (cj) |
// room for ci more]: A(x) = x - si, V(x) = zi + x - sj, W(x) = zi + zj + x - si
// (si, zi: start and size of R_i; sj, zj of R_j). Bucket i's (lo, hi) becomes
// (A lo, W hi), plus (A lo, V hi) appended when hi is in R_j; bucket j's
// (lo, hi) becomes (V lo, W hi). *extra receives the appended count.
__global__ void k_s_pair(uint64_t* __restrict__ w, uint64_t ci, uint64_t cj, uint32_t si, uint32_t zi, uint32_t sj,
                         uint32_t zj, unsigned long long* extra) {
  const uint64_t cnt = ci + cj;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t x = w[k];
    const uint32_t lo = (uint32_t)(x >> 32), hi = (uint32_t)x;
    const uint32_t whi = zi + zj + (hi - si);
    if (k < ci) {
      const uint32_t alo = lo - si;
      w[k] = ((uint64_t)alo << 32) | whi;
      if (hi >= sj && hi - sj < zj) w[cnt + atomicAdd(extra, 1ull)] = ((uint64_t)alo << 32) | (zi + (hi - sj));
    } else {
      w[k] = ((uint64_t)(zi + (lo - sj)) << 32) | whi;
    }
  }
}

// Multi-threaded host copy (page faults of pageable memory dominate).
void host_copy(void* dst, const void* src, size_t bytes) {
  const int nt = (int)std::max<size_t>(1, std::min<size_t>(8, bytes >> 22));
  if (nt == 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  std::vector<std::thread> th;
  const size_t share = (bytes + nt - 1) / nt;
  for (int k = 0; k < nt; ++k) {
    const size_t a = std::min(bytes, k * share), b = std::min(bytes, a + share);
    if (a < b) th.emplace_back([=] { std::memcpy((char*)dst + a, (const char*)src + a, b - a); });
  }
  for (auto& x : th) x.join();
}

void ensure_pinned(tribit_context* c) {
  if (!c->pinned[0])
    for (auto& p : c->pinned) TB_CUDA(cudaMallocHost(&p, kPieceWords * sizeof(uint64_t)));
}

// The device memory a call may use: the context's budget, else what is free
// now plus the context's own reservations (reusable), minus 1 GiB.
uint64_t budget_bytes(tribit_context* c) {
  if (c->device_budget) return c->device_budget;
  size_t fr = 0, tot = 0;
  TB_CUDA(cudaMemGetInfo(&fr, &tot));
  const uint64_t own = c->arena.capacity() + c->stream_arena.capacity();
  const uint64_t margin = 1ull << 30;
  return fr + own > margin ? fr + own - margin : 0;
}

float ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
}


// Host entries streamed through two device piece buffers: pass(fn) calls
// fn(piece, count) per piece on the context's stream. Pinned host entries are
// copied straight from the caller's buffer on the copy stream, piece k + 1
// while piece k's work runs; pageable ones through the context's pinned
// buffers, the host copy of piece k + 1 while piece k's copy and work run.
struct PieceStream {
  tribit_context* c = nullptr;
  const uint64_t* host = nullptr;
  uint64_t E = 0, piece_words = 0;
  bool pinned_src = false;
  uint64_t* pieces[2] = {nullptr, nullptr};

  uint64_t size(uint64_t k) const { return std::min<uint64_t>(piece_words, E - k * piece_words); }
  // Pinned source: upload_ev[1 + b]: buffer b's work done; upload_ev[3 + b]:
  // buffer b's copy done.
  void issue_copy(uint64_t k) const {
    const int b = (int)(k & 1);
    if (k >= 2) TB_CUDA(cudaStreamWaitEvent(c->copy_st, c->upload_ev[1 + b], 0));
    TB_CUDA(cudaMemcpyAsync(pieces[b], host + k * piece_words, size(k) * sizeof(uint64_t), cudaMemcpyHostToDevice,
                            c->copy_st));
    TB_CUDA(cudaEventRecord(c->upload_ev[3 + b], c->copy_st));
  }
  template <typename Fn>
  void pass(Fn&& fn) const {
    cudaStream_t st = c->st;
    const uint64_t npieces = ceil_div<uint64_t>(E, piece_words);
    if (pinned_src) {  // the copies follow all earlier work on the stream
      TB_CUDA(cudaEventRecord(c->upload_ev[0], st));
      TB_CUDA(cudaStreamWaitEvent(c->copy_st, c->upload_ev[0], 0));
      if (npieces) issue_copy(0);
    }
    for (uint64_t k = 0; k < npieces; ++k) {
      const uint64_t cnt = size(k);
      const int b = (int)(k & 1);
      if (pinned_src) {
        if (k + 1 < npieces) issue_copy(k + 1);
        TB_CUDA(cudaStreamWaitEvent(st, c->upload_ev[3 + b], 0));
        fn(static_cast<const uint64_t*>(pieces[b]), cnt);
        TB_CUDA(cudaEventRecord(c->upload_ev[1 + b], st));
      } else {
        void* pin = c->pinned[b];
        pinned_wait(c, b);
        host_copy(pin, host + k * piece_words, cnt * sizeof(uint64_t));
        TB_CUDA(cudaMemcpyAsync(pieces[b], pin, cnt * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        pinned_used(c, b, st);
        fn(static_cast<const uint64_t*>(pieces[b]), cnt);
      }
    }
  }
};

}  // namespace

bool host_is_pinned(const void* p) {
  cudaPointerAttributes pa{};
  const bool pinned = cudaPointerGetAttributes(&pa, p) == cudaSuccess && pa.type == cudaMemoryTypeHost;
  (void)cudaGetLastError();
  return pinned;
}

void stage_pageable(void* ctx, void* dst, const void* src, size_t bytes, cudaStream_t st) {
  tribit_context* c = static_cast<tribit_context*>(ctx);
  ensure_pinned(c);
  const size_t piece = kPieceWords * sizeof(uint64_t);
  for (size_t at = 0; at < bytes; at += piece) {
    const size_t len = std::min(piece, bytes - at);
    const int b = c->pinned_turn;
    c->pinned_turn ^= 1;
    pinned_wait(c, b);
    host_copy(c->pinned[b], (const char*)src + at, len);
    TB_CUDA(cudaMemcpyAsync((char*)dst + at, c->pinned[b], len, cudaMemcpyHostToDevice, st));
    pinned_used(c, b, st);
  }
}

void upload_via_pinned(tribit_context* c, const void* src, size_t bytes, void* dst) {
  ensure_pinned(c);
  const size_t piece = kPieceWords * sizeof(uint64_t);
  TB_CUDA(cudaEventRecord(c->upload_ev[0], c->st));
  TB_CUDA(cudaStreamWaitEvent(c->copy_st, c->upload_ev[0], 0));
  uint64_t k = 0;
  for (size_t at = 0; at < bytes; at += piece, ++k) {
    const size_t len = std::min(piece, bytes - at);
    const int b = (int)(k & 1);
    pinned_wait(c, b);
    host_copy(c->pinned[b], (const char*)src + at, len);
    TB_CUDA(cudaMemcpyAsync((char*)dst + at, c->pinned[b], len, cudaMemcpyHostToDevice, c->copy_st));
    pinned_used(c, b, c->copy_st);
  }
  TB_CUDA(cudaEventRecord(c->upload_ev[3], c->copy_st));
  TB_CUDA(cudaStreamWaitEvent(c->st, c->upload_ev[3], 0));
}

namespace {

// The rows tier's device layout: the oriented graph's rows (kept), then what
// only the build uses -- the row starts, the rank of every vertex and two
// piece buffers (for ranges filled straight from the streamed entries), one
// range's build buffers -- and over those (dead once the rows are built) the
// counting schedule. Returns the arena bytes.
struct RowsLayout {
  DeviceStats* stats = nullptr;
  uint64_t* rp = nullptr;
  uint32_t* col = nullptr;
  uint64_t* bent = nullptr;
  uint64_t* row_start = nullptr;
  uint32_t* rank = nullptr;
  uint64_t* pieces[2] = {nullptr, nullptr};
  RowRangeBuffers build;
  Schedule sched;
};

size_t rows_layout(Arena& ar, bool measure, uint64_t n, uint64_t kept, uint64_t cap, bool hubs, uint64_t piece_words,
                   RowsLayout* L) {
  ar.begin(measure);
  L->stats = ar.take<DeviceStats>(1);
  L->rp = ar.take<uint64_t>(n + 1);
  L->col = ar.take<uint32_t>(kept + 4);  // + 4: 16-byte quad loads may read three ids past the end
  L->bent = ar.take<uint64_t>(kept + 2);  // + 2: 16-byte pair loads may read one entry past the end
  const size_t rows_end = ar.used();
  L->row_start = ar.take<uint64_t>(n + 1);
  L->rank = ar.take<uint32_t>(n);
  L->pieces[0] = ar.take<uint64_t>(piece_words);
  L->pieces[1] = ar.take<uint64_t>(piece_words);
  L->build = take_row_range_buffers(ar, n, cap);
  const size_t build_end = ar.used();
  ar.rewind(rows_end);
  L->sched = take_schedule(ar, n, kept, hubs);
  return std::max(build_end, ar.used());
}

struct RowsPlan {
  uint64_t cap = 0;   // entries of a range's build buffers
  bool hubs = true;   // the schedule holds the hub pass's in-lists
};

// The largest range the budget allows, with the hub in-lists if they fit
// (the merge blocks count without them, more slowly). False when not even a
// range of the longest row fits.
bool plan_rows(Arena& ar, uint64_t n, uint64_t kept, uint32_t max_row, uint64_t budget, uint64_t piece_words,
               RowsPlan* plan) {
  RowsLayout L;
  const uint64_t lo = std::min<uint64_t>(kept, (uint64_t)max_row + 1);
  for (bool hubs : {true, false}) {
    if (rows_layout(ar, true, n, kept, lo, hubs, piece_words, &L) > budget) continue;
    uint64_t a = lo, b = kept;  // the largest cap in [a, b] that fits
    while (a < b) {
      const uint64_t m = b - (b - a) / 2;
      if (rows_layout(ar, true, n, kept, m, hubs, piece_words, &L) <= budget)
        a = m;
      else
        b = m - 1;
    }
    plan->cap = a;
    plan->hubs = hubs;
    return true;
  }
  return false;
}

}  // namespace

// Where the rows tier's ranges come from: host buckets of oriented keys, one
// per range, or the host entries streamed once more per range.
struct RowsSource {
  const std::vector<std::unique_ptr<uint64_t[]>>* bucket = nullptr;  // null: streamed
  const PieceStream* stream = nullptr;
};

// Host copies of phase 1's row starts (n + 1) and ranks (n) for phase 2: the
// context's pinned buffer, kept for later calls (copied straight both ways),
// or pageable memory when that cannot be had.
struct CarryHost {
  uint64_t* off = nullptr;
  uint32_t* rank = nullptr;
  bool pinned = false;
  std::vector<uint64_t> off_v;
  std::vector<uint32_t> rank_v;
};

void carry_host(tribit_context* c, uint64_t n, CarryHost* h) {
  const size_t bytes = (n + 1) * sizeof(uint64_t) + n * sizeof(uint32_t);
  if (c->stream_host_bytes < bytes) {
    if (c->stream_host) cudaFreeHost(c->stream_host);
    c->stream_host = nullptr;
    c->stream_host_bytes = 0;
    if (cudaMallocHost(&c->stream_host, bytes) == cudaSuccess) {
      c->stream_host_bytes = bytes;
    } else {
      (void)cudaGetLastError();
      c->stream_host = nullptr;
    }
  }
  if (c->stream_host) {
    h->off = static_cast<uint64_t*>(c->stream_host);
    h->rank = reinterpret_cast<uint32_t*>(h->off + n + 1);
    h->pinned = true;
  } else {
    h->off_v.resize(n + 1);
    h->rank_v.resize(n);
    h->off = h->off_v.data();
    h->rank = h->rank_v.data();
  }
}

// Phase 2 of the rows tier: each range's rows built in rank order into one
// resident oriented graph, which the context then holds prepared (as a
// one-piece count leaves it) and counts once. size[r]: range r's entries.
void count_rows_tier(tribit_context* c, const RowsSource& src, const std::vector<uint64_t>& size,
                     const std::vector<uint32_t>& hb, const CarryHost& carry, uint64_t n, uint64_t E, uint64_t kept,
                     bool hubs, uint64_t cap, uint64_t piece_words, std::chrono::steady_clock::time_point t0,
                     tribit_result* res) {
  cudaStream_t st = c->st;
  Arena& ar = c->arena;
  RowsLayout L;
  ar.reserve(rows_layout(ar, true, n, kept, cap, hubs, piece_words, &L), false);
  rows_layout(ar, false, n, kept, cap, hubs, piece_words, &L);
  TB_CUDA(cudaMemsetAsync(L.stats, 0, sizeof(DeviceStats), st));
  float h2d_ms = 0.f;
  auto upload = [&](const void* from, size_t bytes, void* dst) {
    const auto tu = std::chrono::steady_clock::now();
    upload_via_pinned(c, from, bytes, dst);
    h2d_ms += ms_since(tu);
  };
  auto upload_carry = [&](const void* from, size_t bytes, void* dst) {
    if (!carry.pinned) return upload(from, bytes, dst);
    TB_CUDA(cudaMemcpyAsync(dst, from, bytes, cudaMemcpyHostToDevice, st));
  };
  upload_carry(carry.off, (n + 1) * sizeof(uint64_t), L.row_start);
  PieceStream ps;
  if (!src.bucket) {
    upload_carry(carry.rank, n * sizeof(uint32_t), L.rank);
    ps = *src.stream;
    ps.pieces[0] = L.pieces[0];
    ps.pieces[1] = L.pieces[1];
  }
  const size_t P = size.size();
  for (size_t r = 0; r < P; ++r) {
    const uint32_t s = hb[r], z = hb[r + 1] - hb[r];
    if (src.bucket) {
      if (size[r]) upload((*src.bucket)[r].get(), size[r] * sizeof(uint64_t), L.build.keys);
      build_row_range(L.build, L.row_start, s, z, size[r], L.rp, L.col, L.bent, &L.stats->err, st);
      continue;
    }
    if (z == 0) continue;
    begin_row_range(L.build, L.row_start, s, z, L.rp, st);
    TB_CUDA(cudaEventRecord(c->ev[0], st));
    ps.pass([&](const uint64_t* piece, uint64_t cnt) {
      k_s_fill<<<grid_for(cnt), kThreads, 0, st>>>(piece, cnt, n, L.rank, s, z, L.build.off, L.build.cursor,
                                                   L.build.nbr, &L.stats->err);
      TB_LAUNCH_CHECK();
    });
    TB_CUDA(cudaEventRecord(c->ev[1], st));
    finish_row_range(L.build, s, z, size[r], L.rp, L.col, L.bent, &L.stats->err, st);
    float pass_ms = 0.f;
    TB_CUDA(cudaEventSynchronize(c->ev[1]));
    TB_CUDA(cudaEventElapsedTime(&pass_ms, c->ev[0], c->ev[1]));
    h2d_ms += pass_ms;
  }
  finalize_rows(L.rp, n, L.stats, st);
  Prepared& p = c->prep;
  p = Prepared{};
  p.view.n = (uint32_t)n;
  p.view.rp = L.rp;
  p.view.col = L.col;
  p.view.bent = L.bent;
  p.stats = L.stats;
  p.n = n;
  p.E = E;
  c->sched = L.sched;
  apply_dispatch(c, st);
  c->per_graph = nullptr;
  c->num_graphs = 0;
  c->prepared = true;
  TB_CUDA(cudaEventRecord(c->ev[2], st));
  c->launch = launch_count(p.view, c->sched, p.stats, nullptr, count_config(c), st);
  TB_CUDA(cudaEventRecord(c->ev[3], st));
  TB_CUDA(cudaMemcpyAsync(c->h_stats, p.stats, sizeof(DeviceStats), cudaMemcpyDeviceToHost, st));
  TB_CUDA(cudaStreamSynchronize(st));
  const DeviceStats& hs = *c->h_stats;
  if (hs.err & (kErrInput | kErrIdRange)) {
    c->prepared = false;
    throw StatusError(TRIBIT_ERR_INVALID_ARGUMENT, "the host entries changed during the count");
  }
  if (hs.count_err & kErrTimeout) throw StatusError(TRIBIT_ERR_TIMEOUT, "a device-side wait gave up");
  if (!res) return;
  std::memset(res, 0, sizeof *res);
  fill_schedule_stats(c, res);
  res->triangles = hs.triangles;
  res->num_nodes = n;
  res->entries = E;
  res->edges = hs.edges;
  res->blocks_of_threads = c->launch.ctas;
  res->count_kernels = c->launch.kernels;
  TB_CUDA(cudaEventElapsedTime(&res->kernel_ms, c->ev[2], c->ev[3]));
  res->total_ms = ms_since(t0);
  res->h2d_ms = h2d_ms;
  res->preprocess_ms = std::max(0.f, res->total_ms - res->kernel_ms - h2d_ms);
  res->stream_tasks = 1;
  res->stream_tier = TRIBIT_STREAM_ROWS;
}

bool count_streamed_if_needed(tribit_context* c, const uint64_t* host, uint64_t E, uint64_t n, tribit_result* res) {
  DeviceGuard dg(c->device);
  if (n == 0 || E == 0) return false;
  const uint64_t budget = budget_bytes(c);
  if (call_bytes(c, E, n, c->opts.order, true) <= budget) return false;
  if (n > 0x7fffffffull)
    throw StatusError(TRIBIT_ERR_TOO_LARGE, "counting in rank ranges takes fewer than 2^31 vertices");
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t st = c->st;
  // Phase 1 and the rows tier run in the context's arena, kept across calls of
  // the same budget (no reallocation); the pairs tier's buffer in its own.
  if (c->arena.capacity() > budget) c->arena.release();
  c->stream_arena.release();
  drop_graph(c);
  c->prepared = false;

  // ---- phase 1: per-vertex buffers and the pieces in flight -----------------
  // A piece of at most 32 MiB of entries and at most 1/2048 of the budget in
  // entries (phase 1's piece buffers take 36 bytes an entry: two piece
  // buffers, keys, ranges, grouped keys; the rows tier's two take 16).
  const uint64_t piece_words = std::max<uint64_t>(1u << 14, std::min<uint64_t>(kPieceWords, budget / 2048));
  Arena& ar = c->arena;
  uint32_t *deg = nullptr, *rank = nullptr, *rows = nullptr, *bounds = nullptr, *hist = nullptr, *rng = nullptr;
  uint64_t *off = nullptr, *otmp = nullptr, *size = nullptr, *keys = nullptr, *part = nullptr;
  uint64_t* pieces[2] = {nullptr, nullptr};
  unsigned int* flags = nullptr;  // [0] error flags, [1] longest row
  RankBuffers rb;
  for (int pass = 0; pass < 2; ++pass) {
    ar.begin(pass == 0);
    deg = ar.take<uint32_t>(n);
    rank = ar.take<uint32_t>(n);
    rows = ar.take<uint32_t>(n + 1);
    off = ar.take<uint64_t>(n + 1);
    otmp = take_scan_temp<uint64_t>(ar, n + 1);
    rb = take_rank_buffers(ar, n);
    bounds = ar.take<uint32_t>(kMaxRanges + 1);
    size = ar.take<uint64_t>(kMaxRanges);
    hist = ar.take<uint32_t>(kMaxRanges);
    flags = ar.take<unsigned int>(2);
    pieces[0] = ar.take<uint64_t>(piece_words);
    pieces[1] = ar.take<uint64_t>(piece_words);
    keys = ar.take<uint64_t>(piece_words);
    rng = ar.take<uint32_t>(piece_words);
    part = ar.take<uint64_t>(piece_words);
    if (pass == 0) {
      if (ar.used() > budget)
        throw StatusError(TRIBIT_ERR_OUT_OF_MEMORY, "the per-vertex arrays alone exceed the device budget");
      ar.reserve(ar.used(), false);
    }
  }
  ensure_pinned(c);
  TB_CUDA(cudaMemsetAsync(flags, 0, 2 * sizeof(unsigned int), st));
  PieceStream ps;
  ps.c = c;
  ps.host = host;
  ps.E = E;
  ps.piece_words = piece_words;
  ps.pinned_src = host_is_pinned(host);
  ps.pieces[0] = pieces[0];
  ps.pieces[1] = pieces[1];
  auto stream_pass = [&](auto&& fn) { ps.pass(fn); };
  auto check_flags = [&](unsigned int* out2) {
    unsigned int h[2] = {0, 0};
    TB_CUDA(cudaMemcpyAsync(h, flags, sizeof h, cudaMemcpyDeviceToHost, st));
    TB_CUDA(cudaStreamSynchronize(st));
    if (h[0] & kErrIdRange) throw StatusError(TRIBIT_ERR_ID_RANGE, "an entry names a vertex id >= num_nodes");
    if (out2) *out2 = h[1];
  };
  // Degrees, then the (degree, id) rank order.
  TB_CUDA(cudaMemsetAsync(deg, 0, n * sizeof(uint32_t), st));
  stream_pass([&](const uint64_t* piece, uint64_t cnt) {
    k_s_degree<<<grid_for(cnt), kThreads, 0, st>>>(piece, cnt, n, deg, flags);
    TB_LAUNCH_CHECK();
  });
  check_flags(nullptr);
  rank_vertices(deg, n, E, rb, rank, st);
  // Oriented entries per row (with duplicates), their prefix, the longest row.
  TB_CUDA(cudaMemsetAsync(rows, 0, (n + 1) * sizeof(uint32_t), st));
  stream_pass([&](const uint64_t* piece, uint64_t cnt) {
    k_s_rows<<<grid_for(cnt), kThreads, 0, st>>>(piece, cnt, n, rank, rows, flags);
    TB_LAUNCH_CHECK();
  });
  k_s_widen<<<grid_for(n + 1), kThreads, 0, st>>>(rows, n + 1, off, flags + 1);
  TB_LAUNCH_CHECK();
  device_scan<uint64_t, OpSum>(off, off, n + 1, true, OpSum{}, 0ull, otmp, st);
  uint64_t kept = 0;
  TB_CUDA(cudaMemcpyAsync(&kept, off + n, sizeof kept, cudaMemcpyDeviceToHost, st));
  unsigned int max_row = 0;
  check_flags(&max_row);

  // ---- the tier and its ranges -------------------------------------------------
  // Rows tier: the oriented rows (rp, col, bent) and the schedule stay on the
  // device, and one range's build buffers of `cap` entries come and go. Pairs
  // tier: a task of ranges i < j holds at most 3 cap entries (bucket i, its
  // entries into R_j again, bucket j) on at most 2n vertices.
  const uint64_t user_cap = c->stream_range_entries;
  if (user_cap && user_cap <= max_row)
    throw StatusError(TRIBIT_ERR_OUT_OF_MEMORY, "the range bound is at or below the longest row");
  RowsPlan plan;
  const bool rows_tier = c->stream_tier != TRIBIT_STREAM_PAIRS && n <= 0xffffffffull && kept <= 0xfffffffeull &&
                         plan_rows(c->arena, n, kept, max_row, budget, piece_words, &plan);
  if (c->stream_tier == TRIBIT_STREAM_ROWS && !rows_tier)
    throw StatusError(TRIBIT_ERR_OUT_OF_MEMORY, "the oriented rows alone exceed the device budget");
  uint64_t cap = 0;
  if (rows_tier) {
    cap = plan.cap;
  } else {
    const uint64_t n2 = 2 * n;
    const uint64_t fixed = call_bytes(c, 0, n2, TRIBIT_ORDER_ID, false);
    const uint64_t probe = 1ull << 20;
    const uint64_t per_entry =
        (call_bytes(c, probe, n2, TRIBIT_ORDER_ID, false) - fixed) / probe + 1 + sizeof(uint64_t);
    if (budget <= fixed)
      throw StatusError(TRIBIT_ERR_OUT_OF_MEMORY, "the device budget is below a range task's per-vertex buffers");
    cap = std::min<uint64_t>((budget - fixed) / per_entry / 3, 0xfffffffeull / 3);
    if (cap <= max_row) throw StatusError(TRIBIT_ERR_OUT_OF_MEMORY, "the device budget is below the longest row's share");
  }
  if (user_cap) cap = std::min(cap, user_cap);
  const uint64_t P = cap >= kept ? 1 : ceil_div<uint64_t>(kept, cap - max_row);
  if (P > kMaxRanges) throw StatusError(TRIBIT_ERR_TOO_LARGE, "the graph needs more rank ranges than supported");
  k_s_bounds<<<1, kMaxRanges + 1, 0, st>>>(off, n, cap >= kept ? kept + 1 : cap - max_row, (uint32_t)P, bounds, size);
  TB_LAUNCH_CHECK();
  std::vector<uint32_t> hb(P + 1);
  std::vector<uint64_t> hsize(P);
  TB_CUDA(cudaMemcpyAsync(hb.data(), bounds, (P + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  TB_CUDA(cudaMemcpyAsync(hsize.data(), size, P * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  // The rows tier builds ranges from the global row starts; with few ranges
  // it fills each one straight from the entries streamed again (the ranks
  // orient them), instead of sending every key to a host bucket and back.
  const bool direct = rows_tier && P <= (ps.pinned_src ? kDirectRangesPinned : kDirectRangesPageable);
  CarryHost carry;
  if (rows_tier) {
    carry_host(c, n, &carry);
    TB_CUDA(cudaMemcpyAsync(carry.off, off, (n + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  }
  if (direct) TB_CUDA(cudaMemcpyAsync(carry.rank, rank, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  TB_CUDA(cudaStreamSynchronize(st));

  if (direct) {  // phase 1 is done: the arena's space goes to phase 2
    RowsSource src;
    src.stream = &ps;
    count_rows_tier(c, src, hsize, hb, carry, n, E, kept, plan.hubs, cap, piece_words, t0, res);
    if (res) res->stream_ranges = (uint32_t)P;
    return true;
  }

  // ---- host buckets of oriented keys, one per range --------------------------
  std::vector<std::unique_ptr<uint64_t[]>> bucket(P);
  std::vector<uint64_t> filled(P, 0);
  for (uint64_t r = 0; r < P; ++r) bucket[r].reset(new uint64_t[std::max<uint64_t>(hsize[r], 1)]);
  std::vector<uint32_t> hh(P), cur(P);
  stream_pass([&](const uint64_t* piece, uint64_t cnt) {
    TB_CUDA(cudaMemsetAsync(hist, 0, P * sizeof(uint32_t), st));
    k_s_keys<<<grid_for(cnt), kThreads, (2 * P + 1) * sizeof(uint32_t), st>>>(piece, cnt, n, rank, bounds,
                                                                               (uint32_t)P, keys, rng, hist, flags);
    TB_LAUNCH_CHECK();
    TB_CUDA(cudaMemcpyAsync(hh.data(), hist, P * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    TB_CUDA(cudaStreamSynchronize(st));
    uint32_t run = 0;
    for (uint64_t r = 0; r < P; ++r) cur[r] = run, run += hh[r];
    TB_CUDA(cudaMemcpyAsync(hist, cur.data(), P * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    k_s_scatter<<<grid_for(cnt), kThreads, 0, st>>>(keys, rng, cnt, hist, part);
    TB_LAUNCH_CHECK();
    // The grouped keys come back through pinned buffer 1 (buffer 0 may hold the next piece).
    pinned_wait(c, 1);
    TB_CUDA(cudaMemcpyAsync(c->pinned[1], part, run * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    pinned_used(c, 1, st);
    TB_CUDA(cudaStreamSynchronize(st));
    const uint64_t* back = static_cast<const uint64_t*>(c->pinned[1]);
    for (uint64_t r = 0; r < P; ++r) {
      if (filled[r] + hh[r] > hsize[r]) throw StatusError(TRIBIT_ERR_INVALID_ARGUMENT, "the host entries changed during the count");
      host_copy(bucket[r].get() + filled[r], back + cur[r], hh[r] * sizeof(uint64_t));
      filled[r] += hh[r];
    }
  });
  check_flags(nullptr);
  for (uint64_t r = 0; r < P; ++r)
    if (filled[r] != hsize[r]) throw StatusError(TRIBIT_ERR_INVALID_ARGUMENT, "the host entries changed during the count");
  const float phase1_ms = ms_since(t0);

  if (rows_tier) {
    RowsSource src;
    src.bucket = &bucket;
    count_rows_tier(c, src, hsize, hb, carry, n, E, kept, plan.hubs, cap, piece_words, t0, res);
    if (res) res->stream_ranges = (uint32_t)P;
    return true;
  }

  // ---- phase 2 of the pairs tier: every pair of ranges i <= j ------------------
  ar.release();  // the tasks size the context's arena themselves
  Arena& wa = c->stream_arena;
  uint64_t tri = 0, edges = 0, ctas = 0, blocks = 0, tasks = 0;
  uint64_t by_variant[TRIBIT_NUM_VARIANTS] = {0, 0, 0};
  float prep_ms = 0.f, kernel_ms = 0.f, h2d_ms = 0.f;
  uint32_t kernels = 0;
  unsigned long long* extra = nullptr;
  uint64_t max_bucket = 0;
  for (uint64_t r = 0; r < P; ++r) max_bucket = std::max(max_bucket, filled[r]);
  uint64_t* w = nullptr;
  for (int pass = 0; pass < 2; ++pass) {
    wa.begin(pass == 0);
    w = wa.take<uint64_t>(3 * max_bucket + 1);
    extra = wa.take<unsigned long long>(1);
    if (pass == 0) wa.reserve(wa.used(), false);
  }
  for (uint64_t i = 0; i < P; ++i) {
    for (uint64_t j = i; j < P; ++j) {
      const uint64_t ci = filled[i], cj = i == j ? 0 : filled[j];
      if (ci == 0) break;  // no rows of R_i: nothing of it to count against any R_j
      const uint32_t si = hb[i], zi = hb[i + 1] - hb[i], sj = hb[j], zj = hb[j + 1] - hb[j];
      if (i != j && cj == 0) continue;
      const auto tu = std::chrono::steady_clock::now();
      upload_via_pinned(c, bucket[i].get(), ci * sizeof(uint64_t), w);
      if (cj) upload_via_pinned(c, bucket[j].get(), cj * sizeof(uint64_t), w + ci);
      uint64_t E2 = ci + cj, n2t = n - si;
      if (i == j) {
        k_s_diag<<<grid_for(ci), kThreads, 0, st>>>(w, ci, si);
        TB_LAUNCH_CHECK();
      } else {
        TB_CUDA(cudaMemsetAsync(extra, 0, sizeof(unsigned long long), st));
        k_s_pair<<<grid_for(ci + cj), kThreads, 0, st>>>(w, ci, cj, si, zi, sj, zj, extra);
        TB_LAUNCH_CHECK();
        unsigned long long ex = 0;
        TB_CUDA(cudaMemcpyAsync(&ex, extra, sizeof ex, cudaMemcpyDeviceToHost, st));
        TB_CUDA(cudaStreamSynchronize(st));
        E2 += ex;
        n2t = (uint64_t)zi + zj + (n - si);
      }
      TB_CUDA(cudaStreamSynchronize(st));
      h2d_ms += ms_since(tu);
      tribit_result r;
      count_device_input(c, w, E2, n2t, TRIBIT_ORDER_ID, &r);
      tri += r.triangles;
      if (i == j) edges += r.edges;
      ctas += r.blocks_of_threads;
      kernels = r.count_kernels;
      prep_ms += r.preprocess_ms;
      kernel_ms += r.kernel_ms;
      if (i == j) {
        blocks += r.row_blocks;
        for (int v = 0; v < TRIBIT_NUM_VARIANTS; ++v) by_variant[v] += r.row_blocks_by_variant[v];
      }
      ++tasks;
    }
  }
  // The tasks' graphs are not the input graph: the context keeps nothing prepared.
  c->prepared = false;
  drop_graph(c);
  wa.release();
  if (res) {
    std::memset(res, 0, sizeof *res);
    res->triangles = tri;
    res->num_nodes = n;
    res->entries = E;
    res->edges = edges;
    res->blocks_of_threads = ctas;
    res->row_blocks = blocks;
    for (int v = 0; v < TRIBIT_NUM_VARIANTS; ++v) res->row_blocks_by_variant[v] = by_variant[v];
    res->h2d_ms = h2d_ms;
    res->preprocess_ms = phase1_ms + prep_ms;
    res->kernel_ms = kernel_ms;
    res->total_ms = ms_since(t0);
    res->count_kernels = kernels;
    res->stream_ranges = (uint32_t)P;
    res->stream_tasks = (uint32_t)tasks;
    res->stream_tier = TRIBIT_STREAM_PAIRS;
  }
  return true;
}

}  // namespace tb

extern "C" tribit_status tribit_set_device_budget(tribit_context* c, uint64_t bytes) {
  if (!c) return TRIBIT_ERR_INVALID_ARGUMENT;
  c->device_budget = bytes;
  return TRIBIT_OK;
}

extern "C" tribit_status tribit_set_stream_options(tribit_context* c, int tier, uint64_t range_entries) {
  if (!c || tier < TRIBIT_STREAM_AUTO || tier > TRIBIT_STREAM_PAIRS) return TRIBIT_ERR_INVALID_ARGUMENT;
  c->stream_tier = tier;
  c->stream_range_entries = range_entries;
  return TRIBIT_OK;
}
