// GPU preprocessing: raw entries -> oriented, deduplicated CSR plus the
// bit-packed 32-column block rows the counting kernels read.
//
// Replaces count_triangles' preprocessing (tribit.cu:666-758): the
// reference sorts the full 64-bit words with CUB, builds separate L and U bit
// matrices with two more 64-bit pair sorts and reduce-by-key, and syncs with
// the host five times. Here one sort of compact keys gives both the CSR and
// the bit rows, and nothing reads back to the host until the final count.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "arena.h"
#include "common.cuh"
#include "scan.cuh"

namespace tb {

// Device view of a prepared graph, in rank space (vertex r = the r-th vertex
// of the chosen order). Row u holds N+(u) = neighbours of higher rank.
struct GraphView {
  uint32_t n;                     // vertices
  const uint64_t* rp;             // n + 1 words: (row_ptr << 32) | brow_ptr
  const uint32_t* col;            // N+(u), ascending, at [row_ptr[u], row_ptr[u+1])
  const uint64_t* bent;           // bit rows: (block << 32) | mask, ascending block,
                                  // at [brow_ptr[u], brow_ptr[u+1]); bit (w & 31) of
                                  // block w >> 5 is set iff w in N+(u)
  const uint32_t* graph_of_rank;  // batch mode: graph id of each rank, else null
  const uint32_t* eflag;          // per CSR position, bit set: the edge is counted by the
                                  // hub pass, not by its row (set by the schedule), or null
};

__device__ __forceinline__ uint32_t rp_row(uint64_t w) { return (uint32_t)(w >> 32); }
__device__ __forceinline__ uint32_t rp_blk(uint64_t w) { return (uint32_t)w; }

// Counters the device writes and the host reads back once per call.
struct DeviceStats {
  unsigned long long triangles;
  unsigned long long edges;        // undirected edges after dedup (m)
  unsigned long long blocks;       // bit-row entries (nb)
  unsigned int err;                // kErr* flags of the preprocessing
  unsigned int count_err;          // kErr* flags of the latest counting launch (cleared by each launch)
  unsigned int cursor[8];          // work cursors of the counting kernels
  unsigned int overflow[8];        // overflow-list lengths
};

// Upload of host entries overlapped with the degree pass: the entries are
// copied in kUploadChunks pieces on copy_stream, and each piece's degree pass
// runs on the preparing stream as soon as the piece has landed. events: at
// least kUploadChunks + 1 (the first orders the copies after the stream's
// earlier work); uploaded is recorded on the preparing stream once every
// piece has landed.
constexpr int kUploadChunks = 8;
struct HostUpload {
  const uint64_t* host = nullptr;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t* events = nullptr;
  cudaEvent_t uploaded = nullptr;
  // Optional: copies bytes from host to device on a stream in its own way
  // (pageable host memory staged through pinned buffers by host threads);
  // null: one cudaMemcpyAsync.
  void (*stage)(void* ctx, void* dst, const void* src, size_t bytes, cudaStream_t st) = nullptr;
  void* stage_ctx = nullptr;
};

struct PrepInput {
  const uint64_t* entries = nullptr;  // device, E words (a << 32) | b
  HostUpload upload{};                // host: fill entries from upload.host first
  uint64_t E = 0;
  uint64_t n = 0;                     // vertices (sum over graphs in batch mode)
  int order = TRIBIT_ORDER_DEGREE;
  // batch mode (G > 0): graph g owns entries [eoff[g], eoff[g+1]) with local
  // ids in [0, voff[g+1] - voff[g]); its vertices are voff[g] + local id.
  uint32_t G = 0;
  const uint64_t* eoff = nullptr;  // device, G + 1
  const uint64_t* voff = nullptr;  // device, G + 1
};

struct Prepared {
  GraphView view{};
  DeviceStats* stats = nullptr;  // device
  uint32_t* rank = nullptr;      // id -> rank
  uint64_t n = 0;
  uint64_t E = 0;
};

// Lays out (measuring arena) or lays out and launches (real arena) the whole
// preprocessing pipeline on stream st. Stats are zeroed here.
void prepare_graph(Arena& ar, const PrepInput& in, cudaStream_t st, Prepared* out);

// The (degree, id) rank order of n vertices from their degrees (E entries
// counted them, which bounds a degree by 2E): rank[v] = position of v. The
// buffers come from take_rank_buffers; launches only.
struct RankBuffers {
  uint32_t *vk = nullptr, *vk2 = nullptr, *vv = nullptr, *vv2 = nullptr;
  RadixTemp tmp{};
};
RankBuffers take_rank_buffers(Arena& ar, uint64_t n);
void rank_vertices(const uint32_t* deg, uint64_t n, uint64_t E, const RankBuffers& b, uint32_t* rank, cudaStream_t st);

// One rank range's rows at a time: the oriented graph's rows [s, s + z) built
// from that range's keys alone (lo << 32 | hi in rank space, lo in the range,
// duplicates allowed), with the row sorts and the CSR / bit-row emission of
// preprocessing, into the same rp / col / bent a one-piece build gives. Built
// in increasing s, the ranges leave rp, col and bent equal to the one-piece
// arrays, with scratch for one range (at most `cap` keys) instead of the graph.
struct RowRangeBuffers {
  uint64_t* keys = nullptr;     // cap + 1 words: the range's keys (the caller fills them)
  uint32_t* scratch = nullptr;  // the same memory: long rows' sort space after the fill
  uint32_t* nbr = nullptr;      // cap: the range's rows
  uint32_t* off = nullptr;      // n + 1: range-relative row starts
  uint32_t* cursor = nullptr;   // n + 1: fill cursors
  uint32_t* big = nullptr;      // n + 1: rows for the CTA sort
  uint32_t* nbig = nullptr;
  uint64_t* carry = nullptr;    // rp of the range's first row before the range is built
  uint64_t* scan_tmp = nullptr;
};
RowRangeBuffers take_row_range_buffers(Arena& ar, uint64_t n, uint64_t cap);
// row_start: n + 1 exclusive prefix of the rows' key counts (duplicates
// included); cnt = row_start[s + z] - row_start[s] keys in b.keys. A key whose
// row or slot is out of place (the entries changed between the passes that
// counted and bucketed them) is dropped and sets kErrInput in *err.
void build_row_range(const RowRangeBuffers& b, const uint64_t* row_start, uint32_t s, uint32_t z, uint64_t cnt,
                     uint64_t* rp, uint32_t* col, uint64_t* bent, unsigned int* err, cudaStream_t st);
// The same in two halves around a fill of the caller's own: begin sets the
// range's row starts and fill cursors (b.off, b.cursor); the caller then
// places each of the range's cnt entries at nbr[atomicAdd(&cursor[row - s], 1)]
// (checking it against off[row - s + 1]); finish checks every row is full and
// sorts, deduplicates and emits the rows.
void begin_row_range(const RowRangeBuffers& b, const uint64_t* row_start, uint32_t s, uint32_t z, uint64_t* rp,
                     cudaStream_t st);
void finish_row_range(const RowRangeBuffers& b, uint32_t s, uint32_t z, uint64_t cnt, uint64_t* rp, uint32_t* col,
                      uint64_t* bent, unsigned int* err, cudaStream_t st);
// Edge and bit-block totals of rp[n] into stats.
void finalize_rows(const uint64_t* rp, uint64_t n, DeviceStats* stats, cudaStream_t st);

}  // namespace tb
