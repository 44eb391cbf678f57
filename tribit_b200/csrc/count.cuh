// Counting kernels over a prepared graph (see prep.cuh).
//
// Triangles = sum over u, over v in N+(u), of |N+(u) & N+(v)|: each triangle
// is counted once, at its lowest-ranked vertex. This is the quantity the
// reference accumulates as sum popc(U(u, blk) & L(v, blk)) in
// compute_binary_popcount_mma_9 (tribit.cu:519-586), whose per-lane binary
// searches and one-row-in-eight b1 MMA tiles it replaces.
//
// Work is scheduled in two levels. The dispatcher assigns every 32-row block
// of the oriented graph one counting variant (row-block features -> plain
// thresholds or the learned MLP). Each variant's rows are then cut into
// pieces of at most piece_width neighbours, so one heavy row is spread
// over many warps; the variant kernels are persistent and pull pieces from a
// device cursor.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "arena.h"
#include "prep.cuh"

namespace tb {

constexpr int kNumFeatures = 16;
constexpr int kTileMaxK = 64;  // bit-tile variant: row blocks spanning at most this many column blocks
constexpr int kFeatSpan = 13;  // feature index of log2(1 + column-block span)
constexpr uint32_t kMinPieceWidth = 32;  // piece_width is a multiple of 32, at least this
// Plain dispatcher: a row block goes to the merge variant when its neighbours'
// bit rows average at least this many times its own rows' length. Set once from
// a sweep over RMAT-18..24, planted partition, Chung-Lu and Erdos-Renyi graphs:
// 0.75 is within 2-6% of the per-graph best ratio on each of them (0.5 wins on
// RMAT-22/24 but loses 48% on planted and Erdos-Renyi, 2.0 loses 96% on RMAT-24).
constexpr float kDefaultMergeRatio = 0.75f;

struct Schedule {
  uint32_t num_row_blocks = 0;
  uint8_t* variant_of = nullptr;   // device, per row block
  uint64_t* pieces = nullptr;      // device, (row << 32) | first neighbour, grouped by variant
  uint64_t piece_cap = 0;
  uint32_t* piece_off = nullptr;   // device, TRIBIT_NUM_VARIANTS + 1 segment starts, the heavy-row count,
                                   // the CTA hub-piece count, all hub pieces, the hub-edge count
  uint32_t* heavy = nullptr;       // device, rows too wide for one warp, counted CTA-cooperatively first
  uint32_t* row_flags = nullptr;   // device, n + 1 scratch for the heavy-row scan
  uint32_t* row_scan_tmp = nullptr;
  uint32_t* list_len = nullptr;    // device, row blocks per variant
  uint32_t* block_pieces = nullptr;// device, pieces per row block
  uint32_t* flags = nullptr;       // device, nrb + 1 scratch for the scans
  uint32_t* scan_tmp = nullptr;
  uint32_t* overflow = nullptr;    // device, rows deferred to the CTA / global passes
  uint32_t overflow_cap = 0;
  float* features = nullptr;       // device, nrb x kNumFeatures
  // Hub pass of the merge variant (absent when taken without hubs).
  uint32_t* eflag = nullptr;       // device, bit per CSR position: edge counted by the hub pass
  uint64_t eflag_words = 0;
  uint64_t* vinfo = nullptr;       // device, n: (row span in blocks << 32) | bit-row length
  unsigned long long* save = nullptr;  // device, n: blocks a hub walk would save
  uint32_t* in_cnt = nullptr;      // device, n + 1
  uint32_t* in_off = nullptr;      // device, n + 1: in-list of hub v at [in_off[v], in_off[v+1])
  uint64_t* inl = nullptr;         // device: (first block of u's tail << 32) | tail length
  uint64_t inl_cap = 0;            // entries inl (and inrow) hold
  uint32_t* inrow = nullptr;       // device: u of each in-list entry (timing mode only: its own buffer)
  uint64_t* hub_pieces = nullptr;  // device: (v << 32) | first in-list entry; CTA pieces, then warp pieces
  uint64_t* hub_pieces2 = nullptr; // device: the pieces in hub order, before the wave sort
  uint8_t* piece_wave = nullptr;   // device: wave of each piece's first tail
  uint32_t* wave_lo = nullptr;     // device: first row of each wave, then n
  uint32_t* wave_bk = nullptr;     // device: bit-row start of each wave's first row
  uint32_t* wave_cp = nullptr;     // device: CSR position of each wave's first row
  uint32_t* wave_cnt = nullptr;    // device: pieces per (list, wave), scanned to positions
  uint32_t* hub_pos = nullptr;     // device, 2n + 2: piece counts, scanned to piece positions
  uint32_t* hub_scan_tmp = nullptr;
  bool hubs = true;                // build the hub lists for merge row blocks
  bool hubs_active = false;        // set by build_pieces
  bool hub_rows = false;           // also write each in-list entry's row (read by the timing mode only)
  uint32_t piece_width = 64;       // neighbours per piece (tuned)
  float tile_min_nnz = 64.f;       // plain dispatcher: fewest edges for a bit-tile row block (tuned)
  float merge_ratio = kDefaultMergeRatio;  // plain dispatcher: merge where neighbours' bit rows are this much longer
  int tile_engine = TRIBIT_TILES_TCGEN05;  // bit-tile product: tcgen05 kind::i8 or b1 mma.sync
  const void* model = nullptr;     // device MLP parameters for learned dispatch
};

// Per-launch configuration chosen by the autotuner (or defaults).
struct CountConfig {
  int ctas_per_sm = 0;  // 0 = default
  int num_sms = 148;
  unsigned long long* block_ns = nullptr;  // optional: per-row-block warp-cycles (SM cycles x warps busy)
  cudaEvent_t variant_start = nullptr;     // optional (timing mode): these events bracket
  cudaEvent_t variant_stop = nullptr;      // all counting kernels
  uint32_t tile_wait_polls = 1u << 22;     // tcgen05 tiles: mbarrier polls before a wait gives up
  int tile_test_no_commit = 0;             // failure-detection test: tile MMAs never committed
  bool queue = false;                      // TRIBIT_LAUNCH_QUEUE (not in the timing mode)
};

// TRIBIT_LAUNCH_AUTO takes the queue kernel up to this many entries: on one
// B200 it counted Chung-Lu n = 7,115 in 0.051 ms instead of 0.085, RMAT-16
// 32% and RMAT-18 12% faster, RMAT-20 (2^24 entries) even, and RMAT-21 to 24
// 3-5% slower (5 CTAs an SM for the row pieces instead of 6-7).
constexpr uint64_t kQueueMaxEntries = 1ull << 24;

// hubs: also take the hub-pass arrays (about 13 bytes per entry).
Schedule take_schedule(Arena& ar, uint64_t n, uint64_t E, bool hubs = true);

// Computes row-block features, the per-block variant (mode: TRIBIT_DISPATCH_*),
// and the per-variant piece lists. full_features adds the neighbour-side
// features (one extra pass over the edges) the learned dispatcher needs.
// Sends the row blocks dispatched to the merge variant to the bitmap sweep.
void merge_blocks_to_bitmap(Schedule& s, cudaStream_t st);
void build_schedule(const GraphView& g, Schedule& s, int mode, bool full_features, cudaStream_t st);

// Row-block features (full adds the neighbour-side ones) and the plain or
// forced variant for every row block; build_schedule = this + build_pieces.
void compute_features(const GraphView& g, Schedule& s, int mode, bool full_features, cudaStream_t st);

// Re-derives the piece lists after variant_of was rewritten (learned dispatch).
void build_pieces(const GraphView& g, Schedule& s, cudaStream_t st);

struct LaunchInfo {
  uint64_t ctas = 0;     // CTAs over all counting kernels
  uint32_t kernels = 0;  // kernel launches
};

// Launches every counting kernel; the exact count lands in stats->triangles
// (and per_graph[g] in batch mode).
LaunchInfo launch_count(const GraphView& g, const Schedule& s, DeviceStats* stats, unsigned long long* per_graph,
                        const CountConfig& cfg, cudaStream_t st);

}  // namespace tb
