// Counting kernels over a prepared graph (see prep.cuh).
//
// Triangles = sum over u, over v in N+(u), of |N+(u) & N+(v)|: each triangle
// is counted once, at its lowest-ranked vertex. This is the quantity the
// reference accumulates as sum popc(U(u, blk) & L(v, blk)) in
// compute_binary_popcount_mma_9 (tribit.cu:519-586), whose per-lane binary
// searches and one-row-in-eight b1 MMA tiles it replaces.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "arena.h"
#include "prep.cuh"

namespace tb {

// Per-32-row-block schedule: which variant counts each row block.
struct Schedule {
  uint32_t num_row_blocks = 0;
  uint8_t* variant_of = nullptr;                   // device, num_row_blocks
  uint32_t* list[TRIBIT_NUM_VARIANTS] = {};        // device, row blocks of each variant
  uint32_t* list_len = nullptr;                    // device, TRIBIT_NUM_VARIANTS
  uint32_t* overflow = nullptr;                    // device, rows deferred to wider paths
  uint32_t overflow_cap = 0;
  float* features = nullptr;                       // device, num_row_blocks x kNumFeatures
  uint32_t* scan_tmp = nullptr;
  uint32_t* flags = nullptr;
};

constexpr int kNumFeatures = 16;

// Per-launch configuration chosen by the autotuner (or defaults).
struct CountConfig {
  int ctas_per_sm = 0;     // 0 = default
  int num_sms = 148;
};

Schedule take_schedule(Arena& ar, uint64_t n);

// Computes row-block features and the per-variant work lists.
// mode: TRIBIT_DISPATCH_* ; mlp_weights: device weights for LEARNED (or null).
void build_schedule(const GraphView& g, Schedule& s, int mode, const void* mlp, cudaStream_t st);

struct LaunchInfo {
  uint64_t ctas = 0;      // CTAs over all counting kernels
  uint32_t kernels = 0;   // kernel launches
};

// Launches every counting kernel; the exact count lands in stats->triangles
// (and per_graph[g] in batch mode).
LaunchInfo launch_count(const GraphView& g, const Schedule& s, DeviceStats* stats, unsigned long long* per_graph,
                      const CountConfig& cfg, cudaStream_t st);

}  // namespace tb
