// The tribit_context behind the C-ABI handle, shared by the C-ABI sources.
#pragma once
#include <cuda_runtime.h>

#include <new>
#include <string>

#include "arena.h"
#include "common.cuh"
#include "count.cuh"
#include "model.cuh"
#include "prep.cuh"
#include "tribit.h"

struct tribit_context {
  tribit_options opts{};
  int device = 0;
  int num_sms = 148;
  cudaStream_t own = nullptr;
  cudaStream_t st = nullptr;
  tb::Arena arena;
  tb::Prepared prep{};
  tb::Schedule sched{};
  unsigned long long* per_graph = nullptr;
  bool prepared = false;
  tb::LaunchInfo launch{};
  cudaEvent_t ev[6] = {};
  cudaStream_t copy_st = nullptr;                       // host uploads (overlapped with the degree pass)
  cudaEvent_t upload_ev[tb::kUploadChunks + 1] = {};
  tb::DeviceStats* h_stats = nullptr;  // pinned
  // Tuned launch parameters (tribit_set_tuning / tribit_autotune).
  int ctas_per_sm = 0;
  uint32_t piece_width = 64;
  int tile_engine = TRIBIT_TILES_TCGEN05;  // measured faster than mma.sync on dense tiles
  float tile_min_nnz = 64.f;
  float merge_ratio = tb::kDefaultMergeRatio;
  uint32_t tile_wait_polls = 0;        // tcgen05 tiles' bounded mbarrier wait (0: the default budget)
  uint32_t num_graphs = 0;             // batch size of the prepared input (0: single graph)
  cudaGraph_t graph = nullptr;         // captured counting launch (tribit_capture_count)
  cudaGraphExec_t graph_exec = nullptr;
  tb::DeviceModel model{};
  // Matrix Market ingest (tribit_load_mtx): the file's text and its segment
  // counts, the parsed entries, and two pinned upload buffers.
  tb::Arena text_arena;
  tb::Arena load_arena;
  void* pinned[2] = {nullptr, nullptr};
  cudaEvent_t pinned_ev[2] = {};       // the last device copy that used pinned[b], on any stream
  int pinned_turn = 0;                 // the pinned buffer the next staged piece takes
  const uint64_t* loaded_entries = nullptr;
  uint64_t loaded_E = 0, loaded_n = 0;
  bool loaded = false;
  float load_ms = 0.f;
  uint32_t load_gpu_parse = 0;
  // Device memory the context may use (tribit_set_device_budget; 0: what the
  // device has free); graphs needing more are counted in rank ranges.
  uint64_t device_budget = 0;
  uint32_t launch_model = TRIBIT_LAUNCH_AUTO;  // tribit_tuning.launch_model
  int stream_tier = 0;                 // TRIBIT_STREAM_* (tribit_set_stream_options)
  uint64_t stream_range_entries = 0;   // bound on a rank range's entries (0: the budget's)
  tb::Arena stream_arena;              // streamed counts: degrees, ranks, row counts, piece buffers
  void* stream_host = nullptr;         // streamed counts: pinned host row starts and ranks (kept)
  size_t stream_host_bytes = 0;
  tb::Arena train_arena;               // training batches and activations
  tb::Arena timing_arena;              // per-row-block cycle counters
  std::string err;
};

namespace tb {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Runs body, mapping library exceptions to statuses (and the message into
// ctx->err); nothing escapes an extern "C" function.
template <typename F>
tribit_status guarded(tribit_context* ctx, F&& body) {
  try {
    body();
    return TRIBIT_OK;
  } catch (const StatusError& e) {
    if (ctx) ctx->err = e.what();
    return e.status;
  } catch (const CudaError& e) {
    if (ctx) ctx->err = e.what();
    return e.code == cudaErrorMemoryAllocation ? TRIBIT_ERR_OUT_OF_MEMORY : TRIBIT_ERR_CUDA;
  } catch (const std::bad_alloc&) {
    if (ctx) ctx->err = "host allocation failed";
    return TRIBIT_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    if (ctx) ctx->err = e.what();
    return TRIBIT_ERR_INTERNAL;
  }
}

// Rebuilds the context's schedule for its dispatch mode (learned mode runs the
// MLP over full features) with its tuned piece width and tile threshold.
void apply_dispatch(tribit_context* c, cudaStream_t st);

// Device bytes of the context's arena for one count of E entries on n
// vertices in `order` (stage: host input staged on the device).
size_t call_bytes(tribit_context* c, uint64_t E, uint64_t n, int order, bool stage);
// One count of E device entries on n vertices in `order` with the context's
// dispatcher (tribit_count_edges_device with an explicit order).
void count_device_input(tribit_context* c, const uint64_t* d_entries, uint64_t E, uint64_t n, int order,
                        tribit_result* res);
// result.row_blocks, row_blocks_by_variant and hub_edges of the schedule in
// the context (synchronises its stream).
void fill_schedule_stats(tribit_context* c, tribit_result* res);
// Counts host entries in rank ranges when their buffers exceed the device
// budget (stream.cu). Returns false, doing nothing, when they fit.
bool count_streamed_if_needed(tribit_context* c, const uint64_t* host, uint64_t E, uint64_t n, tribit_result* res);
// Copies bytes of host memory to device memory through the context's two
// pinned buffers (host threads fill one while the other's copy runs).
void upload_via_pinned(tribit_context* c, const void* src, size_t bytes, void* dst);
// Whether host memory is pinned (page-locked or registered).
bool host_is_pinned(const void* p);
// HostUpload::stage for pageable host memory (ctx: the context): the bytes go
// through the context's pinned buffers in turn, copied in by host threads
// while the previous piece's copy runs, on stream st.
void stage_pageable(void* ctx, void* dst, const void* src, size_t bytes, cudaStream_t st);

// The host writes or reads pinned buffer b only once the last device copy
// that used it has finished; every such copy is followed by pinned_used.
inline void pinned_wait(tribit_context* c, int b) { TB_CUDA(cudaEventSynchronize(c->pinned_ev[b])); }
inline void pinned_used(tribit_context* c, int b, cudaStream_t s) { TB_CUDA(cudaEventRecord(c->pinned_ev[b], s)); }

// Launch configuration of the context's counting kernels.
inline CountConfig count_config(const tribit_context* c) {
  CountConfig cfg;
  cfg.num_sms = c->num_sms;
  cfg.ctas_per_sm = c->ctas_per_sm;
  if (c->tile_wait_polls) cfg.tile_wait_polls = c->tile_wait_polls;
  cfg.queue = c->launch_model == TRIBIT_LAUNCH_QUEUE ||
              (c->launch_model == TRIBIT_LAUNCH_AUTO && c->prep.E <= kQueueMaxEntries);
  return cfg;
}

// Drops a captured counting graph (the schedule it was captured from changed).
inline void drop_graph(tribit_context* c) {
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  c->graph_exec = nullptr;
  c->graph = nullptr;
}

}  // namespace tb
