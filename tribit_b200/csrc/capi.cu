// C-ABI entry points (include/tribit.h).
#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>
#include <algorithm>
#include <vector>

#include "context.h"

namespace {

using tb::CudaError;
using tb::DeviceGuard;
using tb::StatusError;
using tb::guarded;

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  TB_CUDA(cudaEventElapsedTime(&ms, a, b));
  return ms;
}

// Device buffers of one call, laid out identically in the measuring pass and
// the real pass.
struct CallLayout {
  uint64_t* staged = nullptr;     // host-input calls: device copy of the entries
  uint64_t* eoff = nullptr;       // batch: entry offsets
  uint64_t* voff = nullptr;       // batch: vertex offsets
  unsigned long long* per_graph = nullptr;
};

void layout(tribit_context* c, bool measure, const tb::PrepInput& in, bool stage, uint32_t G, CallLayout* L) {
  tb::Arena& ar = c->arena;
  ar.begin(measure);
  L->staged = stage ? ar.take<uint64_t>(in.E ? in.E : 1) : nullptr;
  if (G) {
    L->eoff = ar.take<uint64_t>(G + 1);
    L->voff = ar.take<uint64_t>(G + 1);
    L->per_graph = ar.take<unsigned long long>(G);
  }
  tb::PrepInput pin = in;
  if (stage) pin.entries = L->staged;
  if (G) {
    pin.eoff = L->eoff;
    pin.voff = L->voff;
  }
  if (!measure) return;
  // Measuring: walk the same takes prepare_graph / take_schedule will do.
  tb::Prepared tmp;
  tb::prepare_graph(ar, pin, c->st, &tmp);
  (void)tb::take_schedule(ar, in.n, in.E);
}

// Runs preprocessing + schedule (+ counting when count == true) for one input.
void run_call(tribit_context* c, tb::PrepInput in, const uint64_t* host_entries, const uint64_t* host_eoff,
              const uint64_t* host_voff, uint32_t G, bool count, tribit_result* res) {
  DeviceGuard dg(c->device);
  const bool stage = host_entries != nullptr;
  CallLayout L;
  layout(c, true, in, stage, G, &L);
  c->arena.reserve(c->arena.used(), c->device_budget == 0);
  layout(c, false, in, stage, G, &L);
  cudaStream_t st = c->st;
  TB_CUDA(cudaEventRecord(c->ev[0], st));
  if (G) {
    TB_CUDA(cudaMemcpyAsync(L.eoff, host_eoff, (G + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    TB_CUDA(cudaMemcpyAsync(L.voff, host_voff, (G + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    TB_CUDA(cudaMemsetAsync(L.per_graph, 0, G * sizeof(unsigned long long), st));
  }
  tb::PrepInput pin = in;
  if (stage && in.E) {
    // The entries are uploaded by prepare_graph, overlapped with the degree
    // pass; ev[1] marks the moment the last piece has landed.
    pin.upload.host = host_entries;
    pin.upload.copy_stream = c->copy_st;
    pin.upload.events = c->upload_ev;
    pin.upload.uploaded = c->ev[1];
    // Pageable input of at least one 32 MiB staging piece: copied into the
    // context's pinned buffers by host threads rather than by the driver.
    if (in.E * sizeof(uint64_t) >= (32u << 20) && !tb::host_is_pinned(host_entries)) {
      pin.upload.stage = &tb::stage_pageable;
      pin.upload.stage_ctx = c;
    }
  } else {
    TB_CUDA(cudaEventRecord(c->ev[1], st));
  }
  if (stage) pin.entries = L.staged;
  if (G) {
    pin.eoff = L.eoff;
    pin.voff = L.voff;
  }
  tb::drop_graph(c);
  tb::prepare_graph(c->arena, pin, st, &c->prep);
  c->sched = tb::take_schedule(c->arena, in.n, in.E);
  tb::apply_dispatch(c, st);
  c->per_graph = L.per_graph;
  c->num_graphs = G;
  c->prepared = true;
  TB_CUDA(cudaEventRecord(c->ev[2], st));
  if (count) {
    tb::CountConfig cfg = tb::count_config(c);
    c->launch = tb::launch_count(c->prep.view, c->sched, c->prep.stats, L.per_graph, cfg, st);
  }
  TB_CUDA(cudaEventRecord(c->ev[3], st));
  TB_CUDA(cudaMemcpyAsync(c->h_stats, c->prep.stats, sizeof(tb::DeviceStats), cudaMemcpyDeviceToHost, st));
  TB_CUDA(cudaEventRecord(c->ev[4], st));
  TB_CUDA(cudaEventSynchronize(c->ev[4]));
  TB_CUDA(cudaGetLastError());
  const tb::DeviceStats& hs = *c->h_stats;
  if (hs.err & tb::kErrIdRange) throw StatusError(TRIBIT_ERR_ID_RANGE, "an entry names a vertex id >= num_nodes");
  if (hs.count_err & tb::kErrTimeout) throw StatusError(TRIBIT_ERR_TIMEOUT, "a device-side wait gave up");
  if (res) {
    std::memset(res, 0, sizeof *res);
    res->triangles = count ? hs.triangles : 0;
    res->num_nodes = in.n;
    res->entries = in.E;
    res->edges = hs.edges;
    res->blocks_of_threads = count ? c->launch.ctas : 0;
    res->count_kernels = c->launch.kernels;
    res->h2d_ms = elapsed(c->ev[0], c->ev[1]);
    res->preprocess_ms = elapsed(c->ev[1], c->ev[2]);
    res->kernel_ms = count ? elapsed(c->ev[2], c->ev[3]) : 0.f;
    res->total_ms = elapsed(c->ev[0], c->ev[4]);
  }
}

}  // namespace

namespace tb {

size_t call_bytes(tribit_context* c, uint64_t E, uint64_t n, int order, bool stage) {
  tb::PrepInput in;
  in.E = E;
  in.n = n;
  in.order = order;
  CallLayout L;
  layout(c, true, in, stage, 0, &L);
  return c->arena.used();
}

void count_device_input(tribit_context* c, const uint64_t* d_entries, uint64_t E, uint64_t n, int order,
                        tribit_result* res) {
  tb::PrepInput in;
  in.entries = d_entries;
  in.E = E;
  in.n = n;
  in.order = order;
  run_call(c, in, nullptr, nullptr, nullptr, 0, true, res);
}

void fill_schedule_stats(tribit_context* c, tribit_result* res) {
  uint32_t lens[TRIBIT_NUM_VARIANTS], hub_edges = 0;
  TB_CUDA(cudaMemcpyAsync(lens, c->sched.list_len, sizeof lens, cudaMemcpyDeviceToHost, c->st));
  TB_CUDA(cudaMemcpyAsync(&hub_edges, c->sched.piece_off + TRIBIT_NUM_VARIANTS + 4, sizeof hub_edges,
                          cudaMemcpyDeviceToHost, c->st));
  TB_CUDA(cudaStreamSynchronize(c->st));
  res->hub_edges = hub_edges;
  res->row_blocks = 0;
  for (int v = 0; v < TRIBIT_NUM_VARIANTS; ++v) {
    res->row_blocks_by_variant[v] = lens[v];
    res->row_blocks += lens[v];
  }
}

}  // namespace tb

using tb::fill_schedule_stats;

extern "C" {

void tribit_default_options(tribit_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->order = TRIBIT_ORDER_DEGREE;
  o->dispatch = TRIBIT_DISPATCH_PLAIN;
}

const char* tribit_version(void) { return "tribit_b200 0.1.0 (sm_100a)"; }

const char* tribit_status_string(tribit_status s) {
  switch (s) {
    case TRIBIT_OK: return "ok";
    case TRIBIT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case TRIBIT_ERR_IO: return "cannot open or read file";
    case TRIBIT_ERR_FORMAT: return "malformed Matrix Market file";
    case TRIBIT_ERR_NOT_SQUARE: return "matrix is not square";
    case TRIBIT_ERR_ID_RANGE: return "vertex id out of range";
    case TRIBIT_ERR_TOO_LARGE: return "graph exceeds 32-bit limits";
    case TRIBIT_ERR_CUDA: return "CUDA error";
    case TRIBIT_ERR_OUT_OF_MEMORY: return "out of memory";
    case TRIBIT_ERR_NO_DEVICE: return "no CUDA device";
    case TRIBIT_ERR_TIMEOUT: return "device wait timed out";
    case TRIBIT_ERR_NO_MODEL: return "no dispatcher model loaded";
    case TRIBIT_ERR_INTERNAL: return "internal error";
  }
  return "unknown status";
}

const char* tribit_last_error(const tribit_context* ctx) { return ctx ? ctx->err.c_str() : ""; }

tribit_status tribit_create(const tribit_options* opts, tribit_context** out) {
  if (!out) return TRIBIT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  tribit_options o;
  tribit_default_options(&o);
  if (opts) o = *opts;
  if (o.order != TRIBIT_ORDER_DEGREE && o.order != TRIBIT_ORDER_ID) return TRIBIT_ERR_INVALID_ARGUMENT;
  if (o.dispatch < TRIBIT_DISPATCH_PLAIN || o.dispatch > TRIBIT_DISPATCH_MMA) return TRIBIT_ERR_INVALID_ARGUMENT;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    (void)cudaGetLastError();
    return TRIBIT_ERR_NO_DEVICE;
  }
  if (o.device < 0 || o.device >= count) return TRIBIT_ERR_INVALID_ARGUMENT;
  tribit_context* c = new (std::nothrow) tribit_context();
  if (!c) return TRIBIT_ERR_OUT_OF_MEMORY;
  c->opts = o;
  c->device = o.device;
  c->ctas_per_sm = o.ctas_per_sm;
  tribit_status st = guarded(c, [&] {
    DeviceGuard dg(c->device);
    TB_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device));
    TB_CUDA(cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking));
    c->st = c->own;
    for (auto& e : c->ev) TB_CUDA(cudaEventCreate(&e));
    TB_CUDA(cudaStreamCreateWithFlags(&c->copy_st, cudaStreamNonBlocking));
    for (auto& e : c->upload_ev) TB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& e : c->pinned_ev) TB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    TB_CUDA(cudaMallocHost(&c->h_stats, sizeof(tb::DeviceStats)));
  });
  if (st != TRIBIT_OK) {
    tribit_destroy(c);
    return st;
  }
  *out = c;
  return TRIBIT_OK;
}

void tribit_destroy(tribit_context* c) {
  if (!c) return;
  {
    DeviceGuard dg(c->device);
    if (c->st) cudaStreamSynchronize(c->st);
    c->arena.release();
    c->text_arena.release();
    c->stream_arena.release();
    c->load_arena.release();
    for (auto& p : c->pinned)
      if (p) cudaFreeHost(p);
    if (c->stream_host) cudaFreeHost(c->stream_host);
    tb::drop_graph(c);
    c->train_arena.release();
    c->timing_arena.release();
    tb::model_free(c->model);
    for (auto& e : c->ev)
      if (e) cudaEventDestroy(e);
    if (c->copy_st) cudaStreamSynchronize(c->copy_st);
    for (auto& e : c->upload_ev)
      if (e) cudaEventDestroy(e);
    for (auto& e : c->pinned_ev)
      if (e) cudaEventDestroy(e);
    if (c->copy_st) cudaStreamDestroy(c->copy_st);
    if (c->h_stats) cudaFreeHost(c->h_stats);
    if (c->own) cudaStreamDestroy(c->own);
  }
  delete c;
}

tribit_status tribit_set_stream(tribit_context* c, void* stream) {
  if (!c) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    DeviceGuard dg(c->device);
    // Work already queued on the old stream finishes before any later call
    // queues work on the new one (they share the context's buffers).
    if (c->st) TB_CUDA(cudaStreamSynchronize(c->st));
    c->st = stream ? (cudaStream_t)stream : c->own;
  });
}

tribit_status tribit_count_edges(tribit_context* c, const uint64_t* entries, uint64_t n_entries, uint64_t num_nodes,
                                 tribit_result* out) {
  if (!c || (!entries && n_entries)) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    if (entries && tb::count_streamed_if_needed(c, entries, n_entries, num_nodes, out)) return;
    tb::PrepInput in;
    in.E = n_entries;
    in.n = num_nodes;
    in.order = c->opts.order;
    static const uint64_t dummy = 0;
    run_call(c, in, entries ? entries : &dummy, nullptr, nullptr, 0, true, out);
    if (out) {
      fill_schedule_stats(c, out);
      out->stream_ranges = 1;
      out->stream_tasks = 1;
      out->stream_tier = 0;
    }
  });
}

tribit_status tribit_device_bytes(tribit_context* c, uint64_t n_entries, uint64_t num_nodes, uint64_t* bytes) {
  if (!c || !bytes) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] { *bytes = tb::call_bytes(c, n_entries, num_nodes, c->opts.order, true); });
}

tribit_status tribit_count_edges_device(tribit_context* c, const uint64_t* d_entries, uint64_t n_entries,
                                        uint64_t num_nodes, tribit_result* out) {
  if (!c || (!d_entries && n_entries)) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    tb::PrepInput in;
    in.entries = d_entries;
    in.E = n_entries;
    in.n = num_nodes;
    in.order = c->opts.order;
    run_call(c, in, nullptr, nullptr, nullptr, 0, true, out);
    if (out) fill_schedule_stats(c, out);
  });
}

tribit_status tribit_prepare_device(tribit_context* c, const uint64_t* d_entries, uint64_t n_entries,
                                    uint64_t num_nodes, tribit_result* out) {
  if (!c || (!d_entries && n_entries)) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    tb::PrepInput in;
    in.entries = d_entries;
    in.E = n_entries;
    in.n = num_nodes;
    in.order = c->opts.order;
    run_call(c, in, nullptr, nullptr, nullptr, 0, false, out);
    if (out) fill_schedule_stats(c, out);
  });
}

tribit_status tribit_launch_count(tribit_context* c) {
  if (!c) return TRIBIT_ERR_INVALID_ARGUMENT;
  if (!c->prepared) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    DeviceGuard dg(c->device);
    if (c->graph_exec) {
      if (c->num_graphs) TB_CUDA(cudaMemsetAsync(c->per_graph, 0, c->num_graphs * sizeof(unsigned long long), c->st));
      TB_CUDA(cudaGraphLaunch(c->graph_exec, c->st));
      return;
    }
    tb::CountConfig cfg = tb::count_config(c);
    if (c->num_graphs) TB_CUDA(cudaMemsetAsync(c->per_graph, 0, c->num_graphs * sizeof(unsigned long long), c->st));
    c->launch = tb::launch_count(c->prep.view, c->sched, c->prep.stats, c->per_graph, cfg, c->st);
  });
}

tribit_status tribit_capture_count(tribit_context* c) {
  if (!c || !c->prepared) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    DeviceGuard dg(c->device);
    tb::drop_graph(c);
    tb::CountConfig cfg = tb::count_config(c);
    // One ordinary launch first: one-time function attributes are set outside the capture.
    c->launch = tb::launch_count(c->prep.view, c->sched, c->prep.stats, c->per_graph, cfg, c->st);
    TB_CUDA(cudaStreamSynchronize(c->st));
    TB_CUDA(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    try {
      tb::launch_count(c->prep.view, c->sched, c->prep.stats, c->per_graph, cfg, c->st);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(c->st, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    TB_CUDA(cudaStreamEndCapture(c->st, &c->graph));
    TB_CUDA(cudaGraphInstantiate(&c->graph_exec, c->graph, 0));
  });
}

tribit_status tribit_block_variants(tribit_context* c, uint8_t* out, uint64_t cap, uint64_t* num_row_blocks) {
  if (!c || !c->prepared || !num_row_blocks) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    DeviceGuard dg(c->device);
    const uint64_t nrb = c->sched.num_row_blocks;
    *num_row_blocks = nrb;
    if (!out) return;
    if (cap < nrb) throw StatusError(TRIBIT_ERR_INVALID_ARGUMENT, "output buffer too small");
    if (nrb) TB_CUDA(cudaMemcpyAsync(out, c->sched.variant_of, nrb, cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaStreamSynchronize(c->st));
  });
}

tribit_status tribit_read_batch_counts(tribit_context* c, uint64_t* out, uint32_t num_graphs) {
  if (!c || !c->prepared || !out || num_graphs != c->num_graphs || num_graphs == 0) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    DeviceGuard dg(c->device);
    TB_CUDA(cudaMemcpyAsync(out, c->per_graph, num_graphs * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaStreamSynchronize(c->st));
  });
}

tribit_status tribit_get_tuning(tribit_context* c, tribit_tuning* t) {
  if (!c || !t) return TRIBIT_ERR_INVALID_ARGUMENT;
  t->ctas_per_sm = c->ctas_per_sm;
  t->piece_width = c->piece_width;
  t->tile_min_nnz = c->tile_min_nnz;
  t->count_ms = 0.f;
  t->merge_ratio = c->merge_ratio;
  t->launch_model = c->launch_model;
  return TRIBIT_OK;
}

tribit_status tribit_set_tuning(tribit_context* c, const tribit_tuning* t) {
  if (!c || !t || t->ctas_per_sm < 0 || t->ctas_per_sm > 32 || t->piece_width < tb::kMinPieceWidth ||
      t->piece_width % 32 != 0 || t->piece_width > 4096 || !(t->tile_min_nnz >= 0.f) ||
      !(t->merge_ratio >= 0.f) || t->launch_model > TRIBIT_LAUNCH_AUTO)
    return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    c->launch_model = t->launch_model;
    c->ctas_per_sm = t->ctas_per_sm;
    c->piece_width = t->piece_width;
    c->tile_min_nnz = t->tile_min_nnz;
    c->merge_ratio = t->merge_ratio;
    if (c->prepared) {
      DeviceGuard dg(c->device);
      tb::apply_dispatch(c, c->st);
      TB_CUDA(cudaStreamSynchronize(c->st));
    }
  });
}

tribit_status tribit_set_tile_engine(tribit_context* c, int engine) {
  if (!c || (engine != TRIBIT_TILES_MMA_SYNC && engine != TRIBIT_TILES_TCGEN05)) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    c->tile_engine = engine;
    c->sched.tile_engine = engine;
    tb::drop_graph(c);
  });
}

tribit_status tribit_set_tile_wait_polls(tribit_context* c, uint32_t max_polls) {
  if (!c) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    c->tile_wait_polls = max_polls;
    tb::drop_graph(c);
  });
}

tribit_status tribit_test_tile_timeout(tribit_context* c, uint32_t max_polls) {
  if (!c || !c->prepared || max_polls == 0) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    DeviceGuard dg(c->device);
    tb::drop_graph(c);
    tb::CountConfig cfg = tb::count_config(c);
    cfg.tile_wait_polls = max_polls;
    cfg.tile_test_no_commit = 1;
    c->launch = tb::launch_count(c->prep.view, c->sched, c->prep.stats, c->per_graph, cfg, c->st);
  });
}

tribit_status tribit_autotune(tribit_context* c, uint32_t reps, tribit_tuning* best) {
  if (!c || !c->prepared || !best) return TRIBIT_ERR_INVALID_ARGUMENT;
  if (reps == 0) reps = 2;
  static const int kCtas[] = {4, 6, 7, 0};  // 0: the queue kernel (its CTAs per SM are fixed)
  static const uint32_t kWidths[] = {32, 64, 128};
  static const float kTile[] = {64.f, 1e30f};
  tribit_tuning cur{}, found{};
  found.count_ms = 1e30f;
  cur.merge_ratio = c->merge_ratio;  // the plain rule's merge threshold stays as set
  for (int ctas : kCtas)
    for (uint32_t w : kWidths)
      for (float tile : kTile) {
        cur.launch_model = ctas ? TRIBIT_LAUNCH_KERNELS : TRIBIT_LAUNCH_QUEUE;
        cur.ctas_per_sm = ctas;
        cur.piece_width = w;
        cur.tile_min_nnz = tile;
        tribit_status st = tribit_set_tuning(c, &cur);
        if (st != TRIBIT_OK) return st;
        st = guarded(c, [&] {
          DeviceGuard dg(c->device);
          tb::CountConfig cfg = tb::count_config(c);
          tb::launch_count(c->prep.view, c->sched, c->prep.stats, c->per_graph, cfg, c->st);  // warm
          std::vector<float> ms(reps);
          for (uint32_t r = 0; r < reps; ++r) {
            TB_CUDA(cudaEventRecord(c->ev[0], c->st));
            tb::launch_count(c->prep.view, c->sched, c->prep.stats, c->per_graph, cfg, c->st);
            TB_CUDA(cudaEventRecord(c->ev[1], c->st));
            TB_CUDA(cudaEventSynchronize(c->ev[1]));
            ms[r] = elapsed(c->ev[0], c->ev[1]);
          }
          std::sort(ms.begin(), ms.end());
          cur.count_ms = ms[reps / 2];
        });
        if (st != TRIBIT_OK) return st;
        if (cur.count_ms < found.count_ms) found = cur;
      }
  tribit_status st = tribit_set_tuning(c, &found);
  *best = found;
  return st;
}

tribit_status tribit_read_count(tribit_context* c, tribit_result* out) {
  if (!c || !c->prepared) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    DeviceGuard dg(c->device);
    TB_CUDA(cudaMemcpyAsync(c->h_stats, c->prep.stats, sizeof(tb::DeviceStats), cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaStreamSynchronize(c->st));
    TB_CUDA(cudaGetLastError());
    if (c->h_stats->count_err & tb::kErrTimeout) throw StatusError(TRIBIT_ERR_TIMEOUT, "a device-side wait gave up");
    if (out) {
      std::memset(out, 0, sizeof *out);
      out->triangles = c->h_stats->triangles;
      out->num_nodes = c->prep.n;
      out->entries = c->prep.E;
      out->edges = c->h_stats->edges;
      out->blocks_of_threads = c->launch.ctas;
      out->count_kernels = c->launch.kernels;
      fill_schedule_stats(c, out);
    }
  });
}

tribit_status tribit_count_batch(tribit_context* c, const uint64_t* entries, const uint64_t* entry_offsets,
                                 const uint32_t* num_nodes, uint32_t num_graphs, uint64_t* triangles_out,
                                 tribit_result* out) {
  if (!c || !entry_offsets || !num_nodes || !triangles_out || num_graphs == 0) return TRIBIT_ERR_INVALID_ARGUMENT;
  if (entry_offsets[0] != 0) return TRIBIT_ERR_INVALID_ARGUMENT;
  for (uint32_t g = 0; g < num_graphs; ++g)
    if (entry_offsets[g + 1] < entry_offsets[g]) return TRIBIT_ERR_INVALID_ARGUMENT;
  if (!entries && entry_offsets[num_graphs]) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    std::vector<uint64_t> voff(num_graphs + 1, 0);
    for (uint32_t g = 0; g < num_graphs; ++g) voff[g + 1] = voff[g] + num_nodes[g];
    tb::PrepInput in;
    in.E = entry_offsets[num_graphs];
    in.n = voff[num_graphs];
    in.order = c->opts.order;
    in.G = num_graphs;
    static const uint64_t dummy = 0;
    run_call(c, in, entries ? entries : &dummy, entry_offsets, voff.data(), num_graphs, true, out);
    DeviceGuard dg(c->device);
    TB_CUDA(cudaMemcpyAsync(triangles_out, c->per_graph, num_graphs * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaStreamSynchronize(c->st));
    if (out) fill_schedule_stats(c, out);
  });
}

}  // extern "C"
