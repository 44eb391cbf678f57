// tribit_count_edges_noalloc: the whole count of a small graph without a
// single device allocation.
//
// Who needs it: a caller that cannot allocate device memory while it counts.
// Typical cases are a host process whose framework already owns the device
// memory through its own allocator or a pool reserved up front (the reference
// itself reserves 95% of free HBM in its pool at start-up, tribit.cu:825-838),
// and a latency-sensitive loop that must not pay the implicit device-wide
// synchronisation of cudaMalloc / cudaFree. Such a caller passes device
// buffers for the input entries and for the result; every other buffer the
// pipeline needs comes from one fixed scratch array below.
//
// The scratch is a file-scope __device__ array of kNoAllocScratchBytes
// (32 MiB). Every device on which this module is loaded holds those 32 MiB
// until the process exits. Host code may not use the array's name as a
// device address (on the host it names a host-side shadow), so on the first
// call on each device -- with that device current -- the address is fetched
// with cudaGetSymbolAddress and cached; make that first call before capturing
// any stream work on that device.
//
// All calls on a device share the one array and each call leaves its own
// contents behind; the pipeline clears everything that must start at zero.
// Calls whose GPU work overlaps (two host threads, or two streams without an
// ordering between them) race on the array and give wrong counts: order them
// on one stream or serialise them.
#include <cuda_runtime.h>

#include <mutex>

#include "arena.h"
#include "common.cuh"
#include "count.cuh"
#include "prep.cuh"
#include "tribit.h"

namespace {

constexpr size_t kNoAllocScratchBytes = 32ull << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

static_assert((uint32_t)tb::kErrIdRange == (uint32_t)TRIBIT_NOALLOC_FLAG_ID_RANGE &&
                  (uint32_t)tb::kErrTimeout == (uint32_t)TRIBIT_NOALLOC_FLAG_TIMEOUT,
              "d_result[2] carries the device flags as the header documents them");

__global__ void k_noalloc_result(const tb::DeviceStats* stats, bool hubs, unsigned long long* out) {
  out[0] = stats->triangles;
  out[1] = stats->edges;
  out[2] = stats->err | stats->count_err;
  out[3] = hubs ? 1ull : 0ull;
}

}  // namespace

extern "C" uint64_t tribit_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

extern "C" tribit_status tribit_count_edges_noalloc(const uint64_t* d_entries, uint64_t n_entries, uint64_t num_nodes,
                                                    uint64_t* d_result, void* stream) {
  if ((!d_entries && n_entries) || !d_result) return TRIBIT_ERR_INVALID_ARGUMENT;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return TRIBIT_ERR_NO_DEVICE;
  }
  if (dev < 0 || dev >= kMaxDevices) return TRIBIT_ERR_INVALID_ARGUMENT;
  void* base = nullptr;
  int sms = 0;
  {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
        (void)cudaGetLastError();
        return TRIBIT_ERR_CUDA;
      }
      int s = 0;
      if (cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return TRIBIT_ERR_CUDA;
      }
      g_num_sms[dev] = s;
      g_scratch_addr[dev] = p;
    }
    base = g_scratch_addr[dev];
    sms = g_num_sms[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  try {
    tb::Arena ar;
    ar.attach(base, kNoAllocScratchBytes);
    tb::PrepInput in;
    in.entries = d_entries;
    in.E = n_entries;
    in.n = num_nodes;
    in.order = TRIBIT_ORDER_DEGREE;
    // Layout pass: launches nothing. The merge variant's hub lists (and the
    // full features the plain rule needs to choose merge) when they fit the
    // scratch; else bit tiles and the bitmap sweep only. Rejects graphs that
    // fit neither way.
    bool hubs = true;
    for (;;) {
      ar.begin(true);
      tb::Prepared probe;
      tb::prepare_graph(ar, in, st, &probe);
      (void)tb::take_schedule(ar, num_nodes, n_entries, hubs);
      if (!hubs || ar.used() <= kNoAllocScratchBytes) break;
      hubs = false;
    }
    ar.reserve(ar.used());
    ar.begin(false);
    tb::Prepared prep;
    tb::prepare_graph(ar, in, st, &prep);
    tb::Schedule sched = tb::take_schedule(ar, num_nodes, n_entries, hubs);
    tb::build_schedule(prep.view, sched, TRIBIT_DISPATCH_PLAIN, hubs, st);
    tb::CountConfig cfg;
    cfg.num_sms = sms;
    cfg.queue = true;  // graphs that fit the scratch are small: one queue-driven kernel
    tb::launch_count(prep.view, sched, prep.stats, nullptr, cfg, st);
    k_noalloc_result<<<1, 1, 0, st>>>(prep.stats, hubs, reinterpret_cast<unsigned long long*>(d_result));
    TB_LAUNCH_CHECK();
  } catch (const tb::StatusError& e) {
    return e.status;
  } catch (const tb::CudaError& e) {
    return e.code == cudaErrorMemoryAllocation ? TRIBIT_ERR_OUT_OF_MEMORY : TRIBIT_ERR_CUDA;
  } catch (...) {
    return TRIBIT_ERR_INTERNAL;
  }
  return TRIBIT_OK;
}
