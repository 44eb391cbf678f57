// Matrix Market ingest on the GPU: tribit_load_mtx / tribit_count_loaded /
// tribit_count_mtx.
//
// The reference reads the file with one std::ifstream on one host thread
// (read_mtx, tribit.cu:228-269), the wall-time floor of every run. Here the
// file's bytes go to HBM as they are read: host threads pread() pieces of the
// file into two pinned buffers in turn while the previous piece's DMA runs,
// and the GPU parses the text where it lands. Two passes over 16 KiB
// segments (one CTA each, the segment plus a 1 KiB halo staged in shared
// memory): the first counts each segment's entries, a device scan places the
// segments, and the second writes the folded words in file order. Only the
// entry count crosses back to the host (to size the graph's buffers).
//
// The GPU takes exactly the lines the host reader's strict form takes (ids
// and numbers separated by blanks, newline right after the last token; blank
// lines skipped) and yields the same words in the same order; self-loops are
// dropped, each entry is folded to (min << 32) | max of the 0-based ids. Any
// other line sets a flag, and the file is read again by the host reader's
// exact token grammar (tribit_read_mtx), so every file gives the reference's
// edge list.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

#include "context.h"
#include "mtx.h"
#include "scan.cuh"

namespace tb {
namespace {

constexpr int kParseThreads = 256;
constexpr uint32_t kParseBytesPerThread = 64;
constexpr uint32_t kParseSeg = kParseThreads * kParseBytesPerThread;  // 16 KiB of text per CTA
constexpr uint32_t kParseHalo = 1024;      // staged past the segment: lines that cross its end
constexpr uint32_t kParseLead = 16;        // staged before it: the byte before its first line start
constexpr uint32_t kParseStage = kParseLead + kParseSeg + kParseHalo;
constexpr size_t kPinnedPiece = 32u << 20;  // bytes per pinned upload buffer (two of them)
constexpr int kReadThreads = 8;

__device__ __forceinline__ bool is_blank(uint8_t ch) { return ch == ' ' || ch == '\t'; }
__device__ __forceinline__ bool is_digit(uint8_t ch) { return (uint8_t)(ch - '0') < 10u; }

// Byte i of the text: from the CTA's staged copy [s0, s1) when inside it,
// else from global memory (lines longer than the halo).
struct Text {
  const uint8_t* st;
  uint64_t s0, s1;
  const uint8_t* g;
  __device__ __forceinline__ uint8_t operator[](uint64_t i) const { return (i >= s0 && i < s1) ? st[i - s0] : g[i]; }
};

// The double grammar of the strict form: [sign] digits [. digits]
// [(e|E) [sign] digits], at least one mantissa digit.
__device__ __forceinline__ bool number_token(const Text& t, uint64_t& q) {
  if (t[q] == '+' || t[q] == '-') ++q;
  int nd = 0;
  while (is_digit(t[q])) ++q, ++nd;
  if (t[q] == '.') {
    ++q;
    while (is_digit(t[q])) ++q, ++nd;
  }
  if (nd == 0) return false;
  if (t[q] == 'e' || t[q] == 'E') {
    ++q;
    if (t[q] == '+' || t[q] == '-') ++q;
    int ne = 0;
    while (is_digit(t[q])) ++q, ++ne;
    if (ne == 0) return false;
  }
  return true;
}

enum { kLineBlank = 0, kLineEntry = 1, kLineOther = 2 };

// The line starting at byte j (which ends at a '\n': the body is followed by
// '\n' padding). kLineEntry sets word and keep (false for a self-loop).
__device__ int parse_line(const Text& t, uint64_t j, uint64_t& word, bool& keep) {
  uint64_t q = j;
  while (is_blank(t[q])) ++q;
  if (t[q] == '\n') return kLineBlank;
  uint32_t ids[2];
  for (int k = 0; k < 2; ++k) {
    if (k) {
      if (!is_blank(t[q])) return kLineOther;
      while (is_blank(t[q])) ++q;
    }
    uint64_t v = 0;
    int nd = 0;
    while (is_digit(t[q])) {
      v = v * 10 + (uint64_t)(t[q] - '0');
      ++q;
      if (++nd > 10) return kLineOther;
    }
    if (nd == 0 || v > 0xffffffffull) return kLineOther;
    ids[k] = (uint32_t)v;
  }
  while (t[q] != '\n') {
    if (!is_blank(t[q])) return kLineOther;
    while (is_blank(t[q])) ++q;
    if (t[q] == '\n') return kLineOther;  // trailing blanks: the reference's value loop crosses the line
    if (!number_token(t, q)) return kLineOther;
  }
  // 1-based ids, folded to (min << 32) | max (tribit.cu:258-267).
  const uint32_t r = ids[0] - 1u, c = ids[1] - 1u;
  keep = r != c;
  word = r < c ? ((uint64_t)r << 32) | c : ((uint64_t)c << 32) | r;
  return kLineEntry;
}

// Stages [s0, s1) of the text in shared memory (16-byte loads; the text
// buffer is padded so that s1 never passes its end).
__device__ __forceinline__ void stage_segment(const uint8_t* __restrict__ text, uint64_t seg0, uint8_t* st,
                                              uint64_t& s0, uint64_t& s1) {
  s0 = seg0 >= kParseLead ? seg0 - kParseLead : 0;
  s1 = seg0 + kParseSeg + kParseHalo;
  const uint4* src = reinterpret_cast<const uint4*>(text + s0);
  uint4* dst = reinterpret_cast<uint4*>(st);
  for (uint32_t i = threadIdx.x; i < (uint32_t)((s1 - s0) / 16); i += blockDim.x) dst[i] = src[i];
}

// Pass 1: kept entries of each segment; bad != 0 if any line is outside the strict form.
__global__ void __launch_bounds__(kParseThreads) k_mtx_count(const uint8_t* __restrict__ text, uint64_t B,
                                                             uint32_t* __restrict__ seg_cnt, unsigned int* bad) {
  __shared__ __align__(16) uint8_t st[kParseStage];
  const uint64_t seg0 = (uint64_t)blockIdx.x * kParseSeg;
  uint64_t s0, s1;
  stage_segment(text, seg0, st, s0, s1);
  __syncthreads();
  const Text t{st, s0, s1, text};
  const uint64_t j0 = seg0 + (uint64_t)threadIdx.x * kParseBytesPerThread;
  const uint64_t j1 = j0 + kParseBytesPerThread < B ? j0 + kParseBytesPerThread : B;
  uint32_t cnt = 0;
  bool other = false;
  for (uint64_t j = j0; j < j1; ++j) {
    if (j > 0 && t[j - 1] != '\n') continue;
    uint64_t w;
    bool keep = false;
    const int k = parse_line(t, j, w, keep);
    other |= k == kLineOther;
    cnt += (k == kLineEntry && keep) ? 1u : 0u;
  }
  if (__syncthreads_or(other ? 1 : 0) && threadIdx.x == 0) atomicOr(bad, 1u);
  uint32_t tot;
  (void)block_exclusive_scan<uint32_t>(cnt, OpSum{}, 0u, &tot);
  if (threadIdx.x == 0) seg_cnt[blockIdx.x] = tot;
}

// Pass 2: the segment's words at seg_off[segment], in file order. Each
// thread parses its lines twice (from shared memory): once to count them for
// the CTA's scan, once to write them at their places.
__global__ void __launch_bounds__(kParseThreads) k_mtx_write(const uint8_t* __restrict__ text, uint64_t B,
                                                             const uint32_t* __restrict__ seg_off,
                                                             uint64_t* __restrict__ out) {
  __shared__ __align__(16) uint8_t st[kParseStage];
  const uint64_t seg0 = (uint64_t)blockIdx.x * kParseSeg;
  uint64_t s0, s1;
  stage_segment(text, seg0, st, s0, s1);
  __syncthreads();
  const Text t{st, s0, s1, text};
  const uint64_t j0 = seg0 + (uint64_t)threadIdx.x * kParseBytesPerThread;
  const uint64_t j1 = j0 + kParseBytesPerThread < B ? j0 + kParseBytesPerThread : B;
  uint32_t cnt = 0;
  for (uint64_t j = j0; j < j1; ++j) {
    if (j > 0 && t[j - 1] != '\n') continue;
    uint64_t w;
    bool keep = false;
    cnt += (parse_line(t, j, w, keep) == kLineEntry && keep) ? 1u : 0u;
  }
  uint32_t tot;
  const uint32_t ex = block_exclusive_scan<uint32_t>(cnt, OpSum{}, 0u, &tot);
  uint64_t* dst = out + (uint64_t)seg_off[blockIdx.x] + ex;
  for (uint64_t j = j0; j < j1; ++j) {
    if (j > 0 && t[j - 1] != '\n') continue;
    uint64_t w;
    bool keep = false;
    if (parse_line(t, j, w, keep) == kLineEntry && keep) *dst++ = w;
  }
}

struct FileMap {
  int fd = -1;
  const char* p = nullptr;
  size_t len = 0;
  ~FileMap() {
    if (p && len) munmap((void*)p, len);
    if (fd >= 0) close(fd);
  }
};

// Reads [off, off + len) of the file into dst with up to kReadThreads threads.
bool read_piece(int fd, char* dst, uint64_t off, size_t len) {
  const int nt = (int)std::max<size_t>(1, std::min<size_t>(kReadThreads, len >> 20));
  std::vector<std::thread> th;
  std::vector<char> ok(nt, 1);
  const size_t share = (len + nt - 1) / nt;
  auto work = [&](int k) {
    size_t a = k * share, b = std::min(len, a + share);
    while (a < b) {
      const ssize_t r = pread(fd, dst + a, b - a, (off_t)(off + a));
      if (r <= 0) {
        ok[k] = 0;
        return;
      }
      a += (size_t)r;
    }
  };
  for (int k = 1; k < nt; ++k) th.emplace_back(work, k);
  work(0);
  for (auto& x : th) x.join();
  return std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; });
}

// The text buffer and the segment counts (segs + 1 offsets, then the
// strict-form flag) in the context's text arena.
uint8_t* text_buffer(tribit_context* c, uint64_t text_bytes, uint64_t segs, uint32_t** seg, uint32_t** seg_tmp) {
  Arena& ar = c->text_arena;
  for (int pass = 0; pass < 2; ++pass) {
    ar.begin(pass == 0);
    uint8_t* t = ar.take<uint8_t>(text_bytes);
    uint32_t* s = ar.take<uint32_t>(segs + 2);
    uint32_t* stmp = take_scan_temp<uint32_t>(ar, segs + 1);
    if (pass == 0) {
      ar.reserve(ar.used());
      continue;
    }
    *seg = s;
    *seg_tmp = stmp;
    return t;
  }
  return nullptr;
}

// The loaded graph's device input: `words` entries in the context's load arena.
uint64_t* loaded_buffer(tribit_context* c, uint64_t words) {
  Arena& ar = c->load_arena;
  ar.begin(true);
  ar.take<uint64_t>(words ? words : 1);
  ar.reserve(ar.used());
  ar.begin(false);
  return ar.take<uint64_t>(words ? words : 1);
}

}  // namespace
}  // namespace tb

using tb::DeviceGuard;
using tb::guarded;
using tb::StatusError;

extern "C" {

tribit_status tribit_load_mtx(tribit_context* c, const char* path, uint64_t* num_nodes, uint64_t* n_entries) {
  if (!c || !path) return TRIBIT_ERR_INVALID_ARGUMENT;
  const auto t0 = std::chrono::steady_clock::now();
  tb::FileMap f;
  f.fd = open(path, O_RDONLY);
  if (f.fd < 0) return TRIBIT_ERR_IO;
  struct stat sb;
  if (fstat(f.fd, &sb) != 0) return TRIBIT_ERR_IO;
  f.len = (size_t)sb.st_size;
  if (f.len > 0) {
    void* q = mmap(nullptr, f.len, PROT_READ, MAP_PRIVATE, f.fd, 0);
    if (q == MAP_FAILED) return TRIBIT_ERR_IO;
    f.p = (const char*)q;
  }
  const char* body = nullptr;
  uint64_t n = 0, nnz = 0;
  tribit_status hs = tb::mtx_header(f.p, f.p + f.len, &body, &n, &nnz);
  if (hs != TRIBIT_OK) return hs;
  (void)nnz;  // the entry grammar reads every line whatever the declared count
  const uint64_t off0 = (uint64_t)(body - f.p), B = (uint64_t)f.len - off0;
  c->loaded = false;
  tribit_status st = guarded(c, [&] {
    DeviceGuard dg(c->device);
    const uint64_t segs = tb::ceil_div<uint64_t>(B, tb::kParseSeg);
    // Text plus '\n' padding: every line ends inside it, and the staging of
    // the last segment (plus its halo) stays inside it.
    const uint64_t text_bytes = (segs + 1) * tb::kParseSeg + tb::kParseHalo + 64;
    uint32_t *seg = nullptr, *seg_tmp = nullptr;
    uint8_t* text = tb::text_buffer(c, text_bytes, segs, &seg, &seg_tmp);
    cudaStream_t s = c->st;
    TB_CUDA(cudaMemsetAsync(text + B, '\n', text_bytes - B, s));
    if (!c->pinned[0])
      for (auto& p : c->pinned) TB_CUDA(cudaMallocHost(&p, tb::kPinnedPiece));
    // Pieces of the body: read into pinned buffer k & 1 while the previous
    // piece's copy runs; a buffer is refilled once its copy has finished.
    TB_CUDA(cudaEventRecord(c->upload_ev[0], s));
    TB_CUDA(cudaStreamWaitEvent(c->copy_st, c->upload_ev[0], 0));
    bool io_ok = true;
    uint64_t k = 0;
    for (uint64_t at = 0; at < B; at += tb::kPinnedPiece, ++k) {
      const size_t len = (size_t)std::min<uint64_t>(tb::kPinnedPiece, B - at);
      const int b = (int)(k & 1);
      char* buf = static_cast<char*>(c->pinned[b]);
      tb::pinned_wait(c, b);
      if (!tb::read_piece(f.fd, buf, off0 + at, len)) {
        io_ok = false;
        break;
      }
      TB_CUDA(cudaMemcpyAsync(text + at, buf, len, cudaMemcpyHostToDevice, c->copy_st));
      tb::pinned_used(c, b, c->copy_st);
    }
    TB_CUDA(cudaEventRecord(c->upload_ev[3], c->copy_st));
    TB_CUDA(cudaStreamWaitEvent(s, c->upload_ev[3], 0));
    if (!io_ok) {
      TB_CUDA(cudaStreamSynchronize(s));
      throw StatusError(TRIBIT_ERR_IO, "reading the file failed");
    }
    uint64_t total = 0;
    bool strict = true;
    if (segs) {
      unsigned int* bad = seg + segs + 1;
      TB_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned int), s));
      tb::k_mtx_count<<<(unsigned)segs, tb::kParseThreads, 0, s>>>(text, B, seg, bad);
      TB_LAUNCH_CHECK();
      uint32_t h[2] = {0, 0};
      TB_CUDA(cudaMemcpyAsync(&h[1], bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      tb::device_scan<uint32_t, tb::OpSum>(seg, seg, segs + 1, true, tb::OpSum{}, 0u, seg_tmp, s);
      TB_CUDA(cudaMemcpyAsync(&h[0], seg + segs, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      TB_CUDA(cudaStreamSynchronize(s));
      total = h[0];
      strict = h[1] == 0;
    }
    uint64_t* words = nullptr;
    if (strict) {
      words = tb::loaded_buffer(c, total);
      if (segs) {
        tb::k_mtx_write<<<(unsigned)segs, tb::kParseThreads, 0, s>>>(text, B, seg, words);
        TB_LAUNCH_CHECK();
      }
      c->load_gpu_parse = 1;
    } else {
      // A line outside the strict form: the exact token grammar on the host.
      uint64_t hn = 0, he = 0;
      uint64_t* host = nullptr;
      const tribit_status rs = tribit_read_mtx(path, &hn, &host, &he);
      if (rs != TRIBIT_OK) throw StatusError(rs, "host reader failed");
      struct Free {
        uint64_t* p;
        ~Free() { tribit_free_host(p); }
      } fr{host};
      words = tb::loaded_buffer(c, he);
      TB_CUDA(cudaMemcpyAsync(words, host, he * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
      total = he;
      c->load_gpu_parse = 0;
    }
    TB_CUDA(cudaStreamSynchronize(s));
    c->loaded_entries = words;
    c->loaded_E = total;
    c->loaded_n = n;
    c->loaded = true;
  });
  if (st != TRIBIT_OK) return st;
  c->load_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (num_nodes) *num_nodes = n;
  if (n_entries) *n_entries = c->loaded_E;
  return TRIBIT_OK;
}

tribit_status tribit_count_loaded(tribit_context* c, tribit_result* out) {
  if (!c || !c->loaded) return TRIBIT_ERR_INVALID_ARGUMENT;
  tribit_status st = tribit_count_edges_device(c, c->loaded_entries, c->loaded_E, c->loaded_n, out);
  if (st == TRIBIT_OK && out) {
    out->load_ms = c->load_ms;
    out->load_gpu_parse = c->load_gpu_parse;
  }
  return st;
}

tribit_status tribit_loaded_entries(tribit_context* c, uint64_t* out, uint64_t cap, uint64_t* n_entries) {
  if (!c || !c->loaded || !n_entries) return TRIBIT_ERR_INVALID_ARGUMENT;
  *n_entries = c->loaded_E;
  if (!out) return TRIBIT_OK;
  if (cap < c->loaded_E) return TRIBIT_ERR_INVALID_ARGUMENT;
  return guarded(c, [&] {
    DeviceGuard dg(c->device);
    if (c->loaded_E)
      TB_CUDA(cudaMemcpyAsync(out, c->loaded_entries, c->loaded_E * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->st));
    TB_CUDA(cudaStreamSynchronize(c->st));
  });
}

tribit_status tribit_count_mtx(tribit_context* c, const char* path, tribit_result* out) {
  uint64_t n = 0, e = 0;
  tribit_status st = tribit_load_mtx(c, path, &n, &e);
  if (st != TRIBIT_OK) return st;
  return tribit_count_loaded(c, out);
}

}  // extern "C"
