// WebGraph BVGraph input: tribit_read_bvgraph / tribit_count_bvgraph.
//
// The reference's multi-GPU loader reads the LAW web graphs with the Rust
// webgraph crate (BvGraphSeq::with_basename(..).load(),
// src/multi_gpu/src/main.rs:88) and folds every arc (src, dst), src != dst, to
// (min << 32) | max (main.rs:142-161). This is a C++ reader of the same
// format (Boldi and Vigna, "The WebGraph Framework I: Compression
// Techniques", WWW 2004): basename.properties (nodes, arcs, windowsize,
// maxrefcount, minintervallength, zetak, compressionflags), basename.graph
// (big-endian bit stream of every node's successor list) and, when present,
// basename.offsets (gamma-coded bit offset of every node).
//
// With offsets the nodes are cut into ranges decoded on all host threads: a
// range starting at node s is decoded from s - windowsize * maxrefcount on
// (every node a list of [s, e) copies from, through references, lies there),
// each node from its own bit offset, so a node whose references reach below
// the warm-up start is decoded wrongly without disturbing the next one, and
// is never used. Without offsets the file is decoded in one pass.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "tribit.h"

namespace {

enum Code { kGamma, kDelta, kUnary, kZeta, kBad };

struct Props {
  uint64_t nodes = 0, arcs = 0;
  int window = 7, maxref = 3, minint = 4, zetak = 3;
  Code outdeg = kGamma, refs = kUnary, blocks = kGamma, intervals = kGamma, residuals = kZeta, offsets = kGamma;
};

struct Mapped {
  int fd = -1;
  const uint8_t* p = nullptr;
  size_t len = 0;
  ~Mapped() {
    if (p && len) munmap((void*)p, len);
    if (fd >= 0) close(fd);
  }
  bool open_file(const std::string& path) {
    fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) return false;
    struct stat sb;
    if (fstat(fd, &sb) != 0) return false;
    len = (size_t)sb.st_size;
    if (len) {
      void* q = mmap(nullptr, len, PROT_READ, MAP_PRIVATE, fd, 0);
      if (q == MAP_FAILED) {
        len = 0;
        return false;
      }
      p = (const uint8_t*)q;
    }
    return true;
  }
};

// Big-endian bit reader (most significant bit of each byte first). Reads past
// the end see zero bits and set `over`, which the caller turns into an error.
struct Bits {
  const uint8_t* p;
  uint64_t nbits;
  uint64_t pos = 0;
  bool over = false;

  // The 64 bits from `pos` on, as an integer whose top bit is the bit at pos.
  uint64_t peek64() const {
    const uint64_t byte = pos >> 3;
    const uint64_t nbytes = (nbits + 7) >> 3;
    uint64_t w = 0;
    if (byte + 8 <= nbytes) {
      std::memcpy(&w, p + byte, 8);
      w = __builtin_bswap64(w);
    } else {
      for (int k = 0; k < 8; ++k) w = (w << 8) | (byte + k < nbytes ? p[byte + k] : 0u);
    }
    return w << (pos & 7);
  }
  void skip(uint64_t k) {
    pos += k;
    if (pos > nbits) over = true;
  }
  uint64_t bits(int k) {  // k <= 56
    if (k == 0) return 0;
    const uint64_t v = peek64() >> (64 - k);
    skip((uint64_t)k);
    return v;
  }
  uint64_t bits_long(int k) {  // k <= 64
    if (k <= 56) return bits(k);
    const uint64_t hi = bits(k - 32);
    return (hi << 32) | bits(32);
  }
  uint64_t unary() {  // zeros before the next one
    uint64_t x = 0;
    for (;;) {
      if (pos >= nbits) {
        over = true;
        return x;
      }
      // The top 64 - (pos & 7) bits of the window are stream bits, the rest zeros.
      const uint64_t w = peek64();
      if (w) {
        const int z = __builtin_clzll(w);
        skip((uint64_t)z + 1);
        return x + (uint64_t)z;
      }
      const uint64_t valid = 64 - (pos & 7);
      x += valid;
      skip(valid);
    }
  }
  uint64_t gamma() {
    const uint64_t m = unary();
    if (m > 63) return over = true, 0;
    return ((1ull << m) | bits_long((int)m)) - 1;
  }
  uint64_t delta() {
    const uint64_t m = gamma();
    if (m > 63) return over = true, 0;
    return ((1ull << m) | bits_long((int)m)) - 1;
  }
  uint64_t zeta(int k) {
    const uint64_t h = unary();
    if (h * (uint64_t)k + k > 63) return over = true, 0;
    const uint64_t left = 1ull << (h * k);
    const uint64_t m = bits_long((int)(h * k + k - 1));
    if (m < left) return m + left - 1;
    return (m << 1) + bits(1) - 1;
  }
  uint64_t read(Code c, int k) {
    switch (c) {
      case kGamma: return gamma();
      case kDelta: return delta();
      case kUnary: return unary();
      case kZeta: return zeta(k);
      default: over = true; return 0;
    }
  }
};

inline int64_t unnat(uint64_t x) { return (x & 1) ? -(int64_t)((x + 1) >> 1) : (int64_t)(x >> 1); }

Code code_of(const std::string& s) {
  if (s == "GAMMA") return kGamma;
  if (s == "DELTA") return kDelta;
  if (s == "UNARY") return kUnary;
  if (s == "ZETA") return kZeta;
  return kBad;  // NIBBLE and anything else: not supported
}

tribit_status read_props(const std::string& base, Props* pr) {
  std::ifstream f(base + ".properties");
  if (!f) return TRIBIT_ERR_IO;
  std::map<std::string, std::string> kv;
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#' || line[0] == '!') continue;
    const size_t eq = line.find_first_of("=:");
    if (eq == std::string::npos) continue;
    auto trim = [](std::string s) {
      const size_t a = s.find_first_not_of(" \t\r"), b = s.find_last_not_of(" \t\r");
      return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
    };
    kv[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
  }
  auto num = [&](const char* key, int64_t dflt, int64_t* out) -> bool {
    auto it = kv.find(key);
    if (it == kv.end()) return *out = dflt, true;
    char* end = nullptr;
    const long long v = std::strtoll(it->second.c_str(), &end, 10);
    if (!end || *end || it->second.empty()) return false;
    return *out = v, true;
  };
  int64_t nodes = -1, arcs = 0, w = 7, mr = 3, mi = 4, zk = 3;
  if (!num("nodes", -1, &nodes) || nodes < 0 || !num("arcs", 0, &arcs) || !num("windowsize", 7, &w) ||
      !num("maxrefcount", 3, &mr) || !num("minintervallength", 4, &mi) || !num("zetak", 3, &zk))
    return TRIBIT_ERR_FORMAT;
  if (w < 0 || mi < 0 || zk < 1 || zk > 16) return TRIBIT_ERR_FORMAT;
  auto e = kv.find("endianness");
  if (e != kv.end() && e->second != "big") return TRIBIT_ERR_FORMAT;  // little-endian streams: not supported
  pr->nodes = (uint64_t)nodes;
  pr->arcs = (uint64_t)arcs;
  pr->window = (int)w;
  pr->maxref = (int)mr;
  pr->minint = (int)mi;
  pr->zetak = (int)zk;
  auto f2 = kv.find("compressionflags");
  if (f2 != kv.end()) {
    std::string s = f2->second;
    size_t at = 0;
    while (at <= s.size()) {
      size_t bar = s.find('|', at);
      if (bar == std::string::npos) bar = s.size();
      std::string flag = s.substr(at, bar - at);
      flag.erase(std::remove_if(flag.begin(), flag.end(), [](char ch) { return ch == ' ' || ch == '\t'; }),
                 flag.end());
      at = bar + 1;
      if (flag.empty()) continue;
      const size_t us = flag.find('_');
      if (us == std::string::npos) return TRIBIT_ERR_FORMAT;
      const std::string what = flag.substr(0, us);
      const Code c = code_of(flag.substr(us + 1));
      if (c == kBad) return TRIBIT_ERR_FORMAT;
      if (what == "OUTDEGREES") pr->outdeg = c;
      else if (what == "REFERENCES") pr->refs = c;
      else if (what == "BLOCKS") pr->blocks = c;
      else if (what == "INTERVALS") pr->intervals = c;
      else if (what == "RESIDUALS") pr->residuals = c;
      else if (what == "OFFSETS") pr->offsets = c;
      else return TRIBIT_ERR_FORMAT;
    }
  }
  return TRIBIT_OK;
}

// Decodes nodes [from, to) in order (the window keeps the lists of the last
// `window` nodes), appending the words of nodes >= emit_from to out. With
// offs every node starts at its own offset, and a node whose list cannot be
// decoded -- a warm-up node referring below `from` -- is only marked invalid;
// nodes >= emit_from never depend on one (their reference chains stay within
// windowsize * maxrefcount). Returns false on a bad stream for an emitted node.
bool decode_range(const Props& pr, const uint8_t* data, uint64_t nbits, const uint64_t* offs, uint64_t from,
                  uint64_t to, uint64_t emit_from, std::vector<uint64_t>& out) {
  const int W = pr.window;
  const size_t slots = (size_t)W + 1;
  std::vector<std::vector<uint32_t>> win(slots);
  std::vector<uint64_t> win_node(slots, ~0ull);
  std::vector<char> win_ok(slots, 0);
  std::vector<uint32_t> copied, extra;
  Bits b{data, nbits};
  b.pos = offs ? offs[from] : 0;
  // One node's list into mine; false if the stream or its reference is bad.
  auto node = [&](uint64_t x, std::vector<uint32_t>& mine) -> bool {
    mine.clear();
    const uint64_t d = b.read(pr.outdeg, pr.zetak);
    if (b.over) return false;
    if (d == 0) return true;
    if (d > pr.nodes) return false;
    uint64_t r = 0;
    if (W > 0) r = b.read(pr.refs, pr.zetak);
    if (b.over || r > (uint64_t)W || r > x) return false;
    copied.clear();
    if (r > 0) {
      const uint64_t y = x - r;
      const size_t ys = (size_t)(y % slots);
      if (win_node[ys] != y || !win_ok[ys]) return false;
      const std::vector<uint32_t>& ref = win[ys];
      const uint64_t nb = b.read(pr.blocks, pr.zetak);
      uint64_t i = 0;
      bool copying = true;
      for (uint64_t k = 0; k < nb && !b.over; ++k) {
        const uint64_t len = b.read(pr.blocks, pr.zetak) + (k == 0 ? 0 : 1);
        if (i + len > ref.size()) return false;
        if (copying) copied.insert(copied.end(), ref.begin() + (ptrdiff_t)i, ref.begin() + (ptrdiff_t)(i + len));
        i += len;
        copying = !copying;
      }
      if (copying) copied.insert(copied.end(), ref.begin() + (ptrdiff_t)i, ref.end());
    }
    if (b.over || copied.size() > d) return false;
    uint64_t left_over = d - copied.size();
    extra.clear();
    if (left_over > 0 && pr.minint > 0) {
      const uint64_t ic = b.read(pr.intervals, pr.zetak);
      int64_t prev = 0;
      for (uint64_t k = 0; k < ic && !b.over; ++k) {
        const int64_t left = k == 0 ? (int64_t)x + unnat(b.read(pr.intervals, pr.zetak))
                                    : prev + (int64_t)b.read(pr.intervals, pr.zetak) + 1;
        const uint64_t len = b.read(pr.intervals, pr.zetak) + (uint64_t)pr.minint;
        if (left < 0 || len > left_over || (uint64_t)left + len > pr.nodes) return false;
        for (uint64_t t = 0; t < len; ++t) extra.push_back((uint32_t)(left + (int64_t)t));
        prev = left + (int64_t)len;
        left_over -= len;
      }
    }
    int64_t prev = 0;
    for (uint64_t k = 0; k < left_over && !b.over; ++k) {
      const int64_t y = k == 0 ? (int64_t)x + unnat(b.read(pr.residuals, pr.zetak))
                               : prev + (int64_t)b.read(pr.residuals, pr.zetak) + 1;
      if (y < 0 || (uint64_t)y >= pr.nodes) return false;
      extra.push_back((uint32_t)y);
      prev = y;
    }
    if (b.over) return false;
    // The list: the copied part, intervals and residuals, merged.
    std::sort(extra.begin(), extra.end());
    mine.resize(copied.size() + extra.size());
    std::merge(copied.begin(), copied.end(), extra.begin(), extra.end(), mine.begin());
    return true;
  };
  for (uint64_t x = from; x < to; ++x) {
    if (offs) {
      b.pos = offs[x];
      b.over = false;
    }
    const size_t xs = (size_t)(x % slots);
    win_node[xs] = x;
    const bool ok = node(x, win[xs]);
    win_ok[xs] = ok ? 1 : 0;
    if (!ok) {
      if (x >= emit_from || !offs) return false;
      continue;
    }
    if (x >= emit_from) {
      // main.rs:142-161: (min << 32) | max of every arc, self-loops dropped.
      for (uint32_t y : win[xs])
        if (y != x) out.push_back(y < x ? ((uint64_t)y << 32) | x : ((uint64_t)x << 32) | y);
    }
  }
  return true;
}

// basename.offsets -> nodes + 1 bit offsets; false when absent or short.
bool read_offsets(const std::string& base, const Props& pr, uint64_t nbits, std::vector<uint64_t>& offs) {
  Mapped m;
  if (!m.open_file(base + ".offsets") || (m.len == 0 && pr.nodes > 0)) return false;
  Bits b{m.p, (uint64_t)m.len * 8};
  offs.resize(pr.nodes + 1);
  uint64_t at = 0;
  for (uint64_t x = 0; x <= pr.nodes; ++x) {
    at += b.read(pr.offsets, pr.zetak);
    if (b.over || at > nbits) return false;
    offs[x] = at;
  }
  return true;
}

}  // namespace

extern "C" tribit_status tribit_read_bvgraph(const char* basename, uint64_t* num_nodes, uint64_t** entries,
                                             uint64_t* n_entries) {
  if (!basename || !num_nodes || !entries || !n_entries) return TRIBIT_ERR_INVALID_ARGUMENT;
  *entries = nullptr;
  *n_entries = 0;
  const std::string base(basename);
  Props pr;
  tribit_status st = read_props(base, &pr);
  if (st != TRIBIT_OK) return st;
  if (pr.nodes > 0xffffffffull) return TRIBIT_ERR_TOO_LARGE;
  Mapped g;
  if (!g.open_file(base + ".graph")) return TRIBIT_ERR_IO;
  const uint64_t nbits = (uint64_t)g.len * 8;
  try {
    std::vector<uint64_t> offs;
    const bool have_offs = pr.nodes > 0 && read_offsets(base, pr, nbits, offs);
    unsigned hw = std::thread::hardware_concurrency();
    int threads = (int)std::max(1u, std::min(hw ? hw : 1u, 64u));
    if (!have_offs || pr.nodes < 4096 || pr.maxref < 0) threads = 1;
    std::vector<std::vector<uint64_t>> parts(threads);
    std::atomic<bool> ok{true};
    const uint64_t warm = (uint64_t)pr.window * (uint64_t)std::max(pr.maxref, 0);
    auto work = [&](int t) {
      const uint64_t s = pr.nodes * t / threads, e = pr.nodes * (t + 1) / threads;
      parts[t].reserve((size_t)(pr.arcs / threads + 16));
      const uint64_t from = threads == 1 ? 0 : (s > warm ? s - warm : 0);
      if (!decode_range(pr, g.p, nbits, have_offs ? offs.data() : nullptr, from, e, s, parts[t])) ok = false;
    };
    if (threads == 1) {
      work(0);
    } else {
      std::vector<std::thread> th;
      for (int t = 0; t < threads; ++t) th.emplace_back(work, t);
      for (auto& x : th) x.join();
    }
    if (!ok) return TRIBIT_ERR_FORMAT;
    uint64_t total = 0;
    for (auto& p : parts) total += p.size();
    uint64_t* buf = (uint64_t*)std::malloc(std::max<uint64_t>(total, 1) * sizeof(uint64_t));
    if (!buf) return TRIBIT_ERR_OUT_OF_MEMORY;
    uint64_t at = 0;
    for (auto& p : parts) {
      if (!p.empty()) std::memcpy(buf + at, p.data(), p.size() * sizeof(uint64_t));
      at += p.size();
    }
    *num_nodes = pr.nodes;
    *entries = buf;
    *n_entries = total;
  } catch (const std::bad_alloc&) {
    return TRIBIT_ERR_OUT_OF_MEMORY;
  }
  return TRIBIT_OK;
}

extern "C" tribit_status tribit_count_bvgraph(tribit_context* ctx, const char* basename, tribit_result* out) {
  if (!ctx || !basename) return TRIBIT_ERR_INVALID_ARGUMENT;
  uint64_t n = 0, ne = 0;
  uint64_t* e = nullptr;
  tribit_status st = tribit_read_bvgraph(basename, &n, &e, &ne);
  if (st != TRIBIT_OK) return st;
  st = tribit_count_edges(ctx, e, ne, n, out);
  std::free(e);
  return st;
}
