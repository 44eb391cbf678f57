// Matrix Market reader with the reference's semantics (read_mtx,
// src/single_gpu/tribit.cu:228-269), made fast.
//
// The reference reads with std::ifstream: getline for the banner, getline to
// skip lines starting with '%', a stringstream for "rows cols nnz", then
// `file >> r >> c` and, while the next character is neither '\n' nor EOF,
// `file >> double` to skip values. That token grammar has quirks this reader
// keeps so that every input yields the reference's edge list: whitespace
// other than '\n' after a line's last token makes the value loop consume the
// next line's tokens as values; a token that is not a number ends the entry
// list; a '-' in an id wraps modulo 2^32.
//
// Fast path: the entry section is split across host threads at line breaks
// and parsed in parallel when every entry line is "ids and numbers separated by
// spaces or tabs, newline right after the last token". Any other line sends
// the whole file to the exact sequential token grammar.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "mtx.h"
#include "tribit.h"

namespace {

struct Mapped {
  const char* p = nullptr;
  size_t len = 0;
  int fd = -1;
  ~Mapped() {
    if (p && len) munmap((void*)p, len);
    if (fd >= 0) close(fd);
  }
};

inline bool is_ws(char ch) { return std::isspace((unsigned char)ch) != 0; }

// ---- exact sequential grammar ---------------------------------------------

struct Stream {
  const char* p;
  const char* end;
  bool fail = false;
  int peek() const { return p < end ? (unsigned char)*p : -1; }
  void skip_ws() {
    while (p < end && is_ws(*p)) ++p;
  }
  // operator>>(unsigned int&) of libstdc++.
  bool read_u32(uint32_t* out) {
    if (fail) return false;
    skip_ws();
    bool neg = false;
    if (p < end && (*p == '+' || *p == '-')) neg = *p++ == '-';
    uint64_t v = 0;
    int nd = 0;
    bool ovf = false;
    while (p < end && *p >= '0' && *p <= '9') {
      v = v * 10 + (uint64_t)(*p++ - '0');
      if (v > 0xffffffffull) ovf = true, v = 0xffffffffull;
      ++nd;
    }
    if (nd == 0 || ovf) return !(fail = true);
    *out = neg ? (uint32_t)(0u - (uint32_t)v) : (uint32_t)v;
    return true;
  }
  // operator>>(double&): [sign] digits [. digits] [(e|E) [sign] digits].
  bool read_double() {
    if (fail) return false;
    skip_ws();
    const char* q = p;
    if (q < end && (*q == '+' || *q == '-')) ++q;
    int nd = 0;
    while (q < end && std::isdigit((unsigned char)*q)) ++q, ++nd;
    if (q < end && *q == '.') {
      ++q;
      while (q < end && std::isdigit((unsigned char)*q)) ++q, ++nd;
    }
    if (nd == 0) return !(fail = true);
    if (q < end && (*q == 'e' || *q == 'E')) {
      const char* e = q + 1;
      if (e < end && (*e == '+' || *e == '-')) ++e;
      int ne = 0;
      while (e < end && std::isdigit((unsigned char)*e)) ++e, ++ne;
      if (ne == 0) return !(fail = true);
      q = e;
    }
    p = q;
    return true;
  }
};

inline bool fold(uint32_t r, uint32_t c, uint64_t* out) {
  r -= 1;
  c -= 1;
  if (c < r) {
    *out = ((uint64_t)c << 32) | r;
    return true;
  }
  if (r < c) {
    *out = ((uint64_t)r << 32) | c;
    return true;
  }
  return false;
}

void parse_exact(const char* p, const char* end, std::vector<uint64_t>& out) {
  Stream s{p, end};
  uint32_t r, c;
  while (s.read_u32(&r) && s.read_u32(&c)) {
    while (s.peek() != '\n' && s.peek() != -1)
      if (!s.read_double()) break;
    uint64_t z;
    if (fold(r, c, &z)) out.push_back(z);
  }
}

// ---- strict per-line fast path --------------------------------------------

inline bool number_token(const char*& q, const char* end) {  // double grammar, q at token start
  if (q < end && (*q == '+' || *q == '-')) ++q;
  int nd = 0;
  while (q < end && std::isdigit((unsigned char)*q)) ++q, ++nd;
  if (q < end && *q == '.') {
    ++q;
    while (q < end && std::isdigit((unsigned char)*q)) ++q, ++nd;
  }
  if (nd == 0) return false;
  if (q < end && (*q == 'e' || *q == 'E')) {
    ++q;
    if (q < end && (*q == '+' || *q == '-')) ++q;
    int ne = 0;
    while (q < end && std::isdigit((unsigned char)*q)) ++q, ++ne;
    if (ne == 0) return false;
  }
  return true;
}

// Parses [begin, end) (whole lines). Returns false on any line the strict form
// does not cover.
bool parse_strict(const char* p, const char* end, std::vector<uint64_t>& out) {
  while (p < end) {
    const char* nl = (const char*)std::memchr(p, '\n', (size_t)(end - p));
    const char* le = nl ? nl : end;
    const char* q = p;
    while (q < le && (*q == ' ' || *q == '\t')) ++q;
    if (q == le) {  // blank or whitespace-only line: skipped by operator>>
      p = nl ? nl + 1 : end;
      continue;
    }
    uint64_t ids[2];
    for (int k = 0; k < 2; ++k) {
      if (k) {
        if (q >= le || (*q != ' ' && *q != '\t')) return false;
        while (q < le && (*q == ' ' || *q == '\t')) ++q;
      }
      uint64_t v = 0;
      int nd = 0;
      while (q < le && *q >= '0' && *q <= '9') v = v * 10 + (uint64_t)(*q++ - '0'), ++nd;
      if (nd == 0 || nd > 10 || v > 0xffffffffull) return false;
      ids[k] = v;
    }
    while (q < le) {
      if (*q != ' ' && *q != '\t') return false;
      while (q < le && (*q == ' ' || *q == '\t')) ++q;
      if (q == le) return false;  // trailing blanks: the reference's value loop crosses the line
      if (!number_token(q, le)) return false;
    }
    if (!nl && q != end) return false;
    uint64_t z;
    if (fold((uint32_t)ids[0], (uint32_t)ids[1], &z)) out.push_back(z);
    p = nl ? nl + 1 : end;
  }
  return true;
}

// parse_strict into a caller array of at least (end - p) / 4 + 1 entries
// (every entry line takes at least 4 bytes: "1 2\n"): the common line "id,
// blanks, id, newline" is taken in one pass without a line search; any other
// line goes through parse_strict. Returns the entries written, or SIZE_MAX
// where parse_strict fails.
size_t parse_strict_fast(const char* p, const char* end, uint64_t* out) {
  size_t k = 0;
  std::vector<uint64_t> slow;
  while (p < end) {
    const char* q = p;
    uint64_t v0 = 0, v1 = 0;
    int n0 = 0, n1 = 0;
    while (q < end && (unsigned)(*q - '0') < 10u) v0 = v0 * 10 + (uint64_t)(*q++ - '0'), ++n0;
    if (n0 && q < end && (*q == ' ' || *q == '\t')) {
      while (q < end && (*q == ' ' || *q == '\t')) ++q;
      while (q < end && (unsigned)(*q - '0') < 10u) v1 = v1 * 10 + (uint64_t)(*q++ - '0'), ++n1;
      if (n1 && n0 <= 10 && n1 <= 10 && v0 <= 0xffffffffull && v1 <= 0xffffffffull && q < end && *q == '\n') {
        uint64_t z;
        if (fold((uint32_t)v0, (uint32_t)v1, &z)) out[k++] = z;
        p = q + 1;
        continue;
      }
    }
    // Any other line: the general strict parse of this one line.
    const char* nl = (const char*)std::memchr(p, '\n', (size_t)(end - p));
    const char* le = nl ? nl + 1 : end;
    slow.clear();
    if (!parse_strict(p, le, slow)) return SIZE_MAX;
    for (uint64_t z : slow) out[k++] = z;
    p = le;
  }
  return k;
}

}  // namespace

namespace tb {

tribit_status mtx_header(const char* p, const char* end, const char** body, uint64_t* num_nodes, uint64_t* nnz) {
  // Banner line (tribit.cu:232), then lines starting with '%' (tribit.cu:234-235).
  const char* nl = p < end ? (const char*)std::memchr(p, '\n', (size_t)(end - p)) : nullptr;
  p = nl ? nl + 1 : end;
  const char* line = nullptr;
  const char* line_end = nullptr;
  while (p < end) {
    nl = (const char*)std::memchr(p, '\n', (size_t)(end - p));
    const char* le = nl ? nl : end;
    line = p;
    line_end = le;
    p = nl ? nl + 1 : end;
    if (le == line || *line != '%') break;
    line = nullptr;
  }
  if (!line) return TRIBIT_ERR_FORMAT;
  // "rows cols nnz" (tribit.cu:238-245).
  uint64_t dims[3];
  const char* q = line;
  for (int k = 0; k < 3; ++k) {
    while (q < line_end && is_ws(*q)) ++q;
    uint64_t v = 0;
    int nd = 0;
    while (q < line_end && *q >= '0' && *q <= '9') v = v * 10 + (uint64_t)(*q++ - '0'), ++nd;
    if (!nd) return TRIBIT_ERR_FORMAT;
    dims[k] = v;
  }
  if (dims[0] != dims[1]) return TRIBIT_ERR_NOT_SQUARE;
  *num_nodes = dims[0];
  *nnz = dims[2];
  *body = p;
  return TRIBIT_OK;
}

}  // namespace tb

extern "C" tribit_status tribit_read_mtx(const char* path, uint64_t* num_nodes, uint64_t** entries,
                                         uint64_t* n_entries) {
  if (!path || !num_nodes || !entries || !n_entries) return TRIBIT_ERR_INVALID_ARGUMENT;
  *entries = nullptr;
  *n_entries = 0;
  Mapped m;
  m.fd = open(path, O_RDONLY);
  if (m.fd < 0) return TRIBIT_ERR_IO;
  struct stat sb;
  if (fstat(m.fd, &sb) != 0) return TRIBIT_ERR_IO;
  m.len = (size_t)sb.st_size;
  if (m.len > 0) {
    void* q = mmap(nullptr, m.len, PROT_READ, MAP_PRIVATE, m.fd, 0);
    if (q == MAP_FAILED) return TRIBIT_ERR_IO;
    m.p = (const char*)q;
    madvise(q, m.len, MADV_SEQUENTIAL);
  }
  const char* p = nullptr;
  const char* end = m.p + m.len;
  uint64_t dims[3];
  {
    const tribit_status hs = tb::mtx_header(m.p, end, &p, num_nodes, &dims[2]);
    if (hs != TRIBIT_OK) return hs;
  }

  // Entries: parallel strict parse, else the exact grammar.
  std::vector<uint64_t> all;
  uint64_t* buf = nullptr;
  size_t total = 0;
  const size_t body = (size_t)(end - p);
  unsigned hw = std::thread::hardware_concurrency();
  int threads = (int)std::max(1u, std::min(hw ? hw : 1u, 64u));
  if (body < (8u << 20)) threads = 1;
  std::vector<const char*> cut(threads + 1);
  cut[0] = p;
  cut[threads] = end;
  for (int t = 1; t < threads; ++t) {
    const char* c = p + body * t / threads;
    if (c < cut[t - 1]) c = cut[t - 1];
    const char* x = c < end ? (const char*)std::memchr(c, '\n', (size_t)(end - c)) : nullptr;
    cut[t] = x ? x + 1 : end;
  }
  std::vector<uint64_t*> parts(threads, nullptr);
  std::vector<size_t> got(threads, 0);
  std::atomic<bool> strict_ok{true};
  auto work = [&](int t) {
    const size_t cap = (size_t)(cut[t + 1] - cut[t]) / 4 + 1;
    parts[t] = (uint64_t*)std::malloc(cap * sizeof(uint64_t));
    if (!parts[t]) {
      strict_ok = false;
      return;
    }
    got[t] = parse_strict_fast(cut[t], cut[t + 1], parts[t]);
    if (got[t] == SIZE_MAX) strict_ok = false;
  };
  struct FreeParts {
    std::vector<uint64_t*>& v;
    ~FreeParts() {
      for (uint64_t* x : v) std::free(x);
    }
  } free_parts{parts};
  try {
    if (threads == 1) {
      work(0);
    } else {
      std::vector<std::thread> th;
      for (int t = 0; t < threads; ++t) th.emplace_back(work, t);
      for (auto& x : th) x.join();
    }
    if (strict_ok) {
      // Each thread copies its part into the caller's buffer.
      std::vector<size_t> at(threads + 1, 0);
      for (int t = 0; t < threads; ++t) at[t + 1] = at[t] + got[t];
      total = at[threads];
      buf = (uint64_t*)std::malloc(std::max<size_t>(total, 1) * sizeof(uint64_t));
      if (!buf) return TRIBIT_ERR_OUT_OF_MEMORY;
      auto copy = [&](int t) {
        if (got[t]) std::memcpy(buf + at[t], parts[t], got[t] * sizeof(uint64_t));
      };
      if (threads == 1) {
        copy(0);
      } else {
        std::vector<std::thread> th;
        for (int t = 0; t < threads; ++t) th.emplace_back(copy, t);
        for (auto& x : th) x.join();
      }
    } else {
      all.reserve(dims[2]);
      parse_exact(p, end, all);
      total = all.size();
      buf = (uint64_t*)std::malloc(std::max<size_t>(total, 1) * sizeof(uint64_t));
      if (!buf) return TRIBIT_ERR_OUT_OF_MEMORY;
      std::memcpy(buf, all.data(), total * sizeof(uint64_t));
    }
  } catch (const std::bad_alloc&) {
    std::free(buf);
    return TRIBIT_ERR_OUT_OF_MEMORY;
  }
  *entries = buf;
  *n_entries = total;
  return TRIBIT_OK;
}

extern "C" void tribit_free_host(void* p) { std::free(p); }
