// Host drivers for the seeded graph generators of gen.h, parallel over host
// threads. Output does not depend on the thread count (counter-based RNG).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "gen.h"
#include "tribit.h"

namespace {

int host_threads() {
  unsigned t = std::thread::hardware_concurrency();
  return t == 0 ? 1 : (int)std::min(t, 64u);
}

// Runs fn(lo, hi) over [0, n) in contiguous chunks on all host threads.
template <typename F>
void parallel_for(uint64_t n, F fn) {
  int t = host_threads();
  if (n < 65536 || t == 1) {
    fn(0, n);
    return;
  }
  std::vector<std::thread> th;
  uint64_t chunk = (n + t - 1) / t;
  for (int k = 0; k < t; ++k) {
    uint64_t lo = k * chunk, hi = std::min(n, lo + chunk);
    if (lo >= hi) break;
    th.emplace_back([=] { fn(lo, hi); });
  }
  for (auto& x : th) x.join();
}

uint32_t prob_threshold(double p) {
  double t = std::floor(p * 4294967296.0);
  if (t < 0) t = 0;
  if (t > 4294967295.0) t = 4294967295.0;
  return (uint32_t)t;
}

}  // namespace

extern "C" tribit_status tribit_gen_rmat(int scale, uint64_t edge_factor, double a, double b, double c, uint64_t seed,
                                         uint64_t* out) {
  if (scale < 1 || scale > 31 || !out || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return TRIBIT_ERR_INVALID_ARGUMENT;
  uint64_t m = edge_factor << scale;
  uint32_t ta = prob_threshold(a), tab = prob_threshold(a + b), tabc = prob_threshold(a + b + c);
  parallel_for(m, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo; i < hi; ++i) out[i] = tb_rmat_edge(seed, i, scale, ta, tab, tabc);
  });
  return TRIBIT_OK;
}

extern "C" tribit_status tribit_gen_er(uint32_t n, uint64_t n_entries, uint64_t seed, uint64_t* out) {
  if (n == 0 || !out) return TRIBIT_ERR_INVALID_ARGUMENT;
  parallel_for(n_entries, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo; i < hi; ++i) out[i] = tb_er_edge(seed, i, n);
  });
  return TRIBIT_OK;
}

extern "C" tribit_status tribit_gen_chung_lu(uint32_t n, uint64_t n_entries, double beta, double max_degree,
                                             uint64_t seed, uint64_t* out) {
  if (n == 0 || !out || beta <= 1.0) return TRIBIT_ERR_INVALID_ARGUMENT;
  // Weights w_i = (i + 1)^(-1 / (beta - 1)); the expected degree of vertex i
  // is 2 * n_entries * w_i / sum(w). Weights above the one giving max_degree
  // are clipped, a few times, because clipping lowers the sum.
  std::vector<double> w(n), cdf(n);
  double ex = -1.0 / (beta - 1.0);
  for (uint32_t i = 0; i < n; ++i) w[i] = std::pow((double)i + 1.0, ex);
  for (int it = 0; it < 8 && max_degree > 0 && n_entries > 0; ++it) {
    double s = 0;
    for (double x : w) s += x;
    double cap = max_degree * s / (2.0 * (double)n_entries);
    for (double& x : w) x = std::min(x, cap);
  }
  double s = 0;
  for (uint32_t i = 0; i < n; ++i) cdf[i] = (s += w[i]);
  const double* cp = cdf.data();
  parallel_for(n_entries, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo; i < hi; ++i) out[i] = tb_chung_lu_edge(seed, i, cp, n);
  });
  return TRIBIT_OK;
}

// Planted partition: `communities` groups of `size` vertices; every pair inside
// a group is an edge with probability p_in; every vertex adds
// `inter_per_vertex` entries to uniformly random vertices; finally all ids are
// permuted by a seeded Fisher-Yates shuffle. With out == NULL the entry count
// is returned in *n_entries; otherwise *n_entries is the capacity of `out` on
// input and the count on output.
extern "C" tribit_status tribit_gen_planted(uint32_t communities, uint32_t size, double p_in,
                                            uint32_t inter_per_vertex, uint64_t seed, uint64_t* out,
                                            uint64_t* n_entries) {
  if (!n_entries || communities == 0 || size < 2) return TRIBIT_ERR_INVALID_ARGUMENT;
  uint64_t n = (uint64_t)communities * size;
  if (n > 0xffffffffull) return TRIBIT_ERR_TOO_LARGE;
  uint64_t pairs = (uint64_t)size * (size - 1) / 2;
  uint64_t thr = (uint64_t)std::min(18446744073709551615.0, std::floor(p_in * 18446744073709551616.0));
  if (p_in >= 1.0) thr = ~0ull;
  std::vector<uint64_t> per(communities + 1, 0);
  uint64_t intra_seed = tb_mix64(seed ^ 0x1111), inter_seed = tb_mix64(seed ^ 0x2222), perm_seed = tb_mix64(seed ^ 0x3333);
  parallel_for(communities, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t g = lo; g < hi; ++g) {
      uint64_t k = 0;
      for (uint64_t q = 0; q < pairs; ++q) k += tb_rand(intra_seed, g * pairs + q) < thr || p_in >= 1.0;
      per[g + 1] = k;
    }
  });
  for (uint32_t g = 0; g < communities; ++g) per[g + 1] += per[g];
  uint64_t total = per[communities] + n * inter_per_vertex;
  if (!out) {
    *n_entries = total;
    return TRIBIT_OK;
  }
  if (*n_entries < total) return TRIBIT_ERR_INVALID_ARGUMENT;
  std::vector<uint32_t> perm(n);
  for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
  for (uint64_t i = n - 1; i > 0; --i) {
    uint64_t j = tb_rand(perm_seed, i) % (i + 1);
    std::swap(perm[i], perm[j]);
  }
  const uint32_t* pp = perm.data();
  parallel_for(communities, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t g = lo; g < hi; ++g) {
      uint64_t k = per[g], q = 0;
      uint64_t base = g * size;
      for (uint32_t i = 0; i < size; ++i)
        for (uint32_t j = i + 1; j < size; ++j, ++q)
          if (tb_rand(intra_seed, g * pairs + q) < thr || p_in >= 1.0) out[k++] = tb_zip(pp[base + i], pp[base + j]);
    }
  });
  uint64_t off = per[communities];
  parallel_for(n * inter_per_vertex, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo; i < hi; ++i) {
      uint64_t v = i / inter_per_vertex;
      uint64_t w = ((tb_rand(inter_seed, i) >> 32) * n) >> 32;
      out[off + i] = tb_zip(pp[v], pp[w]);
    }
  });
  *n_entries = total;
  return TRIBIT_OK;
}

// Writes a symmetric pattern Matrix Market file with one line per entry
// (1-based, larger id first as the symmetric format stores the lower triangle).
// Self-loop entries are written as given.
extern "C" tribit_status tribit_write_mtx(const char* path, uint64_t num_nodes, const uint64_t* entries,
                                          uint64_t n_entries) {
  FILE* f = std::fopen(path, "wb");
  if (!f) return TRIBIT_ERR_IO;
  std::fprintf(f, "%%%%MatrixMarket matrix coordinate pattern symmetric\n");
  std::fprintf(f, "%% generated by tribit_b200\n");
  std::fprintf(f, "%llu %llu %llu\n", (unsigned long long)num_nodes, (unsigned long long)num_nodes,
               (unsigned long long)n_entries);
  std::vector<char> buf;
  buf.reserve(1 << 20);
  char line[48];
  for (uint64_t i = 0; i < n_entries; ++i) {
    uint32_t a = (uint32_t)(entries[i] >> 32), b = (uint32_t)entries[i];
    uint32_t hi = a > b ? a : b, lo = a > b ? b : a;
    int k = std::snprintf(line, sizeof line, "%u %u\n", hi + 1, lo + 1);
    buf.insert(buf.end(), line, line + k);
    if (buf.size() > (1 << 20)) {
      std::fwrite(buf.data(), 1, buf.size(), f);
      buf.clear();
    }
  }
  std::fwrite(buf.data(), 1, buf.size(), f);
  return std::fclose(f) == 0 ? TRIBIT_OK : TRIBIT_ERR_IO;
}

namespace {

struct BatchGraph {
  uint32_t n;
  uint64_t entries;
  bool chung_lu;
  double beta;
  uint64_t seed;
};

// Graph g of the batched workload, drawn from stream `seed`.
BatchGraph batch_graph(uint64_t seed, uint32_t g, uint32_t min_n, uint32_t max_n) {
  BatchGraph b;
  const uint64_t s = tb_rand(seed, g);
  const double u1 = tb_unit(tb_rand(s, 1)), u2 = tb_unit(tb_rand(s, 2)), u3 = tb_unit(tb_rand(s, 3)),
               u4 = tb_unit(tb_rand(s, 4));
  const double lo = std::log((double)min_n), hi = std::log((double)max_n);
  b.n = (uint32_t)std::min<double>(max_n, std::floor(std::exp(lo + (hi - lo) * u1)));
  if (b.n < min_n) b.n = min_n;
  const double deg = 8.0 + 56.0 * u3;
  b.entries = (uint64_t)(b.n * deg / 2.0);
  b.chung_lu = u2 >= 0.5;
  b.beta = 2.1 + 0.7 * u4;
  b.seed = tb_rand(s, 5);
  return b;
}

}  // namespace

extern "C" tribit_status tribit_gen_batch(uint32_t num_graphs, uint32_t min_n, uint32_t max_n, uint64_t seed,
                                          uint32_t* num_nodes, uint64_t* entry_offsets, uint64_t* entries) {
  if (num_graphs == 0 || min_n < 2 || max_n < min_n || !num_nodes || !entry_offsets) return TRIBIT_ERR_INVALID_ARGUMENT;
  entry_offsets[0] = 0;
  for (uint32_t g = 0; g < num_graphs; ++g) {
    const BatchGraph b = batch_graph(seed, g, min_n, max_n);
    num_nodes[g] = b.n;
    entry_offsets[g + 1] = entry_offsets[g] + b.entries;
  }
  if (!entries) return TRIBIT_OK;
  // Graphs are independent: hand them out to host threads one at a time.
  std::atomic<uint32_t> next{0};
  auto work = [&] {
    std::vector<double> w, cdf;
    for (uint32_t g; (g = next.fetch_add(1)) < num_graphs;) {
      const BatchGraph b = batch_graph(seed, g, min_n, max_n);
      uint64_t* out = entries + entry_offsets[g];
      if (!b.chung_lu) {
        for (uint64_t i = 0; i < b.entries; ++i) out[i] = tb_er_edge(b.seed, i, b.n);
        continue;
      }
      // Chung-Lu weights (i + 1)^(-1 / (beta - 1)), clipped at an expected
      // degree of sqrt(2 * entries) (the structural cut-off).
      w.assign(b.n, 0.0);
      cdf.assign(b.n, 0.0);
      const double ex = -1.0 / (b.beta - 1.0);
      for (uint32_t i = 0; i < b.n; ++i) w[i] = std::pow((double)i + 1.0, ex);
      const double max_deg = std::sqrt(2.0 * (double)b.entries);
      for (int it = 0; it < 8; ++it) {
        double s = 0;
        for (double x : w) s += x;
        const double cap = max_deg * s / (2.0 * (double)b.entries);
        for (double& x : w) x = std::min(x, cap);
      }
      double s = 0;
      for (uint32_t i = 0; i < b.n; ++i) cdf[i] = (s += w[i]);
      for (uint64_t i = 0; i < b.entries; ++i) out[i] = tb_chung_lu_edge(b.seed, i, cdf.data(), b.n);
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < host_threads(); ++t) th.emplace_back(work);
  for (auto& x : th) x.join();
  return TRIBIT_OK;
}
