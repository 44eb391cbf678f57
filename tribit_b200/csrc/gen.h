// Seeded synthetic graph generators shared by host and device code.
//
// Every generator is counter-based: edge i of a graph is a pure function of
// (seed, i), so the output does not depend on how many host threads or GPU
// threads produce it, and a host copy and a device copy of the same graph are
// identical word for word.
//
// Output entries use the reference's zipped edge word: (row << 32) | col with
// 0-based vertex ids (tribit.cu:258-266 builds the same word after folding).
// Generators emit raw entries -- duplicates and self-loops included -- because
// the counter itself folds, drops self-loops and deduplicates.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define TB_HD __host__ __device__ __forceinline__
#else
#define TB_HD static inline
#endif

// SplitMix64 output function (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014).
TB_HD uint64_t tb_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Independent 64-bit stream value `i` of stream `seed`.
TB_HD uint64_t tb_rand(uint64_t seed, uint64_t i) { return tb_mix64(tb_mix64(seed) ^ (i * 0xD6E8FEB86659FD93ull)); }

// Uniform double in [0,1) from 53 random bits.
TB_HD double tb_unit(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

TB_HD uint64_t tb_zip(uint32_t r, uint32_t c) { return ((uint64_t)r << 32) | (uint64_t)c; }

// Recursive-matrix (R-MAT, Chakrabarti, Zhan and Faloutsos, SDM 2004) edge i of
// a 2^scale-vertex graph. At each of `scale` levels one 32-bit uniform picks a
// quadrant with probabilities a, b, c, d given as cumulative 32-bit thresholds
// t_a = a*2^32, t_ab = (a+b)*2^32, t_abc = (a+b+c)*2^32. Quadrant b sets the
// column bit, c the row bit, d both. No vertex permutation is applied.
TB_HD uint64_t tb_rmat_edge(uint64_t seed, uint64_t i, int scale, uint32_t t_a, uint32_t t_ab, uint32_t t_abc) {
  uint32_t r = 0, c = 0;
  uint64_t h = 0;
  for (int l = 0; l < scale; ++l) {
    if ((l & 1) == 0) h = tb_rand(seed, (i << 5) | (uint64_t)(l >> 1));
    uint32_t x = (uint32_t)(h >> ((l & 1) * 32));
    uint32_t bit = 1u << (scale - 1 - l);
    if (x < t_a) {
    } else if (x < t_ab) {
      c |= bit;
    } else if (x < t_abc) {
      r |= bit;
    } else {
      r |= bit;
      c |= bit;
    }
  }
  return tb_zip(r, c);
}

// Erdos-Renyi G(n, m) style entry i: both endpoints uniform in [0, n).
TB_HD uint64_t tb_er_edge(uint64_t seed, uint64_t i, uint32_t n) {
  uint64_t h = tb_rand(seed, i);
  uint32_t r = (uint32_t)(((h >> 32) * (uint64_t)n) >> 32);
  uint32_t c = (uint32_t)(((h & 0xffffffffull) * (uint64_t)n) >> 32);
  return tb_zip(r, c);
}

// Inverse-CDF lookup: smallest k with cdf[k] > x, cdf strictly covering [0, total).
TB_HD uint32_t tb_cdf_pick(const double* cdf, uint32_t n, double x) {
  uint32_t lo = 0, hi = n - 1;
  while (lo < hi) {
    uint32_t mid = lo + (hi - lo) / 2;
    if (cdf[mid] > x)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

// Chung-Lu entry i: both endpoints drawn independently with probability
// proportional to the vertex weights whose inclusive prefix sums are `cdf`.
TB_HD uint64_t tb_chung_lu_edge(uint64_t seed, uint64_t i, const double* cdf, uint32_t n) {
  uint64_t h1 = tb_rand(seed, 2 * i), h2 = tb_rand(seed, 2 * i + 1);
  double total = cdf[n - 1];
  uint32_t r = tb_cdf_pick(cdf, n, tb_unit(h1) * total);
  uint32_t c = tb_cdf_pick(cdf, n, tb_unit(h2) * total);
  return tb_zip(r, c);
}
