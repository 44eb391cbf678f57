/* CPU oracle for exact triangle counting -- TEST INFRASTRUCTURE ONLY.
 * See oracle.h for what each function restates and where the pins live.
 * Plain C11 + pthreads; no dependency on the product library. */
#define _GNU_SOURCE
#include "oracle.h"

#include <ctype.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

void oracle_free(void* p) { free(p); }

/* ------------------------------------------------------------------------ */
/* Matrix Market reader: restates read_mtx (tribit.cu:228-269).              */
/* ------------------------------------------------------------------------ */

typedef struct {
  const char* p;
  const char* end;
  int fail;
} stream_t;

static int s_peek(stream_t* s) { return s->p < s->end ? (unsigned char)*s->p : EOF; }

static void s_skip_ws(stream_t* s) {
  while (s->p < s->end && isspace((unsigned char)*s->p)) s->p++;
}

/* operator>>(uint32_t&) of libstdc++: skip whitespace, optional sign, digits;
 * a '-' negates modulo 2^32; overflow sets failbit. (tribit.cu:253) */
static int s_read_u32(stream_t* s, uint32_t* out) {
  if (s->fail) return 0;
  s_skip_ws(s);
  int neg = 0;
  if (s->p < s->end && (*s->p == '+' || *s->p == '-')) {
    neg = *s->p == '-';
    s->p++;
  }
  uint64_t v = 0;
  int nd = 0, ovf = 0;
  while (s->p < s->end && *s->p >= '0' && *s->p <= '9') {
    v = v * 10 + (uint64_t)(*s->p - '0');
    if (v > 0xffffffffull) ovf = 1, v = 0xffffffffull;
    s->p++;
    nd++;
  }
  if (nd == 0 || ovf) {
    s->fail = 1;
    return 0;
  }
  *out = neg ? (uint32_t)(0u - (uint32_t)v) : (uint32_t)v;
  return 1;
}

/* operator>>(double&): [sign] digits [. digits] [e [sign] digits]; at least
 * one mantissa digit. The value itself is discarded by the reference
 * (tribit.cu:255-256), so only the token extent and success matter. */
static int s_read_double(stream_t* s) {
  if (s->fail) return 0;
  s_skip_ws(s);
  const char* q = s->p;
  if (q < s->end && (*q == '+' || *q == '-')) q++;
  int nd = 0;
  while (q < s->end && isdigit((unsigned char)*q)) q++, nd++;
  if (q < s->end && *q == '.') {
    q++;
    while (q < s->end && isdigit((unsigned char)*q)) q++, nd++;
  }
  if (nd == 0) {
    s->fail = 1;
    return 0;
  }
  if (q < s->end && (*q == 'e' || *q == 'E')) {
    const char* e = q + 1;
    if (e < s->end && (*e == '+' || *e == '-')) e++;
    int ne = 0;
    while (e < s->end && isdigit((unsigned char)*e)) e++, ne++;
    if (ne == 0) {
      s->fail = 1; /* "1e" is a failed extraction in libstdc++ */
      return 0;
    }
    q = e;
  }
  s->p = q;
  return 1;
}

static int read_whole_file(const char* path, char** buf, size_t* len) {
  FILE* f = fopen(path, "rb");
  if (!f) return 2;
  if (fseek(f, 0, SEEK_END) != 0) {
    fclose(f);
    return 2;
  }
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  char* b = (char*)malloc((size_t)sz + 1);
  if (!b) {
    fclose(f);
    return 8;
  }
  size_t got = fread(b, 1, (size_t)sz, f);
  fclose(f);
  b[got] = 0;
  *buf = b;
  *len = got;
  return 0;
}

int oracle_read_mtx(const char* path, uint64_t* num_nodes, uint64_t** entries, uint64_t* n_entries) {
  char* buf;
  size_t len;
  int st = read_whole_file(path, &buf, &len);
  if (st) return st;
  const char* p = buf;
  const char* end = buf + len;
  /* std::getline of the banner line (tribit.cu:232). */
  const char* nl = memchr(p, '\n', (size_t)(end - p));
  p = nl ? nl + 1 : end;
  /* Skip lines whose first character is '%'; the first other line is the
   * size line (tribit.cu:234-235). */
  const char* line = NULL;
  const char* line_end = NULL;
  while (p < end) {
    nl = memchr(p, '\n', (size_t)(end - p));
    const char* le = nl ? nl : end;
    line = p;
    line_end = le;
    p = nl ? nl + 1 : end;
    if (le == line || *line != '%') break;
    line = NULL;
  }
  if (!line) {
    free(buf);
    return 3;
  }
  /* stringstream >> n_rows >> n_cols >> nnz (tribit.cu:238-240). */
  stream_t ls = {line, line_end, 0};
  uint64_t dims[3];
  for (int k = 0; k < 3; ++k) {
    s_skip_ws(&ls);
    uint64_t v = 0;
    int nd = 0;
    while (ls.p < ls.end && isdigit((unsigned char)*ls.p)) v = v * 10 + (uint64_t)(*ls.p++ - '0'), nd++;
    if (!nd) {
      free(buf);
      return 3;
    }
    dims[k] = v;
  }
  if (dims[0] != dims[1]) {
    free(buf);
    return 4;
  }
  *num_nodes = dims[0];
  /* Entry loop (tribit.cu:250-268). */
  uint64_t cap = dims[2] > 0 ? dims[2] : 16, cnt = 0;
  uint64_t* out = (uint64_t*)malloc(cap * sizeof(uint64_t));
  if (!out) {
    free(buf);
    return 8;
  }
  stream_t s = {p, end, 0};
  uint32_t r, c;
  while (s_read_u32(&s, &r) && s_read_u32(&s, &c)) {
    while (s_peek(&s) != '\n' && s_peek(&s) != EOF) {
      if (!s_read_double(&s)) break;
    }
    r = r - 1;
    c = c - 1;
    uint64_t z;
    if (c < r)
      z = ((uint64_t)c << 32) | r;
    else if (r < c)
      z = ((uint64_t)r << 32) | c;
    else
      continue;
    if (cnt == cap) {
      cap *= 2;
      uint64_t* o2 = (uint64_t*)realloc(out, cap * sizeof(uint64_t));
      if (!o2) {
        free(out);
        free(buf);
        return 8;
      }
      out = o2;
    }
    out[cnt++] = z;
  }
  free(buf);
  *entries = out;
  *n_entries = cnt;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Fold + sort + dedup (tribit.cu:258-267, 666-667).                         */
/* ------------------------------------------------------------------------ */

static int bits_for(uint64_t n) {
  int b = 1;
  while (b < 64 && (1ull << b) < n) b++;
  return b;
}

/* LSD radix sort of 64-bit keys on their low `bits` bits, 11 bits a pass. */
static void radix_sort_u64(uint64_t* a, uint64_t n, int bits) {
  if (n < 2) return;
  uint64_t* tmp = (uint64_t*)malloc(n * sizeof(uint64_t));
  uint64_t* src = a;
  uint64_t* dst = tmp;
  uint64_t* cnt = (uint64_t*)malloc(2048 * sizeof(uint64_t));
  for (int sh = 0; sh < bits; sh += 11) {
    memset(cnt, 0, 2048 * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; ++i) cnt[(src[i] >> sh) & 2047]++;
    uint64_t s = 0;
    for (int d = 0; d < 2048; ++d) {
      uint64_t t = cnt[d];
      cnt[d] = s;
      s += t;
    }
    for (uint64_t i = 0; i < n; ++i) dst[cnt[(src[i] >> sh) & 2047]++] = src[i];
    uint64_t* t = src;
    src = dst;
    dst = t;
  }
  if (src != a) memcpy(a, src, n * sizeof(uint64_t));
  free(tmp);
  free(cnt);
}

uint64_t oracle_fold_dedup(uint64_t* e, uint64_t n_entries) {
  uint64_t k = 0;
  uint32_t maxid = 0;
  for (uint64_t i = 0; i < n_entries; ++i) {
    uint32_t a = (uint32_t)(e[i] >> 32), b = (uint32_t)e[i];
    if (a == b) continue;
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    if (hi > maxid) maxid = hi;
    e[k++] = ((uint64_t)lo << 32) | hi;
  }
  /* Compact the key to (lo << B) | hi so the sort only touches 2B bits. */
  int B = bits_for((uint64_t)maxid + 1);
  for (uint64_t i = 0; i < k; ++i) e[i] = ((e[i] >> 32) << B) | (e[i] & 0xffffffffull);
  radix_sort_u64(e, k, 2 * B);
  uint64_t m = 0;
  for (uint64_t i = 0; i < k; ++i)
    if (m == 0 || e[i] != e[m - 1]) e[m++] = e[i];
  uint64_t mask = (1ull << B) - 1;
  for (uint64_t i = 0; i < m; ++i) e[i] = ((e[i] >> B) << 32) | (e[i] & mask);
  return m;
}

/* ------------------------------------------------------------------------ */
/* Oriented CSR                                                              */
/* ------------------------------------------------------------------------ */

int oracle_csr_build(const uint64_t* edges, uint64_t m, uint64_t n, int order, oracle_csr* g) {
  uint32_t* rank = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
  uint64_t* deg = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
  if (!rank || !deg) return 8;
  if (order == 1) {
    for (uint64_t i = 0; i < m; ++i) {
      deg[edges[i] >> 32]++;
      deg[edges[i] & 0xffffffffull]++;
    }
    /* Stable counting sort by degree: rank = position in (deg, id) order. */
    uint64_t maxd = 0;
    for (uint64_t v = 0; v < n; ++v)
      if (deg[v] > maxd) maxd = deg[v];
    uint64_t* start = (uint64_t*)calloc(maxd + 2, sizeof(uint64_t));
    for (uint64_t v = 0; v < n; ++v) start[deg[v] + 1]++;
    for (uint64_t d = 1; d <= maxd + 1; ++d) start[d] += start[d - 1];
    for (uint64_t v = 0; v < n; ++v) rank[v] = (uint32_t)start[deg[v]]++;
    free(start);
  } else {
    for (uint64_t v = 0; v < n; ++v) rank[v] = (uint32_t)v;
  }
  memset(deg, 0, (n + 1) * sizeof(uint64_t));
  uint64_t* o = (uint64_t*)malloc((m ? m : 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < m; ++i) {
    uint32_t a = rank[edges[i] >> 32], b = rank[(uint32_t)edges[i]];
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    o[i] = ((uint64_t)lo << 32) | hi;
  }
  int B = bits_for(n);
  for (uint64_t i = 0; i < m; ++i) o[i] = ((o[i] >> 32) << B) | (o[i] & 0xffffffffull);
  radix_sort_u64(o, m, 2 * B);
  g->n = n;
  g->m = m;
  g->row_ptr = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
  g->col = (uint32_t*)malloc((m ? m : 1) * sizeof(uint32_t));
  uint64_t mask = (1ull << B) - 1;
  for (uint64_t i = 0; i < m; ++i) {
    g->row_ptr[(o[i] >> B) + 1]++;
    g->col[i] = (uint32_t)(o[i] & mask);
  }
  for (uint64_t v = 0; v < n; ++v) g->row_ptr[v + 1] += g->row_ptr[v];
  free(o);
  free(rank);
  free(deg);
  return 0;
}

void oracle_csr_free(oracle_csr* g) {
  free(g->row_ptr);
  free(g->col);
  g->row_ptr = NULL;
  g->col = NULL;
}

static uint64_t merge_count(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb) {
  uint64_t i = 0, j = 0, c = 0;
  while (i < na && j < nb) {
    if (a[i] < b[j])
      i++;
    else if (b[j] < a[i])
      j++;
    else
      c++, i++, j++;
  }
  return c;
}

static uint64_t row_triangles(const oracle_csr* g, uint64_t u) {
  const uint32_t* nu = g->col + g->row_ptr[u];
  uint64_t du = g->row_ptr[u + 1] - g->row_ptr[u], t = 0;
  for (uint64_t k = 0; k < du; ++k) {
    uint32_t v = nu[k];
    t += merge_count(nu + k + 1, du - k - 1, g->col + g->row_ptr[v], g->row_ptr[v + 1] - g->row_ptr[v]);
  }
  return t;
}

typedef struct {
  const oracle_csr* g;
  uint64_t next; /* shared cursor over 32-row blocks, advanced atomically */
  uint64_t total;
  uint64_t stride; /* count row blocks b with b % stride == offset */
  uint64_t offset;
} count_job;

static void* count_worker(void* arg) {
  count_job* j = (count_job*)arg;
  uint64_t local = 0;
  uint64_t nblk = (j->g->n + 31) / 32;
  for (;;) {
    uint64_t lo = __atomic_fetch_add(&j->next, 8, __ATOMIC_RELAXED);
    if (lo >= nblk) break;
    uint64_t hi = lo + 8 < nblk ? lo + 8 : nblk;
    for (uint64_t b = lo; b < hi; ++b) {
      if (b % j->stride != j->offset) continue;
      uint64_t uend = b * 32 + 32 < j->g->n ? b * 32 + 32 : j->g->n;
      for (uint64_t u = b * 32; u < uend; ++u) local += row_triangles(j->g, u);
    }
  }
  __atomic_fetch_add(&j->total, local, __ATOMIC_RELAXED);
  return NULL;
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + ts.tv_nsec * 1e-9;
}

uint64_t oracle_count_csr(const oracle_csr* g, int threads, double* seconds) {
  return oracle_count_csr_sample(g, threads, 1, 0, seconds);
}

uint64_t oracle_count_csr_sample(const oracle_csr* g, int threads, uint64_t stride, uint64_t offset, double* seconds) {
  if (threads < 1) threads = 1;
  if (stride < 1) stride = 1;
  count_job job = {g, 0, 0, stride, offset % stride};
  double t0 = now_s();
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
  for (int i = 0; i < threads; ++i) pthread_create(&th[i], NULL, count_worker, &job);
  for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
  free(th);
  if (seconds) *seconds = now_s() - t0;
  return job.total;
}

void oracle_count_rows(const oracle_csr* g, uint64_t* out) {
  for (uint64_t u = 0; u < g->n; ++u) out[u] = row_triangles(g, u);
}

uint64_t oracle_count_entries(const uint64_t* entries, uint64_t n_entries, uint64_t n, int order, int threads,
                              uint64_t* edges_out) {
  uint64_t* e = (uint64_t*)malloc((n_entries ? n_entries : 1) * sizeof(uint64_t));
  memcpy(e, entries, n_entries * sizeof(uint64_t));
  uint64_t m = oracle_fold_dedup(e, n_entries);
  oracle_csr g;
  oracle_csr_build(e, m, n, order, &g);
  free(e);
  uint64_t t = oracle_count_csr(&g, threads, NULL);
  oracle_csr_free(&g);
  if (edges_out) *edges_out = m;
  return t;
}

/* ------------------------------------------------------------------------ */
/* Restatement of the reference's bit-block algorithm                        */
/* (count_triangles tribit.cu:656-786, kernel tribit.cu:519-586).            */
/* ------------------------------------------------------------------------ */

/* L(v, cb): bits of v's lower neighbours w (w < v) in 32-column block cb, bit
 * (31 - w % 32) (create_non_compact_mask_l tribit.cu:588-594, OR-reduced by
 * (cb, v) key tribit.cu:672-682). Found, as in the kernel (tribit.cu:552-555),
 * by a search among v's lower neighbours. */
static uint32_t lower_mask(const uint64_t* lptr, const uint32_t* lcol, uint32_t v, uint32_t cb) {
  const uint32_t* a = lcol + lptr[v];
  uint64_t n = lptr[v + 1] - lptr[v], lo = 0, hi = n;
  while (lo < hi) { /* first w with w / 32 >= cb */
    uint64_t mid = (lo + hi) / 2;
    if (a[mid] / 32 < cb)
      lo = mid + 1;
    else
      hi = mid;
  }
  uint32_t m = 0;
  for (uint64_t k = lo; k < n && a[k] / 32 == cb; ++k) m |= 1u << (31 - a[k] % 32);
  return m;
}

/* Only the work decomposition of the reference (compute_n_blocks_per_row
 * tribit.cu:645-654, total_num_blocks tribit.cu:758): sum over U entries
 * (u, rb) of ceil(neighbours of u in blocks >= rb / 32) warps, 4 warps a CTA.
 * entries must be folded, deduplicated and (c, r)-sorted (oracle_fold_dedup). */
uint64_t oracle_tribit_blocks(const uint64_t* e, uint64_t m) {
  uint64_t warps = 0, i = 0;
  while (i < m) {
    uint32_t c = (uint32_t)(e[i] >> 32);
    uint64_t j = i;
    while (j < m && (uint32_t)(e[j] >> 32) == c) j++;
    uint64_t du = j - i;
    if (du >= 2) {
      uint64_t k = i;
      while (k < j) {
        uint32_t rb = (uint32_t)e[k] / 32;
        warps += (j - k + 31) / 32;
        while (k < j && (uint32_t)e[k] / 32 == rb) k++;
      }
    }
    i = j;
  }
  return (warps + 3) / 4;
}

uint64_t oracle_count_tribit(const uint64_t* entries, uint64_t n_entries, uint64_t n, uint64_t* blocks_of_threads) {
  uint64_t* e = (uint64_t*)malloc((n_entries ? n_entries : 1) * sizeof(uint64_t));
  memcpy(e, entries, n_entries * sizeof(uint64_t));
  uint64_t m = oracle_fold_dedup(e, n_entries); /* sorted by (c, r), c < r */
  /* Higher-neighbour lists (U side, before the purge) in edge order. */
  uint64_t* uptr = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
  uint64_t* lptr = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
  uint32_t* ucol = (uint32_t*)malloc((m ? m : 1) * sizeof(uint32_t));
  uint32_t* lcol = (uint32_t*)malloc((m ? m : 1) * sizeof(uint32_t));
  for (uint64_t i = 0; i < m; ++i) {
    uptr[(e[i] >> 32) + 1]++;
    lptr[(uint32_t)e[i] + 1]++;
  }
  for (uint64_t v = 0; v < n; ++v) uptr[v + 1] += uptr[v], lptr[v + 1] += lptr[v];
  uint64_t* lfill = (uint64_t*)malloc((n + 1) * sizeof(uint64_t));
  memcpy(lfill, lptr, (n + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < m; ++i) {
    uint32_t c = (uint32_t)(e[i] >> 32), r = (uint32_t)e[i];
    ucol[i] = r; /* edges sorted by (c, r): row c's higher neighbours in order */
    lcol[lfill[r]++] = c; /* ascending c for each r because edges are (c, r)-sorted */
  }
  free(lfill);
  free(e);
  uint64_t tri = 0, warps = 0;
  for (uint64_t u = 0; u < n; ++u) {
    const uint32_t* nu = ucol + uptr[u];
    uint64_t du = uptr[u + 1] - uptr[u];
    /* Purge: rows with exactly one higher neighbour carry no U entry
     * (flag_non_singletons tribit.cu:604-615, select tribit.cu:698-707). */
    if (du < 2) continue;
    uint64_t k = 0;
    while (k < du) {
      uint32_t rb = nu[k] / 32;
      uint32_t umask = 0;
      uint64_t k2 = k;
      while (k2 < du && nu[k2] / 32 == rb) umask |= 1u << (31 - nu[k2] % 32), k2++;
      /* Work for this U entry: ceil(remaining neighbours / 32) warps
       * (compute_n_blocks_per_row tribit.cu:645-654). */
      uint64_t remaining = du - k;
      warps += (remaining + 31) / 32;
      /* Each covered neighbour v adds popc(U(u, rb) & L(v, rb))
       * (tribit.cu:547-583). Neighbours before block rb contribute 0. */
      for (uint64_t q = k; q < du; ++q) tri += (uint64_t)__builtin_popcount(umask & lower_mask(lptr, lcol, nu[q], rb));
      k = k2;
    }
  }
  if (blocks_of_threads) *blocks_of_threads = (warps + 3) / 4; /* tribit.cu:758 */
  free(uptr);
  free(lptr);
  free(ucol);
  free(lcol);
  return tri;
}

/* ---- seeded R-MAT generator (for the reference arm of the benchmark) ------
 * The benchmark's reference arm must not load the product library, yet it has
 * to count the same graph. This restates the product's counter-based R-MAT
 * generator (Chakrabarti, Zhan and Faloutsos, SDM 2004) from its definition:
 * entry i draws one SplitMix64 value per two levels, stream value
 * mix(mix(seed) ^ (i * 32 + level / 2) * 0xD6E8FEB86659FD93), and at level l
 * the (l & 1)-th 32-bit half picks a quadrant against the cumulative 32-bit
 * thresholds floor(p * 2^32) of a, a + b, a + b + c: b sets the column bit,
 * c the row bit, d both. Word i = (row << 32) | col. A CPU test checks it
 * against the product's tribit_gen_rmat word for word. */
static uint64_t g_splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static uint32_t g_threshold(double p) {
  double t = floor(p * 4294967296.0);
  if (t < 0) t = 0;
  if (t > 4294967295.0) t = 4294967295.0;
  return (uint32_t)t;
}

typedef struct {
  uint64_t seed_mix, lo, hi;
  int scale;
  uint32_t ta, tab, tabc;
  uint64_t* out;
} rmat_job;

static void* rmat_worker(void* arg) {
  const rmat_job* j = (const rmat_job*)arg;
  for (uint64_t i = j->lo; i < j->hi; ++i) {
    uint32_t r = 0, c = 0;
    uint64_t h = 0;
    for (int l = 0; l < j->scale; ++l) {
      if ((l & 1) == 0) h = g_splitmix(j->seed_mix ^ (((i << 5) | (uint64_t)(l >> 1)) * 0xD6E8FEB86659FD93ull));
      const uint32_t x = (uint32_t)(h >> ((l & 1) * 32));
      const uint32_t bit = 1u << (j->scale - 1 - l);
      if (x >= j->tabc) {
        r |= bit;
        c |= bit;
      } else if (x >= j->tab) {
        r |= bit;
      } else if (x >= j->ta) {
        c |= bit;
      }
    }
    j->out[i] = ((uint64_t)r << 32) | c;
  }
  return NULL;
}

int oracle_gen_rmat(int scale, uint64_t edge_factor, double a, double b, double c, uint64_t seed, int threads,
                    uint64_t* out) {
  if (scale < 1 || scale > 31 || !out || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return 1;
  if (threads < 1) threads = 1;
  const uint64_t m = edge_factor << scale;
  rmat_job* jobs = (rmat_job*)malloc(sizeof(rmat_job) * (size_t)threads);
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
  if (!jobs || !th) {
    free(jobs);
    free(th);
    return 8;
  }
  const uint64_t chunk = (m + (uint64_t)threads - 1) / (uint64_t)threads;
  for (int k = 0; k < threads; ++k) {
    jobs[k].seed_mix = g_splitmix(seed);
    jobs[k].lo = (uint64_t)k * chunk < m ? (uint64_t)k * chunk : m;
    jobs[k].hi = jobs[k].lo + chunk < m ? jobs[k].lo + chunk : m;
    jobs[k].scale = scale;
    jobs[k].ta = g_threshold(a);
    jobs[k].tab = g_threshold(a + b);
    jobs[k].tabc = g_threshold(a + b + c);
    jobs[k].out = out;
    pthread_create(&th[k], NULL, rmat_worker, &jobs[k]);
  }
  for (int k = 0; k < threads; ++k) pthread_join(th[k], NULL);
  free(jobs);
  free(th);
  return 0;
}

/* Writes entries as a symmetric pattern Matrix Market file, one 1-based
 * "max min" line per entry (self-loops and duplicates kept as given), the
 * input the reference's read_mtx (tribit.cu:228-269) parses. 0 ok, 2 I/O. */
int oracle_write_mtx(const char* path, uint64_t num_nodes, const uint64_t* entries, uint64_t n_entries) {
  FILE* f = fopen(path, "wb");
  if (!f) return 2;
  char* buf = (char*)malloc(1 << 22);
  if (!buf) {
    fclose(f);
    return 8;
  }
  size_t used = (size_t)snprintf(buf, 256, "%%%%MatrixMarket matrix coordinate pattern symmetric\n%llu %llu %llu\n",
                                 (unsigned long long)num_nodes, (unsigned long long)num_nodes,
                                 (unsigned long long)n_entries);
  int bad = 0;
  for (uint64_t i = 0; i < n_entries && !bad; ++i) {
    const uint32_t a = (uint32_t)(entries[i] >> 32), b = (uint32_t)entries[i];
    const uint32_t hi = a > b ? a : b, lo = a > b ? b : a;
    used += (size_t)snprintf(buf + used, 32, "%u %u\n", hi + 1, lo + 1);
    if (used > (1 << 22) - 64) {
      bad = fwrite(buf, 1, used, f) != used;
      used = 0;
    }
  }
  if (!bad && used) bad = fwrite(buf, 1, used, f) != used;
  free(buf);
  if (fclose(f) != 0) bad = 1;
  return bad ? 2 : 0;
}
