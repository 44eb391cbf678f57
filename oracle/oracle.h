/* CPU oracle for exact triangle counting -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker for the tribit_b200 GPU counter. Only the test
 * suite, the smoke check and the benchmark's CPU-baseline leg load it; the
 * product never links or calls it.
 *
 * It restates, in plain C, the semantics of the reference single-GPU counter
 * (sixt99/TriBIT, src/single_gpu/tribit.cu):
 *   - oracle_read_mtx          follows read_mtx              (tribit.cu:228-269)
 *   - oracle_fold_dedup        follows the fold at read time  (tribit.cu:258-267)
 *                              and radix_sort+unique          (tribit.cu:666-667)
 *   - oracle_count_tribit      restates the L/U bit-block algorithm of
 *                              count_triangles / compute_binary_popcount_mma_9
 *                              (tribit.cu:656-786, 519-586) including its
 *                              "Blocks of threads" figure (tribit.cu:758)
 *   - oracle_csr_build + oracle_count_csr
 *                              a merge-intersection counter over the oriented
 *                              CSR (id order or (degree, id) order); its count
 *                              equals the reference's for any orientation.
 *
 * Parity pins: tests/golden holds closed-form known answers (K_n, wheels,
 * stars, disjoint cliques) and the count of the reference's bundled
 * wiki-Vote.mtx (608,389 triangles, 100,762 edges), plus counts printed by the
 * reference binary itself on generated graphs (tests/golden/ref_counts.json).
 */
#ifndef TRIBIT_ORACLE_H
#define TRIBIT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status: 0 ok, 2 cannot open, 3 malformed, 4 not square, 8 out of memory. */
int oracle_read_mtx(const char* path, uint64_t* num_nodes, uint64_t** entries, uint64_t* n_entries);
void oracle_free(void* p);

/* Fold every entry to (min << 32) | max, drop self-loops, sort and dedup in
 * place. Returns the number of undirected edges kept. */
uint64_t oracle_fold_dedup(uint64_t* entries, uint64_t n_entries);

/* Oriented CSR. order 0: u -> v iff u < v (the reference's id order).
 * order 1: u -> v iff (deg u, u) < (deg v, v), relabelled to that rank. */
typedef struct {
  uint64_t n;
  uint64_t m;
  uint64_t* row_ptr; /* n + 1 */
  uint32_t* col;     /* m, sorted within each row */
} oracle_csr;

/* entries must be folded and deduplicated (oracle_fold_dedup). */
int oracle_csr_build(const uint64_t* edges, uint64_t m, uint64_t n, int order, oracle_csr* out);
void oracle_csr_free(oracle_csr* g);

/* Merge-intersection count over the oriented CSR with `threads` host threads.
 * Returns the triangle count; *seconds (if non-null) receives wall time. */
uint64_t oracle_count_csr(const oracle_csr* g, int threads, double* seconds);

/* Same over the sample of 32-row blocks b with b % stride == offset: the
 * triangles whose lowest vertex lies in those blocks. */
uint64_t oracle_count_csr_sample(const oracle_csr* g, int threads, uint64_t stride, uint64_t offset, double* seconds);

/* Per-row triangle counts: out[u] = sum over v in N+(u) of |N+(u) & N+(v)|. */
void oracle_count_rows(const oracle_csr* g, uint64_t* out);

/* Whole pipeline on raw entries (copied): fold, dedup, orient, count. */
uint64_t oracle_count_entries(const uint64_t* entries, uint64_t n_entries, uint64_t n, int order, int threads,
                              uint64_t* edges_out);

/* Restatement of the reference's own bit-block algorithm (id order, 32-column
 * L and U blocks, MSB-first masks, singleton purge). Single threaded; for small
 * and medium graphs. *blocks_of_threads receives ceil(total_warps / 4). */
uint64_t oracle_count_tribit(const uint64_t* entries, uint64_t n_entries, uint64_t n, uint64_t* blocks_of_threads);

/* The reference's CTA count alone (ceil(total warps / 4), tribit.cu:758) for
 * folded, deduplicated, sorted edges; cheap at any size. */
uint64_t oracle_tribit_blocks(const uint64_t* edges, uint64_t m);

/* Seeded R-MAT entries, word for word those of the product's tribit_gen_rmat
 * (edge_factor << scale words, (row << 32) | col, duplicates and self-loops
 * kept), on `threads` host threads. 0 ok, 1 bad argument, 8 out of memory. */
int oracle_gen_rmat(int scale, uint64_t edge_factor, double a, double b, double c, uint64_t seed, int threads,
                    uint64_t* out);

/* Entries as a symmetric pattern .mtx (1-based "max min" lines, as given):
 * the reference binary's input. 0 ok, 2 I/O error, 8 out of memory. */
int oracle_write_mtx(const char* path, uint64_t num_nodes, const uint64_t* entries, uint64_t n_entries);

#ifdef __cplusplus
}
#endif
#endif
