/* tribit_b200 -- exact triangle counting on one NVIDIA B200 (sm_100a).
 *
 * C-ABI boundary of the counter. Plain pointers and sizes only; every entry
 * point returns a tribit_status and never exits the process.
 *
 * Reference interfaces replaced (paths within sixt99/TriBIT):
 *   count_triangles(zipped, nnz, cfg, print)  src/single_gpu/tribit.cu:656
 *     -> tribit_count_edges / tribit_count_edges_device
 *   read_mtx(path, zipped)                     src/single_gpu/tribit.cu:228
 *     -> tribit_read_mtx, tribit_count_mtx
 *   allocate_memory() + cudaMalloc_log pool    src/single_gpu/tribit.cu:825, :48
 *     -> tribit_create (per-device context owning a reusable device arena)
 *   init_gpu_kernel5(gpu_id)                   src/multi_gpu/cuda/main5_multi.cu:578
 *     -> tribit_create (options.device)
 *   count_partial_triangles_diagonal(...)      src/multi_gpu/cuda/main5_multi.cu:589
 *     (the reference's FFI precedent, declared at src/multi_gpu/src/main.rs:15-36)
 *     -> tribit_count_edges (host zipped entries in, uint64 count out)
 *   main / program_options                     src/single_gpu/tribit.cu:282, :840
 *     -> the `tribit` CLI, a thin caller of this header
 *
 * Entry words use the reference's zipped layout (a << 32) | b with 0-based
 * vertex ids (tribit.cu:258-266). The counter folds each entry to
 * (min, max), drops self-loops (a == b) and deduplicates, so both the folded
 * words read_mtx produces and raw, unfolded edge lists are accepted.
 *
 * Threading: a context belongs to one device and may be used by one host
 * thread at a time. Distinct contexts are independent.
 */
#ifndef TRIBIT_H
#define TRIBIT_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tribit_status {
  TRIBIT_OK = 0,
  TRIBIT_ERR_INVALID_ARGUMENT = 1,
  TRIBIT_ERR_IO = 2,          /* cannot open / read / write a file        (ref: tribit.cu:230 throws) */
  TRIBIT_ERR_FORMAT = 3,      /* malformed Matrix Market size line         */
  TRIBIT_ERR_NOT_SQUARE = 4,  /* rows != cols                              (ref: tribit.cu:241-245 throws) */
  TRIBIT_ERR_ID_RANGE = 5,    /* an entry names a vertex >= num_nodes      (ref: unchecked) */
  TRIBIT_ERR_TOO_LARGE = 6,   /* beyond the 32-bit id / edge-count limits  (ref: tribit.cu:773 throws) */
  TRIBIT_ERR_CUDA = 7,        /* CUDA runtime error; see tribit_last_error */
  TRIBIT_ERR_OUT_OF_MEMORY = 8, /* device or host allocation failed      (ref: tribit.cu:62-65 exit(1)) */
  TRIBIT_ERR_NO_DEVICE = 9,   /* no usable CUDA device                     */
  TRIBIT_ERR_TIMEOUT = 10,    /* a bounded device-side wait gave up        */
  TRIBIT_ERR_NO_MODEL = 11,   /* learned dispatch requested without a model */
  TRIBIT_ERR_INTERNAL = 12
} tribit_status;

/* Vertex orientation: every triangle is counted once, at its lowest vertex. */
enum {
  TRIBIT_ORDER_DEGREE = 0, /* rank by (degree, id), orient low -> high rank (default) */
  TRIBIT_ORDER_ID = 1      /* orient u -> v iff u < v, as the reference does (tribit.cu:261-267) */
};

/* How each 32-row block of the oriented graph picks its counting variant. */
enum {
  TRIBIT_DISPATCH_PLAIN = 0,   /* fixed thresholds on row-block features */
  TRIBIT_DISPATCH_LEARNED = 1, /* MLP over row-block features (tribit_model_*) */
  TRIBIT_DISPATCH_MERGE = 2,   /* force sorted-list merge everywhere */
  TRIBIT_DISPATCH_BITMAP = 3,  /* force LOP3 + popc on bit-packed rows everywhere */
  TRIBIT_DISPATCH_MMA = 4      /* force b1 AND+POPC tensor-core tiles everywhere */
};

/* Counting variants, in the order used by per-variant arrays below. */
enum { TRIBIT_VARIANT_MMA = 0, TRIBIT_VARIANT_BITMAP = 1, TRIBIT_VARIANT_MERGE = 2, TRIBIT_NUM_VARIANTS = 3 };

typedef struct tribit_options {
  int device;            /* CUDA device ordinal */
  int order;             /* TRIBIT_ORDER_* */
  int dispatch;          /* TRIBIT_DISPATCH_* */
  int ctas_per_sm;       /* counting-kernel CTAs per SM; 0 = tuned default */
  uint32_t reserved[8];  /* must be zero */
} tribit_options;

/* Bit-tile variant: the product's arithmetic. */
enum { TRIBIT_TILES_MMA_SYNC = 0, /* legacy warp-level mma.sync m16n8k256 b1 AND+POPC */
       TRIBIT_TILES_TCGEN05 = 1   /* tcgen05.mma kind::i8 on bits unpacked to 0/1, s32 in TMEM */ };

typedef struct tribit_result {
  uint64_t triangles;         /* exact count */
  uint64_t num_nodes;         /* n as given */
  uint64_t entries;           /* input entries */
  uint64_t edges;             /* undirected edges after fold, self-loop removal, dedup */
  uint64_t blocks_of_threads; /* CTAs of the counting launch ("Blocks of threads") */
  uint64_t row_blocks;        /* non-empty 32-row blocks of the oriented graph */
  uint64_t row_blocks_by_variant[TRIBIT_NUM_VARIANTS];
  float h2d_ms;               /* host -> device copy of the entries (host-input calls; the degree
                                 pass of each uploaded piece runs while the next one is copied) */
  float preprocess_ms;        /* fold, dedup, orient, CSR and bit-block build (after the upload) */
  float kernel_ms;            /* counting kernel(s) */
  float total_ms;             /* whole call, device time */
  uint32_t count_kernels;     /* kernels one counting launch issues */
  uint32_t hub_edges;         /* edges the merge variant counts by walking u's tail against the
                                 staged row of v (the hub pass) */
  float load_ms;              /* tribit_count_mtx / tribit_count_loaded: wall time of reading the
                                 file into device memory (tribit_load_mtx); else 0 */
  uint32_t load_gpu_parse;    /* 1 when the GPU parsed the file, 0 when the host grammar did */
  uint32_t stream_ranges;     /* tribit_count_edges: 1 when the graph fit the device budget, else the
                                 rank ranges it was counted in (see tribit_set_device_budget) */
  uint32_t stream_tasks;      /* device counts those ranges took: 1 in one piece and with
                                 TRIBIT_STREAM_ROWS, one per pair of ranges with TRIBIT_STREAM_PAIRS */
  uint32_t stream_tier;       /* 0 (one piece), TRIBIT_STREAM_ROWS or TRIBIT_STREAM_PAIRS */
} tribit_result;

/* How tribit_count_edges counts a graph past the device budget. */
enum {
  TRIBIT_STREAM_AUTO = 0,  /* ROWS when the oriented rows fit the budget, else PAIRS */
  TRIBIT_STREAM_ROWS = 1,  /* rows built one rank range at a time, kept on the device, counted once */
  TRIBIT_STREAM_PAIRS = 2  /* each pair of rank ranges counted as a graph of its own */
};

typedef struct tribit_context tribit_context;

/* ---- context --------------------------------------------------------- */
void tribit_default_options(tribit_options* opts);
tribit_status tribit_create(const tribit_options* opts, tribit_context** ctx);
void tribit_destroy(tribit_context* ctx);
/* Run all later work of this context on `cuda_stream` (a cudaStream_t; NULL
 * restores the context's own stream). Waits for work queued on the previous
 * stream. Device inputs given to later calls must be complete on the device
 * when the call is made, or be produced on this stream. */
tribit_status tribit_set_stream(tribit_context* ctx, void* cuda_stream);
const char* tribit_status_string(tribit_status st);
const char* tribit_last_error(const tribit_context* ctx);
const char* tribit_version(void);

/* ---- single graph ------------------------------------------------------ */
/* Host entries -> exact count (H2D copy, preprocessing, counting, D2H).
 * A graph whose device buffers exceed the context's device budget (all the
 * memory the device has free, unless tribit_set_device_budget says less) is
 * counted in pieces: its entries are streamed through the GPU to rank them
 * and sort them into host buckets by rank range (result.stream_ranges > 1).
 * Then either each range's rows are built on the device in turn into one
 * oriented graph that stays resident and is counted once (TRIBIT_STREAM_ROWS:
 * the preprocessing scratch is what did not fit), or, when even the rows do
 * not fit, each pair of ranges is counted on the device as a graph of its own
 * (TRIBIT_STREAM_PAIRS). The reference splits a graph too large for a GPU into
 * partitions and tasks of at most 1e9 entries over several GPUs
 * (src/multi_gpu/src/main.rs:98-220). A TRIBIT_STREAM_ROWS count leaves the
 * graph prepared for tribit_launch_count; a TRIBIT_STREAM_PAIRS count leaves
 * none (tribit_launch_count then fails). */
tribit_status tribit_count_edges(tribit_context* ctx, const uint64_t* entries, uint64_t n_entries, uint64_t num_nodes,
                                 tribit_result* out);
/* Device memory (bytes) a one-piece tribit_count_edges of n_entries entries on
 * num_nodes vertices takes in this context (its arena, staged input included). */
tribit_status tribit_device_bytes(tribit_context* ctx, uint64_t n_entries, uint64_t num_nodes, uint64_t* bytes);
/* Caps the device memory later tribit_count_edges calls of this context may
 * use (bytes; 0 = what the device has free at the call). */
tribit_status tribit_set_device_budget(tribit_context* ctx, uint64_t bytes);
/* Streamed counts of later tribit_count_edges calls: `tier` one of
 * TRIBIT_STREAM_*, `range_entries` an upper bound on the oriented entries of a
 * rank range (0: as many as the budget allows; a bound at or below the
 * longest row fails with TRIBIT_ERR_OUT_OF_MEMORY). A forced tier that cannot
 * fit the budget fails with TRIBIT_ERR_OUT_OF_MEMORY. */
tribit_status tribit_set_stream_options(tribit_context* ctx, int tier, uint64_t range_entries);
/* Same with the entries already in device memory. */
tribit_status tribit_count_edges_device(tribit_context* ctx, const uint64_t* d_entries, uint64_t n_entries,
                                        uint64_t num_nodes, tribit_result* out);
/* Two-phase form: build the oriented, bit-packed graph once, then launch the
 * counting kernel(s) any number of times. tribit_launch_count only enqueues
 * work on the context's stream; tribit_read_count waits and returns it. */
tribit_status tribit_prepare_device(tribit_context* ctx, const uint64_t* d_entries, uint64_t n_entries,
                                    uint64_t num_nodes, tribit_result* out);
tribit_status tribit_launch_count(tribit_context* ctx);
tribit_status tribit_read_count(tribit_context* ctx, tribit_result* out);

/* ---- launch tuning and CUDA-graph replay (no counterpart in the reference) - */
typedef struct tribit_tuning {
  int ctas_per_sm;      /* CTAs per SM of the warp-per-piece kernels; 0 = default (6) */
  uint32_t piece_width; /* neighbours per work piece: a multiple of 32, >= 32 (default 64) */
  float tile_min_nnz;   /* plain dispatch: fewest edges of a row block sent to the bit tiles, which
                           also need 1/8 of the tile's cells set (default 64; 1e30 = off) */
  float count_ms;       /* tribit_autotune: measured counting time of this setting */
  float merge_ratio;    /* plain dispatch: a row block not sent to the tiles goes to the sorted-list
                           merge when its neighbours' bit rows average at least merge_ratio times
                           its own rows' length, else to the bitmap sweep (default 0.75; 1e30 = never) */
  uint32_t launch_model; /* TRIBIT_LAUNCH_KERNELS: one persistent kernel per variant;
                            TRIBIT_LAUNCH_QUEUE: the row-piece and hub work in one persistent
                            kernel whose CTAs take heavy rows, hub CTA pieces, then per warp
                            bitmap, merge and hub pieces from the device cursors (the bit tiles
                            and the fallback rows keep their kernels; ctas_per_sm unused);
                            TRIBIT_LAUNCH_AUTO (default): the queue up to 2^24 entries, where
                            kernel boundaries weigh most, else the kernels */
} tribit_tuning;
enum { TRIBIT_LAUNCH_KERNELS = 0, TRIBIT_LAUNCH_QUEUE = 1, TRIBIT_LAUNCH_AUTO = 2 };
tribit_status tribit_get_tuning(tribit_context* ctx, tribit_tuning* out);
/* Applies to later calls, and rebuilds the schedule of the prepared graph. */
tribit_status tribit_set_tuning(tribit_context* ctx, const tribit_tuning* in);
/* Times `reps` counting launches of the prepared graph for each setting of a
 * small grid (launch model x CTAs/SM x piece width x tile threshold), keeps
 * the fastest (median) and returns it. Counts stay exact under every setting. */
tribit_status tribit_autotune(tribit_context* ctx, uint32_t reps, tribit_tuning* best);
/* Arithmetic of the bit-tile variant (TRIBIT_TILES_*), for later launches;
 * rebuilds nothing, drops a captured launch. Default TRIBIT_TILES_TCGEN05. */
tribit_status tribit_set_tile_engine(tribit_context* ctx, int engine);
/* Poll budget of the tcgen05 tile kernel's bounded mbarrier wait, for later
 * launches (0 = the default, 2^22 polls). When one wait runs out, the CTA
 * stops as a whole, waits (with its own bound) for the MMAs it committed,
 * frees its TMEM and returns; tribit_read_count then reports
 * TRIBIT_ERR_TIMEOUT. A count is therefore either exact or an error, never
 * wrong, whatever the budget. Drops a captured launch. */
tribit_status tribit_set_tile_wait_polls(tribit_context* ctx, uint32_t max_polls);
/* Failure-detection test: one counting launch of the prepared graph in which
 * the tcgen05 tile kernel issues no MMA, so its bounded mbarrier wait runs out
 * after max_polls polls; the kernel frees its TMEM and returns, and
 * tribit_read_count then reports TRIBIT_ERR_TIMEOUT. Preparing again clears it. */
tribit_status tribit_test_tile_timeout(tribit_context* ctx, uint32_t max_polls);
/* Captures the counting launch of the prepared graph (or batch) into a CUDA
 * graph; tribit_launch_count then replays it with one graph launch. Preparing
 * another input or changing the tuning drops the capture. */
tribit_status tribit_capture_count(tribit_context* ctx);
/* After tribit_count_batch: per-graph counts of the latest counting launch. */
tribit_status tribit_read_batch_counts(tribit_context* ctx, uint64_t* triangles_out, uint32_t num_graphs);

/* ---- Matrix Market ------------------------------------------------------ */
/* Reads a coordinate .mtx with the reference's semantics (tribit.cu:228-269):
 * banner line, '%' lines skipped, "rows cols nnz", rows must equal cols,
 * 1-based "r c [values...]" entries, values ignored, self-loops dropped, each
 * entry folded to (min << 32) | max. *entries is allocated with malloc and
 * released with tribit_free_host. */
tribit_status tribit_read_mtx(const char* path, uint64_t* num_nodes, uint64_t** entries, uint64_t* n_entries);
void tribit_free_host(void* p);
/* Reads a Matrix Market file into the context's device memory, with the
 * semantics of tribit_read_mtx (the same entries in the same order), for
 * tribit_count_loaded. The file's bytes are read by host threads into pinned
 * buffers and copied to the GPU piece by piece (each piece's copy overlaps
 * the reading of the next), and the GPU parses the text: the reference's
 * read_mtx (tribit.cu:228-269) parses on one host thread. A file with any
 * line outside the common form "id blanks id [blanks number]*" (blank lines
 * allowed) is parsed by the host's exact grammar instead. The loaded graph
 * stays until the next load or tribit_destroy. */
tribit_status tribit_load_mtx(tribit_context* ctx, const char* path, uint64_t* num_nodes, uint64_t* n_entries);
/* Counts the graph of the latest tribit_load_mtx (as tribit_count_edges_device). */
tribit_status tribit_count_loaded(tribit_context* ctx, tribit_result* out);
/* Copies the loaded entries (n_entries words) to host memory; out may be NULL
 * to query the count. */
tribit_status tribit_loaded_entries(tribit_context* ctx, uint64_t* out, uint64_t cap, uint64_t* n_entries);
/* tribit_load_mtx + tribit_count_loaded. */
tribit_status tribit_count_mtx(tribit_context* ctx, const char* path, tribit_result* out);

/* ---- WebGraph BVGraph ---------------------------------------------------- */
/* Reads a graph in WebGraph's BVGraph format (basename.properties,
 * basename.graph and, when present, basename.offsets), the input of the
 * reference's multi-GPU loader (src/multi_gpu/src/main.rs:88, the Rust
 * webgraph crate), and folds every arc (src, dst), src != dst, to
 * (min << 32) | max as that loader does (main.rs:142-161). Big-endian streams
 * with gamma, delta, unary and zeta codes; with offsets the nodes are decoded
 * in parallel. *entries is allocated with malloc (tribit_free_host). */
tribit_status tribit_read_bvgraph(const char* basename, uint64_t* num_nodes, uint64_t** entries, uint64_t* n_entries);
/* tribit_read_bvgraph + tribit_count_edges. */
tribit_status tribit_count_bvgraph(tribit_context* ctx, const char* basename, tribit_result* out);

/* ---- batches ----------------------------------------------------------- */
/* num_graphs independent graphs in one persistent counting launch. Graph g's
 * entries are entries[entry_offsets[g] .. entry_offsets[g + 1]) with vertex
 * ids in [0, num_nodes[g]). triangles_out[g] receives graph g's exact count. */
tribit_status tribit_count_batch(tribit_context* ctx, const uint64_t* entries, const uint64_t* entry_offsets,
                                 const uint32_t* num_nodes, uint32_t num_graphs, uint64_t* triangles_out,
                                 tribit_result* out);

/* ---- counting without device allocation ---------------------------------- */
/* No counterpart in the reference. For callers that cannot allocate device
 * memory while they count: a process whose framework owns the device memory
 * through its own allocator or a pool reserved up front (as the reference
 * reserves 95% of free memory at start-up), or a latency-bound loop that must
 * not pay the implicit synchronisation of cudaMalloc / cudaFree.
 * Counts the graph in d_entries (device memory, zipped words as for
 * tribit_count_edges; degree order; the plain dispatch rule over bit tiles,
 * the bitmap sweep and the merge variant with its hub lists, as a context's
 * TRIBIT_DISPATCH_PLAIN does, when the hub lists fit the scratch; else bit
 * tiles and the bitmap sweep only, which on power-law graphs take 2-3 times
 * longer) on `stream` (a
 * cudaStream_t; NULL = the legacy default stream), taking every intermediate
 * buffer from one fixed scratch array compiled into the library
 * (tribit_noalloc_scratch_bytes() = 32 MiB, held on each device that loads it
 * until exit). Allocates no device or host memory and needs no context.
 * Asynchronous: when the stream reaches the end of the work, d_result (device,
 * 4 x uint64) holds [0] triangles, [1] undirected edges, [2] error flags
 * (TRIBIT_NOALLOC_FLAG_*; any flag set means [0] is not a valid count), [3] 1
 * when the hub lists fitted (the merge variant was open to the plain rule),
 * else 0.
 * Returns TRIBIT_ERR_TOO_LARGE, launching nothing, for a graph whose buffers
 * do not fit the scratch array (roughly 25 bytes per entry + 80 per vertex
 * without the hub lists, 33 + 155 with them).
 * The first call on a device looks up the array's device address: make it
 * before capturing stream work on that device. All calls share the array, so
 * calls whose GPU work overlaps race: order them on one stream. */
enum {
  TRIBIT_NOALLOC_FLAG_ID_RANGE = 1u << 0, /* an entry named a vertex >= num_nodes */
  TRIBIT_NOALLOC_FLAG_RESERVED = 1u << 1, /* never set */
  TRIBIT_NOALLOC_FLAG_TIMEOUT = 1u << 2   /* a bounded wait of the tcgen05 tile kernel gave up
                                             (the count is incomplete; tribit_count_edges
                                             reports the same event as TRIBIT_ERR_TIMEOUT) */
};
tribit_status tribit_count_edges_noalloc(const uint64_t* d_entries, uint64_t n_entries, uint64_t num_nodes,
                                         uint64_t* d_result, void* stream);
uint64_t tribit_noalloc_scratch_bytes(void);

/* ---- learned dispatcher (no counterpart in the reference) ----------------- */
/* A 16 -> 64 -> 64 -> 3 MLP (ReLU; BF16 weights, FP32 activations and
 * accumulation) maps the 16 features of a 32-row block to the predicted
 * log2(1 + SM cycles) each counting variant spends on it; learned dispatch
 * runs every row block on the variant with the smallest prediction. It only
 * schedules: counts are exact under any dispatcher. */
uint32_t tribit_model_num_params(void); /* 5443 */
/* Fresh model: weights uniform in +-sqrt(6 / fan_in) from `seed`, zero biases;
 * norm = in_mean[16], in_std[16], out_mean[3], out_std[3]. */
tribit_status tribit_model_init(tribit_context* ctx, uint64_t seed, const float* norm);
tribit_status tribit_model_load(tribit_context* ctx, const char* path);
tribit_status tribit_model_save(tribit_context* ctx, const char* path);
/* effective != 0: the parameters as the kernels use them (weights rounded to BF16). */
tribit_status tribit_model_get_params(tribit_context* ctx, float* out, int effective);
tribit_status tribit_model_set_params(tribit_context* ctx, const float* in);
/* y[rows x 3] = predicted log2(1 + cycles) per variant for features x[rows x 16]. */
tribit_status tribit_model_predict(tribit_context* ctx, const float* x, uint64_t rows, float* y);
/* Gradient of the mean squared error on normalised targets over all rows
 * (one batch), with respect to the effective parameters; *loss receives it. */
tribit_status tribit_model_gradients(tribit_context* ctx, const float* x, const float* y, uint64_t rows, float* grad,
                                     float* loss);
/* Adam (0.9, 0.999, 1e-8) on the GPU; *loss receives the last epoch's mean loss. */
tribit_status tribit_model_train(tribit_context* ctx, const float* x, const float* y, uint64_t rows, uint32_t epochs,
                                 uint32_t batch, float lr, uint64_t seed, float* loss);

/* ---- per-row-block data for the dispatcher (after tribit_prepare_device) -- */
/* Features of every 32-row block (num_row_blocks x 16 floats; out may be NULL
 * to query the count). */
tribit_status tribit_block_features(tribit_context* ctx, float* out, uint64_t cap, uint64_t* num_row_blocks);
/* The counting variant (TRIBIT_VARIANT_*) the context's dispatcher chose for
 * every 32-row block (out may be NULL to query the count). Blocks without
 * work keep their choice but get no pieces. */
tribit_status tribit_block_variants(tribit_context* ctx, uint8_t* out, uint64_t cap, uint64_t* num_row_blocks);
/* Counts with every row block on `variant` (TRIBIT_VARIANT_*) and records the
 * SM cycles each row block's pieces took (cycles_out[num_row_blocks]);
 * *triangles receives the count, which equals the normal one, and
 * *variant_ms the device time of the variant kernels (the rows too wide for
 * a warp, which every variant shares, run before it and are excluded). */
tribit_status tribit_block_times(tribit_context* ctx, int variant, float* cycles_out, uint64_t cap,
                                 uint64_t* triangles, float* variant_ms);

/* ---- synthetic graphs (host, seeded, thread-count independent) ---------- */
tribit_status tribit_gen_rmat(int scale, uint64_t edge_factor, double a, double b, double c, uint64_t seed,
                              uint64_t* out);
tribit_status tribit_gen_er(uint32_t n, uint64_t n_entries, uint64_t seed, uint64_t* out);
tribit_status tribit_gen_chung_lu(uint32_t n, uint64_t n_entries, double beta, double max_degree, uint64_t seed,
                                  uint64_t* out);
tribit_status tribit_gen_planted(uint32_t communities, uint32_t size, double p_in, uint32_t inter_per_vertex,
                                 uint64_t seed, uint64_t* out, uint64_t* n_entries);
tribit_status tribit_write_mtx(const char* path, uint64_t num_nodes, const uint64_t* entries, uint64_t n_entries);
/* The batched workload: num_graphs graphs, graph g with n log-uniform in
 * [min_n, max_n] and, by seed, Erdos-Renyi or Chung-Lu (exponent 2.1-2.8),
 * mean degree uniform in [8, 64], n * degree / 2 entries. Call with
 * entries == NULL to fill num_nodes[num_graphs] and entry_offsets[num_graphs+1]
 * only, then again with entries[entry_offsets[num_graphs]]. */
tribit_status tribit_gen_batch(uint32_t num_graphs, uint32_t min_n, uint32_t max_n, uint64_t seed, uint32_t* num_nodes,
                               uint64_t* entry_offsets, uint64_t* entries);

#ifdef __cplusplus
}
#endif
#endif
