/*
 * mnmgdl.h -- C-ABI of the B200 semi-naive Datalog engine (libmnmgdl.so).
 *
 * Plain C types only: device pointers are `void *` / `dl_entity *`, sizes are
 * int64_t, streams are `cudaStream_t` passed as `void *`. Every entry point
 * returns a dl_status; on failure dl_last_error() gives a message for the
 * calling thread. Device-side waits are bounded: a wait that runs out returns
 * DL_ERR_DEVICE_TIMEOUT instead of hanging.
 *
 * Reference interface each group replaces (paths within harp-lab/MNMGDatalog):
 *   dl_build_hash_table      <- get_hash_table            common/hash_table.cu:24-55
 *   dl_join                  <- get_join                  common/join.cu:51-87
 *   dl_join_sorted           <- get_join_nl               common/join.cu:144-180
 *   dl_sort_unique           <- thrust::sort(set_cmp) + thrust::unique(is_equal)   tc.cu:250-253
 *   dl_set_difference        <- thrust::set_difference(set_cmp)                    tc.cu:260-263
 *   dl_merge                 <- thrust::merge(set_cmp)                             tc.cu:276-279
 *   dl_unique_by_key_min     <- thrust::unique(is_equal_key) on set_cmp order       wcc.cu:320-323
 *   dl_remove_self_pairs     <- thrust::remove_if(is_key_equal_value)              sg.cu:176-179
 *   dl_diff_merge            <- set_difference + merge pair of one iteration       tc.cu:260-286
 *   dl_run_program / dl_run_tc / dl_run_sg / dl_run_wcc / dl_run_single_join
 *                            <- the program drivers       tc.cu:42-423, sg.cu:40-477,
 *                                                          wcc.cu:58-585, single_join.cu:39-396
 *   dl_generate_rows         <- parallel_generate         common/parallel_io.cu:79-108
 * The reference's exact C++ signatures (Entity*, int sizes, exit on error)
 * are provided on top of this ABI by include/mnmgdl_compat.h.
 */
#ifndef MNMGDL_H
#define MNMGDL_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define DL_API __attribute__((visibility("default")))
#else
#define DL_API
#endif

typedef enum dl_status {
    DL_OK = 0,
    DL_ERR_INVALID_ARGUMENT = 1,
    DL_ERR_CUDA = 2,
    DL_ERR_OUT_OF_MEMORY = 3,
    DL_ERR_DEVICE_TIMEOUT = 4,
    DL_ERR_OVERFLOW = 5,
    DL_ERR_NO_DEVICE = 6,
    DL_ERR_INTERNAL = 7
} dl_status;

/* Same layout as the reference's Entity (common/utils.cu:8-11). Relations
 * are ordered by the reference's set_cmp: signed key, then signed value. */
typedef struct dl_entity {
    int32_t key;
    int32_t value;
} dl_entity;

typedef struct dl_context dl_context;
typedef struct dl_hash_table dl_hash_table;
typedef struct dl_run dl_run;

typedef enum dl_program {
    DL_PROGRAM_TC = 0,          /* path(x,z) :- path(x,y), edge(y,z)          tc.cu */
    DL_PROGRAM_SG = 1,          /* same generation                            sg.cu */
    DL_PROGRAM_WCC = 2,         /* weakly connected components (min label)    wcc.cu */
    DL_PROGRAM_SINGLE_JOIN = 3  /* R(a,b), R(b,c) -> (a,c), deduplicated       single_join.cu */
} dl_program;

typedef enum dl_wcc_stop {
    /* Stop when |delta_k| == |delta_{k-1}| (wcc.cu:366-383): bit-exact with
     * the reference, including its early stop on some graphs. */
    DL_WCC_STOP_REFERENCE = 0,
    /* Stop when |delta_k| == 0: the true connected components. */
    DL_WCC_STOP_FIXPOINT = 1
} dl_wcc_stop;

/* How TC removes known tuples from a join output (same results either way). */
typedef enum dl_dedup {
    DL_DEDUP_AUTO = 0,  /* the engine's choice: BITMAP for TC when the bit matrix (and the column
                           offsets of its result rows, 1/16 of its size) fit in
                           dl_tuning.bitmap_max_gib and half the free device memory, else SORT */
    DL_DEDUP_SORT = 1,  /* radix sort of the join output + merge-path difference against sorted full */
    DL_DEDUP_HASH = 2,  /* full as a hash set of tuple words; one sort of the result at the end
                           (no per-iteration sort, but random-access bound: 1.7x slower on
                           the 1.9e9-tuple TC benchmark) */
    DL_DEDUP_BITMAP = 3 /* full as an n x n bit matrix over node ranks (n = distinct node ids):
                           each join word is one atomic test-and-set, no sort or merge per
                           iteration; needs 2 * n * n / 8 bytes (12.6 GB each for 317K nodes) */
} dl_dedup;

typedef struct dl_options {
    int32_t wcc_stop;        /* dl_wcc_stop */
    int32_t max_iterations;  /* 0 = run to the fixpoint */
    int32_t phase_timing;    /* 1 = record per-phase device times (adds events) */
    int32_t dedup;           /* dl_dedup (TC runs; SG and sessions always sort) */
    int32_t reserved[4];
} dl_options;

typedef struct dl_run_info {
    int32_t program;             /* dl_program */
    int32_t iterations;          /* counted like the reference (final empty pass included) */
    int64_t input_rows;
    int64_t output_rows;         /* rows of the program's output file */
    int64_t output_tuples;       /* TC/SG/single_join: |result|; WCC: # components */
    int64_t largest_component;   /* WCC only */
    int64_t nodes;               /* node ranks of the run: the distinct node ids of the input (TC on the
                                    bit-matrix path over a dense id range: every id of that range) */
    double seconds_total;        /* device time, H2D of the input through the last iteration */
    double seconds_init;         /* phase times (phase_timing = 1), reference CSV columns */
    double seconds_join;
    double seconds_dedup;
    double seconds_merge;
    double seconds_finalize;
    int64_t join_rows_total;     /* join output rows over all iterations (before dedup) */
    int64_t join_rows_max;       /* largest join output of one iteration */
} dl_run_info;

DL_API const char *dl_status_string(dl_status s);
DL_API const char *dl_last_error(void);
DL_API const char *dl_version(void);

/* Context: one CUDA device + stream (NULL = a stream owned by the context). */
DL_API dl_status dl_context_create(int32_t device, void *stream, dl_context **out);
DL_API dl_status dl_context_destroy(dl_context *ctx);
DL_API dl_status dl_context_synchronize(dl_context *ctx);
/* Waits for the context's stream, then frees the device memory the context keeps between
 * calls: its workspace and cached buffers (e.g. the bit matrix of the last TC run, 2 x n*n/8
 * bytes). Results of live runs and sessions are not touched; the next call allocates again.
 * No counterpart in the reference (its drivers free everything per iteration). */
DL_API dl_status dl_context_release_memory(dl_context *ctx);
DL_API dl_status dl_free(dl_context *ctx, void *device_ptr);

/* Engine knobs of a context (no counterpart in the reference; set by the
 * autotuner, mnmgdatalog_b200/autotune.py). Results never depend on them. */
typedef struct dl_tuning {
    int32_t sort_algorithm;       /* 1 = three-kernel LSD radix pass (default), 0 = onesweep */
    int32_t sort_ranking;         /* 1 = shared-memory peer masks (default), 0 = warp ballots */
    int32_t sort_keys_per_thread; /* onesweep tile: 16 (default) or 12 */
    int32_t dense_ratio;          /* TC/SG: one fused rewrite of full when |J| * ratio >= |large run| (1..64, default 4) */
    int32_t small_ratio;          /* TC/SG: small run folded into the large one at |small| * ratio >= |large| (1..64, default 4) */
    int32_t sort_input_tma;       /* three-kernel pass input: 1 = TMA double buffer (default), 0 = direct loads */
    double hash_load_factor;      /* dl_build_hash_table's default load factor (0 < lf < 1, default 0.5) */
    int32_t join_first_pass;      /* TC: 1 = the join emit also does the sort's first radix pass (default), 0 = not */
    int32_t bitmap_max_gib;       /* TC dedup AUTO: largest bit matrix + column offsets, GiB (0..1024, default 48; 0 = never) */
    int32_t bitmap_unit_rows;     /* bit-matrix TC: delta rows per work unit (1..16777216, default 65536) */
    int32_t cache_max_gib;        /* outgrown or released device buffers the context keeps for reuse, at most
                                     this many GiB (0..1024, default 96; 0 = free them at once) */
    int32_t bitmap_result;        /* bit-matrix TC: how the result rows leave the matrix (same rows):
                                     0 = through its transpose when a second matrix fits in bitmap_max_gib
                                     and the free memory, else from its columns (default); 1 = transpose;
                                     2 = columns (per 512-row block and target offsets, 1/16 of a matrix) */
} dl_tuning;
DL_API dl_status dl_context_get_tuning(const dl_context *ctx, dl_tuning *out);
DL_API dl_status dl_context_set_tuning(dl_context *ctx, const dl_tuning *tuning);
/* Copy `bytes` between any two host/device buffers on the context's stream
 * and wait for it (cudaMemcpyDefault). */
DL_API dl_status dl_memcpy(dl_context *ctx, void *dst, const void *src, int64_t bytes);

/* ---- relational operators on device arrays of dl_entity (set_cmp order) ---- */

/* Sort in place and drop duplicates; *n_out = new length. */
DL_API dl_status dl_sort_unique(dl_context *ctx, dl_entity *rel, int64_t n, int64_t *n_out);
/* Sort in place (duplicates kept). */
DL_API dl_status dl_sort(dl_context *ctx, dl_entity *rel, int64_t n);
/* out = a \ b for sorted duplicate-free a and b; out may alias a. */
DL_API dl_status dl_set_difference(dl_context *ctx, const dl_entity *a, int64_t na, const dl_entity *b,
                                   int64_t nb, dl_entity *out, int64_t *n_out);
/* out = stable merge of sorted a and b, duplicates kept (ties: a first). */
DL_API dl_status dl_merge(dl_context *ctx, const dl_entity *a, int64_t na, const dl_entity *b, int64_t nb,
                          dl_entity *out);
/* One semi-naive step on sets: delta_out = dedup(j) \ full, full_out = full u j.
 * full sorted duplicate-free, j sorted (duplicates allowed). full_out holds
 * nfull + *n_delta rows afterwards. Either output may be NULL. */
DL_API dl_status dl_diff_merge(dl_context *ctx, const dl_entity *full, int64_t nfull, const dl_entity *j,
                               int64_t nj, dl_entity *full_out, dl_entity *delta_out, int64_t *n_delta);
/* Keep the first row of every key run of a sorted relation (= minimum value). */
DL_API dl_status dl_unique_by_key_min(dl_context *ctx, dl_entity *rel, int64_t n, int64_t *n_out);
/* Drop rows with key == value, order kept. */
DL_API dl_status dl_remove_self_pairs(dl_context *ctx, dl_entity *rel, int64_t n, int64_t *n_out);

/* Multi-GPU exchange, send side: out = rel's rows grouped by destination
 * rank, rank 0's rows first; counts[r] (a host array of `ranks` entries)
 * receives the number of rows rank r owns. owner(row) = murmur3 fmix32 of
 * its key's unsigned 32-bit pattern, mod ranks -- the reference's
 * get_rank / get_send_count / get_rank_data (common/kernels.cu:199-242),
 * whose signed modulo is replaced by an unsigned one. With swap_columns != 0
 * every row (a, b) is written as (b, a) and owned by b (the reference's
 * reverse_entity_ar before an exchange, common/kernels.cu:313-324). The
 * order inside a destination's rows is unspecified. 1 <= ranks <= 4096;
 * out must not overlap rel. Returns after the rows are written. */
DL_API dl_status dl_partition(dl_context *ctx, const dl_entity *rel, int64_t n, int32_t ranks, int32_t swap_columns,
                              dl_entity *out, int64_t *counts);

/* dl_sort_unique without any memory allocation. No counterpart in the
 * reference. For callers that cannot call cudaMalloc at sort time -- device
 * memory already owned by another allocator's pool, a fixed device footprint
 * after start-up, or no room for the device-wide synchronisation an
 * allocation can cause. Scratch comes from a fixed device array built into
 * the library (about 10 MiB on every GPU that loads it, held until the
 * process exits), so at most dl_sort_unique_noalloc_max_rows() rows
 * (1,048,576) are accepted; more is DL_ERR_INVALID_ARGUMENT. `stream` is a
 * cudaStream_t (NULL = default stream). Every call synchronises `stream`:
 * it returns only after its own GPU work is done. The first call on a device
 * looks the array up and clears its control words (set-up), and should come
 * before any stream capture. All calls share the array and it keeps the last
 * call's contents: calls whose GPU work overlapped would race, so concurrent
 * host calls are serialised. */
DL_API dl_status dl_sort_unique_noalloc(dl_entity *rel, int64_t n, int64_t *n_out, void *stream);
DL_API int64_t dl_sort_unique_noalloc_max_rows(void);

/* ---- hash table and joins ---- */

/* Index a relation by key. load_factor <= 0 selects the default (0.5). The
 * table keeps its own copy; rel may be freed afterwards. */
DL_API dl_status dl_build_hash_table(dl_context *ctx, const dl_entity *rel, int64_t n, double load_factor,
                                     dl_hash_table **out);
DL_API dl_status dl_hash_table_info(const dl_hash_table *ht, int64_t *slots, int64_t *distinct_keys,
                                    int64_t *rows);
DL_API dl_status dl_hash_table_destroy(dl_hash_table *ht);
/* For every probe row (k, v) and every indexed row (k, w) emit (w, v).
 * *out is a new device buffer of *n_out rows (NULL when empty); release it
 * with dl_free. Rows are grouped by probe row, probe order kept. */
DL_API dl_status dl_join(dl_context *ctx, const dl_hash_table *ht, const dl_entity *probe, int64_t n,
                         dl_entity **out, int64_t *n_out);
/* Same result through binary search of a key-sorted relation. */
DL_API dl_status dl_join_sorted(dl_context *ctx, const dl_entity *sorted_rel, int64_t n_rel,
                                const dl_entity *probe, int64_t n, dl_entity **out, int64_t *n_out);

/* ---- programs ---- */

/* Run one program on an edge relation of `rows` int32 pairs (the binary
 * edge-file layout). `edges_on_device` = 1 if `edges` is device memory.
 * For DL_PROGRAM_SINGLE_JOIN the pairs are the relation R. */
DL_API dl_status dl_run_program(dl_context *ctx, int32_t program, const int32_t *edges, int64_t rows,
                                int32_t edges_on_device, const dl_options *opts, dl_run **out);
DL_API dl_status dl_run_tc(dl_context *ctx, const int32_t *edges, int64_t rows, int32_t edges_on_device,
                           const dl_options *opts, dl_run **out);
DL_API dl_status dl_run_sg(dl_context *ctx, const int32_t *edges, int64_t rows, int32_t edges_on_device,
                           const dl_options *opts, dl_run **out);
DL_API dl_status dl_run_wcc(dl_context *ctx, const int32_t *edges, int64_t rows, int32_t edges_on_device,
                            const dl_options *opts, dl_run **out);
DL_API dl_status dl_run_single_join(dl_context *ctx, const int32_t *rel, int64_t rows, int32_t rel_on_device,
                                    const dl_options *opts, dl_run **out);
DL_API dl_status dl_run_get_info(const dl_run *run, dl_run_info *info);
/* Output rows exactly as the reference writes its output file:
 * TC (x,z) ordered by (z,x); SG (x,y) ordered by (x,y); WCC (component,0)
 * ascending; single_join (a,c) ordered by (c,a). dst holds capacity_rows
 * int32 pairs, host memory unless dst_on_device = 1. */
DL_API dl_status dl_run_copy_output(const dl_run *run, int32_t *dst, int64_t capacity_rows,
                                    int32_t dst_on_device);
/* |delta| after each iteration (length = iterations). */
DL_API dl_status dl_run_copy_deltas(const dl_run *run, int64_t *dst, int64_t capacity);
/* Per iteration: join output rows (before dedup) and the size of the full
 * relation after the iteration (TC/SG; WCC: number of labelled nodes). */
DL_API dl_status dl_run_copy_iteration_stats(const dl_run *run, int64_t *join_rows, int64_t *full_rows,
                                             int64_t capacity);
/* WCC: every node id (ascending) and its final component label. */
DL_API dl_status dl_run_copy_labels(const dl_run *run, int32_t *node_ids, int32_t *labels, int64_t capacity);
DL_API dl_status dl_run_destroy(dl_run *run);

/* ---- sessions: many fixpoint instances at once (batched and served forms) ----
 *
 * No counterpart in the reference, whose drivers run one program on one
 * edge file per process (tc.cu:42-423, sg.cu:40-477, wcc.cu:58-585). A
 * session runs every admitted instance of one program (TC, SG or WCC) as one
 * union fixpoint: each iteration's joins, sorts, set difference and merge
 * process all active instances in the same launches. Instances can be
 * admitted between any two steps (continuous batching) and leave the union
 * at their own fixpoint. Each instance's outputs, iteration count and delta
 * sizes are those of dl_run_program on the same edges and options.
 * A session runs on its context's device and stream and takes the context's
 * cached buffers; dl_session_destroy hands all its memory back to the
 * context, so destroy every session before its context. Calls on one session
 * must not run concurrently. */
typedef struct dl_session dl_session;

/* max_nodes bounds the node count of the instances alive at once
 * (0 = 2^32 - 1); admitting past it fails with DL_ERR_OVERFLOW. */
DL_API dl_status dl_session_create(dl_context *ctx, int32_t program, const dl_options *opts, int64_t max_nodes,
                                   dl_session **out);
/* Adds an instance on `rows` int32 edge pairs; *instance receives its id
 * (ids count up from 0). Its first iteration runs in the next step. An
 * instance with no edges finishes at once. */
DL_API dl_status dl_session_admit(dl_session *s, const int32_t *edges, int64_t rows, int32_t edges_on_device,
                                  int64_t *instance);
/* Adds `count` instances at once (edges[i] holds rows[i] pairs); their ids
 * are consecutive, the first one in *first_instance. One admission of many
 * instances ranks and sorts them together. */
DL_API dl_status dl_session_admit_many(dl_session *s, const int32_t *const *edges, const int64_t *rows,
                                       int64_t count, int32_t edges_on_device, int64_t *first_instance);
/* One iteration of every active instance; *active = instances still running. */
DL_API dl_status dl_session_step(dl_session *s, int64_t *active);
/* Ids of the instances finished since the last poll, in finishing order;
 * at most `capacity` are returned and the rest stay queued. */
DL_API dl_status dl_session_poll(dl_session *s, int64_t *ids, int64_t capacity, int64_t *count);
DL_API dl_status dl_session_get_info(const dl_session *s, int64_t instance, dl_run_info *info);
/* Same layouts as dl_run_copy_output / dl_run_copy_deltas / dl_run_copy_labels. */
DL_API dl_status dl_session_copy_output(dl_session *s, int64_t instance, int32_t *dst, int64_t capacity_rows,
                                        int32_t dst_on_device);
DL_API dl_status dl_session_copy_deltas(const dl_session *s, int64_t instance, int64_t *dst, int64_t capacity);
DL_API dl_status dl_session_copy_labels(dl_session *s, int64_t instance, int32_t *node_ids, int32_t *labels,
                                        int64_t capacity);
/* Frees a finished instance's result memory (its info stays readable). */
DL_API dl_status dl_session_release(dl_session *s, int64_t instance);
/* Device bytes the session's live buffers and unreleased results hold (its
 * cache of free buffers not included) and the number of active instances. */
DL_API dl_status dl_session_memory(const dl_session *s, int64_t *device_bytes, int64_t *active);
DL_API dl_status dl_session_destroy(dl_session *s);
/* Batched form: admits `count` edge sets (edges[i] holds rows[i] pairs) and
 * steps until every instance has finished; results are read from *out. */
DL_API dl_status dl_run_batch(dl_context *ctx, int32_t program, const int32_t *const *edges, const int64_t *rows,
                              int64_t count, int32_t edges_on_device, const dl_options *opts, dl_session **out);

/* ---- live kernel profile (CUDA events on the context stream) ---- */

typedef struct dl_kernel_stat {
    char name[32];          /* kernel class, e.g. "sort_onesweep_pass" */
    int64_t launches;       /* launches since the last dl_profile_enable */
    int64_t timed_launches; /* launches bracketed by events (profiling on) */
    double seconds;         /* summed device time of the timed launches */
    double bytes;           /* summed algorithmic HBM bytes of the timed launches */
} dl_kernel_stat;

/* Reset the counters; enabled = 1 also times every launch with events. */
DL_API dl_status dl_profile_enable(dl_context *ctx, int32_t enabled);
/* Copy up to `capacity` kernel classes; *count = number of classes. */
DL_API dl_status dl_profile_read(dl_context *ctx, dl_kernel_stat *out, int32_t capacity, int32_t *count);

/* The reference's synthetic single-join rows: C library srand(seed) then
 * rand() % rand_range + 1 for 2*rows values (glibc generator). */
DL_API dl_status dl_generate_rows(int64_t rows, int32_t rand_range, uint32_t seed, int32_t *host_out);

#ifdef __cplusplus
}
#endif
#endif
