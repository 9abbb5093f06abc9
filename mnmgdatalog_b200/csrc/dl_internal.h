// Host-side internals shared by the engine's translation units (not part of
// the C-ABI; see include/mnmgdl.h for that).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mnmgdl.h"
#include "dl_device.cuh"

namespace dl {

// Sets the calling thread's dl_last_error() text.
void set_last_error(const std::string &msg);

// Error raised inside the engine; the C-ABI layer converts it to a dl_status.
struct Error : std::runtime_error {
    dl_status status;
    Error(dl_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

#define DL_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            throw ::dl::Error(e_ == cudaErrorMemoryAllocation ? DL_ERR_OUT_OF_MEMORY : DL_ERR_CUDA, \
                              std::string(#call) + ": " + cudaGetErrorString(e_));             \
        }                                                                                      \
    } while (0)

#define DL_CHECK_LAUNCH() DL_CUDA(cudaGetLastError())

// Brackets one kernel launch for the live profile:
//   DL_LAUNCH(ctx, K_SORT_PASS, 16.0 * n, kernel<<<g, b, s, ctx.stream>>>(...));
#define DL_LAUNCH(ctx, kid, bytes, ...)   \
    do {                                  \
        (ctx).prof_begin();               \
        __VA_ARGS__;                      \
        DL_CHECK_LAUNCH();                \
        (ctx).prof_end((kid), (bytes));   \
    } while (0)

// Grow-only device buffer; no allocation happens inside a fixpoint iteration
// once the capacities have reached their high-water mark.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    bool fixed = false;  // a slice of memory the buffer does not own: never grown or freed
    void reserve(size_t bytes, bool zero = false);
    void release();
    template <typename T>
    T *as() const { return static_cast<T *>(p); }
};

// Kernel classes for the live profile (launch counts, device time from CUDA
// events on the context stream, algorithmic HBM bytes).
enum KernelId : int {
    K_PREP = 0,        // init / finalize transforms (pack, rank, CSR, unpack)
    K_SORT_HIST,       // radix histogram (upsweep): 8 B per key
    K_SORT_BUCKET,     // radix spine scan of the (digit, CTA) counts
    K_SORT_PASS,       // radix scatter pass (downsweep or onesweep): 16 B per key
    K_SELECT,          // unique / remove_if compaction: 8 B read + 8 B per kept word
    K_JOIN_COUNT,      // join count + scan: 8 B probe read + 8 B offset write per probe row
    K_JOIN_PARTITION,  // merge-path partition of the emit
    K_JOIN_EMIT,       // join emit: 8 B per probe row + 16 B per output word
    K_WCC_PROPAGATE,   // WCC min-label propagation: 8 B per delta row + 4 B per edge + 32 B per atomicMin
    K_MERGE_PARTITION, // merge-path partition of set operations
    K_DIFF_MERGE,      // fused unique/set-difference/merge: 8 B x (|full| + |J| + |full'| + |delta|)
    K_MERGE,           // plain merge: 16 B per word
    K_HASH_BUILD,      // C-ABI hash table insert / value extraction
    K_SPARSE_DIFF,     // sparse set difference probes (+ run sampling)
    K_HASH_INSERT,     // hash-set dedup: 8 B read + 32 B probe sector per word, 40 B per new word
    K_BITMAP_EXPAND,   // bit-matrix TC step: 4 B per delta row in and out + 16 B per unit in and out +
                       // 4 B edge target per join word
    K_BITMAP_COLUMNS,  // TC result set-up from the bit matrix: its transpose with per-target counts
                       // (2 x matrix), or per (row block, target) counts and their offsets
    K_BITMAP_EXTRACT,  // result rows from the bit matrix: matrix (+ TC offsets) read + 8 B per result row (+ count scan)
    // host-side costs, counted with or without profiling (seconds = host wall time)
    K_HOST_MALLOC,     // cudaMalloc of a buffer that had to grow (bytes = size)
    K_HOST_FREE,       // cudaFree of a cached buffer dropped from the cache
    K_HOST_SYNC,       // host waits for the stream (cudaStreamSynchronize)
    K_COUNT
};
const char *kernel_name(int kid);

struct KernelStat {
    u64 launches = 0;
    u64 timed = 0;
    double seconds = 0;
    double bytes = 0;
};

// Engine scratch reused across runs of one context (capacities only grow).
struct Workspace {
    DevBuf input;          // device copy of host edge rows
    DevBuf ids;            // sorted distinct node ids (int32)
    DevBuf w0, w1;         // word buffers for the initial sorts
    DevBuf csr_off, csr_val;
    DevBuf full[2];        // full relation (large run), ping-pong
    DevBuf small[2];       // full relation (small run), ping-pong
    DevBuf tiny[2];        // full relation (tiny run, plain runs only), ping-pong
    DevBuf sample;         // sample of the large run for sparse probes
    DevBuf sample_small;   // sample of the small run for sparse probes
    DevBuf jbuf[2];        // join output / sort ping-pong / delta
    DevBuf offsets;        // join count offsets
    DevBuf offsets_next;   // bit-matrix TC: the next delta's join offsets
    DevBuf wcc_label, wcc_flag, wcc_next;
    DevBuf bitmat[2];      // full relation as a bit matrix; TC's column offsets of the result rows
    DevBuf bit_hasout;     // bit-matrix TC: nodes with out-edges (one bit each)
};

// Engine knobs the autotuner sets per context (mnmgdatalog_b200/autotune.py);
// the defaults are the measured best on B200. DL_SORT_ALGO, DL_SORT_RANK,
// DL_SORT_KPT, DL_SORT_TMA and DL_JOIN_FIRST_PASS override the defaults.
struct Tuning {
    int sort_algo = 1;          // 1 = three-kernel LSD pass, 0 = onesweep
    int rank = 1;               // 1 = shared-memory peer masks, 0 = warp ballots
    int sort_kpt = 16;          // onesweep keys per thread: 12 or 16
    int sort_tma = 1;           // three-kernel pass input: 1 = TMA double buffer, 0 = direct loads
    int join_first_pass = 1;    // 1 = TC join emit does the first radix pass (bits 0-7), 0 = separate pass
    u64 dense_ratio = 4;        // fused full rewrite when |J| * dense_ratio >= |large run|
    u64 small_ratio = 4;        // small run folded when |small| * small_ratio >= |large run|
    double hash_load = 0.5;     // default load factor of dl_build_hash_table
    int bitmap_max_gib = 48;    // TC dedup AUTO: bit matrix (+ its column offsets) at most this many GiB (0 = never)
    u32 bitmap_unit_rows = 65536;  // bit-matrix TC: delta rows per unit (one shared-memory row fold each)
    int cache_max_gib = 96;        // cached spare buffers of the context, at most this many GiB
    int bitmap_result = 0;         // bit-matrix TC result: 0 transpose when it fits, else columns; 1 transpose; 2 columns
};
Tuning default_tuning();

struct Context {
    int device = 0;
    Tuning tune = default_tuning();
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t copy_stream = nullptr;  // result copies to the host beside `stream` (created on first use)
    int sm_count = 148;
    bool no_alloc = false;          // every buffer is a fixed slice; a new allocation is an internal error
    Ctrl *ctrl = nullptr;           // device control block
    u32 epoch = 0;                  // look-back epoch of the last launch
    DevBuf lookback;                // look-back words (zeroed at allocation)
    DevBuf sort_hist;               // radix histograms / bucket bases
    DevBuf lbs_splits;              // join emit partition points
    DevBuf radix_part;              // per-(digit, CTA) counts and offsets of a radix pass
    DevBuf merge_splits;            // merge-path split points of a set operation
    DevBuf bucket_cursor;           // per-digit output cursors of the bucketed join emit
    DevBuf part_cursor;             // per-destination counts and cursors of a hash partition
    u64 *host_scalars = nullptr;    // pinned mirror for small D2H reads
    Workspace ws;
    u64 run_join_total = 0, run_join_max = 0;  // join statistics of the current run
    std::vector<DevBuf> spares;     // buffers handed back by destroyed runs and sessions
    // Freeing a multi-GB buffer costs milliseconds and synchronises the
    // device, so outgrown buffers stay cached; an allocation that fails
    // drops the whole cache and retries (Context::allocate).
    static constexpr size_t kSpareCount = 256;  // and at most tune.cache_max_gib GiB

    // Live profile: every launch is counted; with prof_on each launch is
    // bracketed by events that are resolved at the next sync().
    bool prof_on = false;
    KernelStat kstat[K_COUNT];
    struct Pending {
        int kid;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> ev_pool;
    cudaEvent_t prof_open = nullptr;
    void prof_begin();
    void prof_end(int kid, double bytes);
    void prof_add_bytes(int kid, double bytes);
    void prof_resolve();
    void prof_reset();

    // Ensure buf holds `bytes`, preferring a spare buffer over cudaMalloc.
    void reserve(DevBuf &buf, size_t bytes, bool zero = false);
    void give_back(DevBuf &buf);
    void trim_spares();
    // Fresh allocation of `bytes` into an empty buf; on failure frees every
    // cached buffer and tries once more (with `minimum` bytes if given).
    void allocate(DevBuf &buf, size_t bytes, bool zero = false, size_t minimum = 0);
    void release_all();
    cudaStream_t copy_stream_get();

    // Next look-back epoch; clears the look-back buffer when the 14-bit epoch
    // wraps so that no stale word can alias the current launch.
    u32 next_epoch();
    // Look-back buffer with room for `words` words.
    u64 *lookback_words(size_t words);
    // Tile counter `slot` (reset to zero on the stream before use).
    u32 *tile_counter(int slot);
    void check_device_error();
    void sync();
};

// ---- radix sort (dl_radix.cu) ----------------------------------------------
enum class Codec { Raw = 0, Entity = 1 };
// Sorts n keys from `a` (using `b` as the ping-pong buffer) in ascending
// order. If `known_bits` > 0 only digits covering bits [0, known_bits) are
// sorted (keys must be zero above that); otherwise a histogram pass finds the
// digits that vary (one host read). Returns the buffer holding the result.
u64 *radix_sort(Context &ctx, u64 *a, u64 *b, u64 n, Codec codec, int known_bits,
                u64 *hist_accumulated = nullptr);
// Sorts by the 8-bit windows at the given ascending bit shifts (raw words).
// Correct when every bit outside the windows is the same in all keys;
// windows may overlap.
u64 *radix_sort_windows(Context &ctx, u64 *a, u64 *b, u64 n, const int *shifts, int nwin);
// Fewest 8-bit windows covering the bits that vary in words
// (hi << field_bits | lo) whose fields are below 2^used_bits; fills shifts
// (at most 8) and returns their number.
int plan_windows(int field_bits, int used_bits, int *shifts);
// Histogram of the digits [0, ndigits) accumulated by producers (join emit)
// into ctx.sort_hist; lets radix_sort skip its own histogram pass.
u64 *radix_hist_buffer(Context &ctx);
void radix_hist_clear(Context &ctx);
// True when radix_sort benefits from a producer-accumulated histogram
// (the onesweep variant); the three-kernel variant counts per chunk itself.
bool radix_wants_histogram(const Context &ctx);

// ---- compaction / scan (dl_scan.cu) ------------------------------------------
// out[i] = in[i] for the first of each run of equal words; returns count.
// `out` may alias `in`. With `by_key_shift` < 64, words compare on bits
// >= by_key_shift only (unique by key, keeps the first = smallest value).
u64 unique_words(Context &ctx, const u64 *in, u64 n, u64 *out, int by_key_shift = 64,
                 Codec codec = Codec::Raw);
// Drops entity words whose key equals value. `out` may alias `in`.
u64 remove_self_pairs_words(Context &ctx, const u64 *in, u64 n, u64 *out);

// ---- hash partition for the multi-GPU exchange (dl_partition.cu) ------------
constexpr u32 kMaxPartitionRanks = 4096;
// out = rel's rows grouped by owner(key) = fmix32(key) % ranks, destination
// 0 first (order inside a group unspecified); counts[r] = rows owned by r.
// swap: rows leave as (value, key) and are owned by their value.
void partition_rows(Context &ctx, const int32_t *rel, u64 n, u32 ranks, bool swap, int32_t *out, i64 *counts);
// Drops all-ones words (the engine's "removed" marker). `out` may alias `in`.
// `kind` is unused (reserved).
u64 select_words(Context &ctx, const u64 *in, u64 n, u64 *out, int kind);

// ---- merge path (dl_setops.cu) -------------------------------------------------
// Stable merge (ties take `a` first), keeps duplicates: thrust::merge.
void merge_words(Context &ctx, const u64 *a, u64 na, const u64 *b, u64 nb, u64 *out, Codec codec);
// full_out = unique(merge(full, j)); delta_out = (j \ full) deduplicated.
// `j` sorted (duplicates allowed), `full` sorted unique. Either output may be
// null. Returns |delta|. full_out receives |full| + |delta| words.
u64 diff_merge_words(Context &ctx, const u64 *full, u64 nfull, const u64 *j, u64 nj,
                     u64 *full_out, u64 *delta_out, Codec codec);
// Sample of a sorted run for sparse_diff_words (every 4096th word).
void run_sample(Context &ctx, const u64 *run, u64 n, DevBuf &sample, u64 &ns);
// out = dedup(j) \ run for sorted j (duplicates allowed) and a sorted
// duplicate-free run of compact words, by binary probes: O(|j| log) instead
// of O(|run|). out may alias nothing in j/run; returns |out|.
u64 sparse_diff_words(Context &ctx, const u64 *run, u64 nrun, const u64 *sample, u64 ns, const u64 *j, u64 nj,
                      u64 *out);

// ---- hash set of tuple words (dl_hashset.cu) ---------------------------------
// Open addressing over 64-bit words (empty slot = all ones), linear probing,
// capacity a power of two, never more than 3/4 full.
struct WordSet {
    int cur = 0;      // which of the two buffers holds the table
    u64 cap = 0;      // slots (power of two)
    u64 size = 0;     // words stored
};
// Makes room for `incoming` more words (rehash into the other buffer when
// size + incoming would exceed 3/4 of the capacity).
void wordset_reserve(Context &ctx, WordSet &ws, DevBuf buf[2], u64 incoming);
// Inserts n words; the ones not present before go to `fresh` (if not null),
// in no particular order. Returns how many were new.
u64 wordset_insert(Context &ctx, WordSet &ws, DevBuf buf[2], const u64 *in, u64 n, u64 *fresh);
// Copies the stored words (unsorted) to out (size words); returns size.
u64 wordset_extract(Context &ctx, const WordSet &ws, DevBuf buf[2], u64 *out);

// ---- joins (dl_join.cu) --------------------------------------------------------
struct Csr {            // relation grouped by dense key index
    u32 *off = nullptr; // n_keys + 1 offsets into val
    u32 *val = nullptr; // value indices
    u32 n_keys = 0;
    u64 n_vals = 0;
};
enum class EmitKind : int {
    ZV = 0,        // (z, v): TC, WCC-style
    VZ = 1,        // (v, z): join + column swap fused (SG rules)
    ZV_NOSELF = 2, // (z, v) with z == v replaced by an all-ones word (SG base)
};
// Join probe words (k << bits | v) against the CSR: every match (k, z)
// emits one word per EmitKind. Returns the number of words written to
// `out` (which must hold the count returned by join_count). `offsets` holds
// n_probe u64 exclusive offsets computed by join_count.
u64 join_count(Context &ctx, const Csr &csr, const u64 *probe, u64 n_probe, int bits, u64 *offsets);
void join_emit(Context &ctx, const Csr &csr, const u64 *probe, u64 n_probe, int bits, const u64 *offsets,
               u64 total, EmitKind kind, u64 *out, u64 *hist, int hist_digits, u64 *self_pairs);

}  // namespace dl
