// Program runs (dl_run) of the engine; see dl_engine.cu.
#pragma once

#include "dl_internal.h"

namespace dl {

struct Run {
    Context *ctx = nullptr;
    dl_program program = DL_PROGRAM_TC;
    dl_run_info info{};
    std::vector<i64> deltas;  // |delta| after each iteration
    std::vector<i64> joins;   // join output rows of each iteration
    std::vector<i64> fulls;   // |full| after each iteration
    DevBuf words;             // TC/SG/single_join: sorted result words
    u64 n_words = 0;
    DevBuf ids;               // node id of each rank
    u32 n_ids = 0;
    bool ids_affine = false;  // ids[r] == id_base + r
    int32_t id_base = 0;
    int bits = 1;             // bits per rank in a word
    DevBuf aux;               // WCC: component ranks, ascending
    u64 n_aux = 0;
    DevBuf labels;            // WCC: label rank of every node
    // TC / SG on the bit matrix: the result stays as a matrix with each
    // row's (or target's) first output position; rows are extracted when
    // they are copied out. bm_t is TC's transpose (row = target), SG's
    // matrix, or (bm_cols) TC's matrix itself with per (512-row block,
    // target) offsets in bm_off.
    bool from_bitmat = false;
    bool bm_row_first = false;  // SG: rows (row id, column id) from the matrix rows
    bool bm_cols = false;       // TC: rows from the matrix's columns
    DevBuf bm_t, bm_first, bm_off;
    DevBuf bm_live;             // TC column form: the matrix rows that were written (one bit per row)
    u64 bm_n = 0, bm_stride = 0, bm_words = 0;
};

Run *run_program(Context &ctx, int program, const int32_t *rows, u64 n, bool on_device, const dl_options &opt);
void run_copy_output(const Run &r, int32_t *dst, u64 capacity, bool dst_on_device);
void run_copy_labels(const Run &r, int32_t *node_ids, int32_t *labels, u64 capacity);
void run_destroy(Run *r);
u64 bitmat_units(const Run &r);
u64 bitmat_unit_index(const Run &r, u64 unit);
void bitmat_extract_rows(Context &ctx, const Run &r, int32_t *out, u64 u0, u64 u1);

}  // namespace dl
