// Multi-instance fixpoint session (batched and served forms); see dl_session.cu.
#pragma once

#include <memory>

#include "dl_internal.h"

namespace dl {

struct SessionInstance {
    i64 id = 0;
    i64 input_rows = 0;
    u64 rank_lo = 0, rank_hi = 0;  // union ranks [rank_lo, rank_hi) of this instance
    std::shared_ptr<DevBuf> ids_block;  // node ids of the admission this instance came with
    u64 ids_off = 0;                    // first local rank's entry in ids_block
    u32 n_ids = 0;
    const int32_t *ids() const { return ids_block ? ids_block->as<int32_t>() + ids_off : nullptr; }
    std::vector<i64> deltas;       // |delta| of this instance after each iteration
    i64 prev_delta = 0;            // WCC reference stop rule
    bool active = false, done = false, released = false;
    // TC/SG: sorted union words; WCC: component ranks (local). Instances that
    // finish in the same step share one block.
    std::shared_ptr<DevBuf> result_block;
    u64 result_off = 0;
    u64 n_result = 0;
    std::shared_ptr<DevBuf> labels_block;  // WCC: union label rank of every local node
    u64 labels_off = 0;
    i64 largest = 0;               // WCC: largest component size
    const u64 *result_words() const { return result_block->as<u64>() + result_off; }
    const u32 *result_u32() const { return result_block->as<u32>() + result_off; }
    const u32 *labels() const { return labels_block->as<u32>() + labels_off; }
};

struct SessionImpl;

// program: DL_PROGRAM_TC, _SG or _WCC. max_nodes bounds the total node count
// of the instances alive at once (0: 2^30 for TC/SG, 2^32 - 1 for WCC).
SessionImpl *session_create(Context &parent, int program, const dl_options &opt, u64 max_nodes);
void session_destroy(SessionImpl *s);
// Adds an instance; its first iteration runs with the next session_step.
i64 session_admit(SessionImpl &s, const int32_t *rows, u64 n, bool on_device);
// Adds `count` instances at once (one ranking sort and one edge sort for
// all of them); returns their ids in order.
std::vector<i64> session_admit_many(SessionImpl &s, const int32_t *const *rows, const u64 *n, u64 count,
                                    bool on_device);
// One semi-naive iteration of every active instance; returns how many remain active.
u64 session_step(SessionImpl &s);
// Moves up to `capacity` ids of the instances finished since the last poll
// (in finishing order) to `ids`; returns how many were moved.
u64 session_poll(SessionImpl &s, int64_t *ids, u64 capacity);
// Adds the session's kernel counters to the parent context's live profile
// and follows the parent's profiling switch from here on.
void session_fold_profile(SessionImpl &s, Context &parent);
const SessionInstance &session_instance(const SessionImpl &s, i64 id);
void session_info(const SessionImpl &s, i64 id, dl_run_info &info);
void session_copy_output(SessionImpl &s, i64 id, int32_t *dst, u64 capacity, bool on_device);
void session_copy_labels(SessionImpl &s, i64 id, int32_t *node_ids, int32_t *labels, u64 capacity);
void session_release(SessionImpl &s, i64 id);
u64 session_device_bytes(const SessionImpl &s);
u64 session_active(const SessionImpl &s);
u64 session_instance_count(const SessionImpl &s);

}  // namespace dl
