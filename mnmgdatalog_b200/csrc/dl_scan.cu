// Compaction operators: unique (thrust::unique(is_equal) / unique(is_equal_key))
// and remove_if(is_key_equal_value), as single-pass select kernels.
#include "dl_internal.h"
#include "dl_scan.cuh"

namespace dl {
namespace {

// Keep the first word of every run of words equal under `mask`.
struct KeepRunHead {
    u64 mask;
    __device__ bool operator()(u64 cur, u64 prev, bool has_prev) const {
        return !has_prev || ((cur ^ prev) & mask) != 0;
    }
};

// Keep words other than the all-ones "removed" marker.
struct KeepMarked {
    __device__ bool operator()(u64 cur, u64, bool) const { return cur != ~0ull; }
};

// Keep Entity words whose key differs from their value.
struct KeepNotSelfEntity {
    __device__ bool operator()(u64 cur, u64, bool) const { return (u32) cur != (u32) (cur >> 32); }
};

template <class Keep>
u64 run_select(Context &ctx, const u64 *in, u64 n, u64 *out, Keep keep) {
    if (n == 0) return 0;
    const u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    u64 *lb = ctx.lookback_words(tiles);
    u32 *ctr = ctx.tile_counter(32);
    u64 *cnt = &ctx.ctrl->scalar[0];
    DL_CUDA(cudaMemsetAsync(ctr, 0, sizeof(u32), ctx.stream));
    DL_LAUNCH(ctx, K_SELECT, 8.0 * n, select_kernel<Keep><<<(unsigned) tiles, SCAN_THREADS, 0, ctx.stream>>>(in, n, out, keep, lb, ctr,
                                                                          ctx.next_epoch(), &ctx.ctrl->err, cnt));
    DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, cnt, sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    ctx.prof_add_bytes(K_SELECT, 8.0 * ctx.host_scalars[0]);
    return ctx.host_scalars[0];
}

}  // namespace

u64 unique_words(Context &ctx, const u64 *in, u64 n, u64 *out, int by_key_shift, Codec codec) {
    u64 mask = ~0ull;
    if (by_key_shift < 64) {
        // Raw Entity words keep the key in the low half; compact/encoded
        // words keep it above `by_key_shift`.
        mask = (codec == Codec::Entity) ? 0xFFFFFFFFull : (~0ull << by_key_shift);
    }
    return run_select(ctx, in, n, out, KeepRunHead{mask});
}

u64 select_words(Context &ctx, const u64 *in, u64 n, u64 *out, int) {
    return run_select(ctx, in, n, out, KeepMarked{});
}

u64 remove_self_pairs_words(Context &ctx, const u64 *in, u64 n, u64 *out) {
    return run_select(ctx, in, n, out, KeepNotSelfEntity{});
}

}  // namespace dl
