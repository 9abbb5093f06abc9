// Single-pass device-wide scan and stream compaction (decoupled look-back).
// Templates shared by the compaction operators (unique, remove_if) and the
// join's count pass.
#pragma once

#include "dl_device.cuh"

namespace dl {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_IPT = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_IPT;

// Stream compaction of 64-bit words: keeps in[i] when keep(in[i], in[i-1],
// i > 0) holds.
// Output order = input order. `out` may alias `in` (every tile has read its
// input before it publishes, and a tile's output range ends at or before
// its own input range). The last tile stores the kept count to *count.
template <class Keep>
__global__ void __launch_bounds__(SCAN_THREADS)
select_kernel(const u64 *in, u64 n, u64 *out, Keep keep, u64 *lb, u32 *tile_ctr, u32 epoch, u32 *err,
              u64 *count) {
    __shared__ u64 s_items[SCAN_TILE];
    __shared__ u32 s_scratch[SCAN_THREADS / 32 + 1];
    __shared__ u32 s_tile;
    __shared__ u64 s_excl;
    __shared__ LookbackScratch s_lbs;
    const int tid = threadIdx.x;
    if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const u32 tile = s_tile;
    const u64 base = (u64) tile * SCAN_TILE;
    const u32 nv = (u32) min((u64) SCAN_TILE, n - base);

    // Striped coalesced load, then each thread owns SCAN_IPT consecutive items.
#pragma unroll
    for (int j = 0; j < SCAN_IPT; ++j) {
        const u32 li = j * SCAN_THREADS + tid;
        if (li < nv) s_items[li] = in[base + li];
    }
    __syncthreads();
    u32 flags = 0;
#pragma unroll
    for (int j = 0; j < SCAN_IPT; ++j) {
        const u32 li = tid * SCAN_IPT + j;
        if (li < nv) {
            const u64 cur = s_items[li];
            const bool has_prev = (base + li) > 0;
            const u64 prev = has_prev ? (li > 0 ? s_items[li - 1] : in[base - 1]) : 0ull;
            if (keep(cur, prev, has_prev)) flags |= 1u << j;
        }
    }
    u32 tot;
    const u32 off = block_exclusive_sum<SCAN_THREADS / 32>((u32) __popc(flags), s_scratch, &tot);
    {
        u64 excl = 0;
        if (tile == 0) {
            if (tid == 0) st_relaxed_u64(lb, lb_word(kStatusInc, epoch, tot));
        } else {
            if (tid == 0) st_relaxed_u64(lb + tile, lb_word(kStatusAgg, epoch, tot));
            excl = lookback_block<SCAN_THREADS / 32>(lb, tile, epoch, err, s_lbs);
            if (tid == 0) st_relaxed_u64(lb + tile, lb_word(kStatusInc, epoch, excl + tot));
        }
        if (tid == 0) s_excl = excl;
    }
    // Compact into shared memory (positions < own, so in-place is safe after
    // every thread has read its items).
    u64 mine[SCAN_IPT];
#pragma unroll
    for (int j = 0; j < SCAN_IPT; ++j) mine[j] = s_items[tid * SCAN_IPT + j];
    __syncthreads();
    u32 o = off;
#pragma unroll
    for (int j = 0; j < SCAN_IPT; ++j)
        if ((flags >> j) & 1u) s_items[o++] = mine[j];
    __syncthreads();
    const u64 excl = s_excl;
    for (u32 j = tid; j < tot; j += SCAN_THREADS) out[excl + j] = s_items[j];
    if (base + nv == n && tid == 0) *count = excl + tot;
}

// Exclusive scan of value(i) for i < n (64-bit): out[i] = sum_{j<i} value(j).
// The last tile stores the grand total to *total.
template <class Value>
__global__ void __launch_bounds__(SCAN_THREADS)
scan_kernel(Value value, u64 n, u64 *out, u64 *lb, u32 *tile_ctr, u32 epoch, u32 *err, u64 *total) {
    __shared__ u64 s_scratch[SCAN_THREADS / 32 + 1];
    __shared__ u64 s_items[SCAN_TILE];
    __shared__ u32 s_tile;
    __shared__ u64 s_excl;
    __shared__ LookbackScratch s_lbs;
    const int tid = threadIdx.x;
    if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const u32 tile = s_tile;
    const u64 base = (u64) tile * SCAN_TILE;
    const u32 nv = (u32) min((u64) SCAN_TILE, n - base);
#pragma unroll
    for (int j = 0; j < SCAN_IPT; ++j) {
        const u32 li = j * SCAN_THREADS + tid;
        s_items[li] = (li < nv) ? value(base + li) : 0ull;
    }
    __syncthreads();
    u64 x[SCAN_IPT];
    u64 sum = 0;
#pragma unroll
    for (int j = 0; j < SCAN_IPT; ++j) {
        x[j] = s_items[tid * SCAN_IPT + j];
        sum += x[j];
    }
    u64 tot;
    u64 off = block_exclusive_sum<SCAN_THREADS / 32>(sum, s_scratch, &tot);
    {
        u64 excl = 0;
        if (tile == 0) {
            if (tid == 0) st_relaxed_u64(lb, lb_word(kStatusInc, epoch, tot));
        } else {
            if (tid == 0) st_relaxed_u64(lb + tile, lb_word(kStatusAgg, epoch, tot));
            excl = lookback_block<SCAN_THREADS / 32>(lb, tile, epoch, err, s_lbs);
            if (tid == 0) st_relaxed_u64(lb + tile, lb_word(kStatusInc, epoch, excl + tot));
        }
        if (tid == 0) s_excl = excl;
    }
    __syncthreads();
    off += s_excl;
#pragma unroll
    for (int j = 0; j < SCAN_IPT; ++j) {
        s_items[tid * SCAN_IPT + j] = off;
        off += x[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < SCAN_IPT; ++j) {
        const u32 li = j * SCAN_THREADS + tid;
        if (li < nv) out[base + li] = s_items[li];
    }
    if (base + nv == n && tid == 0) *total = s_excl + tot;
}

}  // namespace dl
