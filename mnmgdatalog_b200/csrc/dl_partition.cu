// Hash partition of a relation by the owner of its key: the send-buffer
// preparation of the multi-GPU exchange. The reference computes, per row,
// get_rank(key) = murmur3 fmix32(key) % ranks, counts rows per destination
// and scatters them into per-destination runs (common/kernels.cu:199-242,
// get_send_count / get_rank_data). Here the mixer runs on the key's unsigned
// 32-bit pattern and the modulo is unsigned, so every owner is in
// [0, ranks); the row order inside a destination's run is unspecified (the
// receiver sorts). With swap_columns each row (a, b) leaves as (b, a) and is
// owned by b -- the reference's reverse_entity_ar before an exchange.
#include "dl_engine_detail.h"

namespace dl {
namespace {

constexpr int PT_THREADS = 256;
constexpr int PT_ROWS = 8;  // rows per thread per scatter tile

__device__ __forceinline__ u32 key_owner(int32_t key, u32 ranks) {
    u32 h = (u32) key;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h % ranks;
}

__device__ __forceinline__ int2 oriented(int2 r, bool swap) { return swap ? make_int2(r.y, r.x) : r; }

// counts[o] += rows owned by o (per-CTA shared histogram, one global atomic
// per CTA and non-empty owner).
__global__ void __launch_bounds__(PT_THREADS) partition_count_kernel(const int2 *__restrict__ rel, u64 n, u32 ranks,
                                                                     int swap,
                                                                     unsigned long long *__restrict__ counts) {
    extern __shared__ u32 hist[];
    for (u32 i = threadIdx.x; i < ranks; i += PT_THREADS) hist[i] = 0;
    __syncthreads();
    for (u64 i = (u64) blockIdx.x * PT_THREADS + threadIdx.x; i < n; i += (u64) gridDim.x * PT_THREADS)
        atomicAdd(&hist[key_owner(oriented(rel[i], swap).x, ranks)], 1u);
    __syncthreads();
    for (u32 i = threadIdx.x; i < ranks; i += PT_THREADS)
        if (hist[i]) atomicAdd(counts + i, (unsigned long long) hist[i]);
}

// Rows of a tile of PT_THREADS * PT_ROWS rows: ranked per owner in shared
// memory, one global cursor atomic per (tile, owner), then scattered.
__global__ void __launch_bounds__(PT_THREADS) partition_scatter_kernel(const int2 *__restrict__ rel, u64 n,
                                                                       u32 ranks, int swap,
                                                                       unsigned long long *__restrict__ cursor,
                                                                       int2 *__restrict__ out) {
    extern __shared__ unsigned long long sh[];
    unsigned long long *base = sh;                    // [ranks]
    u32 *hist = reinterpret_cast<u32 *>(sh + ranks);  // [ranks]
    const u64 tile_rows = (u64) PT_THREADS * PT_ROWS;
    for (u64 t0 = (u64) blockIdx.x * tile_rows; t0 < n; t0 += (u64) gridDim.x * tile_rows) {
        for (u32 i = threadIdx.x; i < ranks; i += PT_THREADS) hist[i] = 0;
        __syncthreads();
        int2 row[PT_ROWS];
        u32 own[PT_ROWS], loc[PT_ROWS];
#pragma unroll
        for (int j = 0; j < PT_ROWS; ++j) {
            const u64 i = t0 + (u64) j * PT_THREADS + threadIdx.x;
            own[j] = ranks;
            if (i < n) {
                row[j] = oriented(rel[i], swap);
                own[j] = key_owner(row[j].x, ranks);
                loc[j] = atomicAdd(&hist[own[j]], 1u);
            }
        }
        __syncthreads();
        for (u32 i = threadIdx.x; i < ranks; i += PT_THREADS)
            base[i] = hist[i] ? atomicAdd(cursor + i, (unsigned long long) hist[i]) : 0ull;
        __syncthreads();
#pragma unroll
        for (int j = 0; j < PT_ROWS; ++j)
            if (own[j] < ranks) out[base[own[j]] + loc[j]] = row[j];
        __syncthreads();
    }
}

}  // namespace

void partition_rows(Context &ctx, const int32_t *rel, u64 n, u32 ranks, bool swap, int32_t *out, i64 *counts) {
    if (ranks == 0 || ranks > kMaxPartitionRanks) throw Error(DL_ERR_INVALID_ARGUMENT, "ranks must be in [1, 4096]");
    for (u32 r = 0; r < ranks; ++r) counts[r] = 0;
    if (n == 0) return;
    ctx.reserve(ctx.part_cursor, 2 * (size_t) ranks * 8);
    unsigned long long *cnt = ctx.part_cursor.as<unsigned long long>();
    unsigned long long *cur = cnt + ranks;
    DL_CUDA(cudaMemsetAsync(cnt, 0, ranks * 8, ctx.stream));
    const int2 *in = reinterpret_cast<const int2 *>(rel);
    DL_LAUNCH(ctx, K_PREP, 8.0 * n,
              partition_count_kernel<<<detail::grid_for(n, PT_THREADS, ctx, 4), PT_THREADS, ranks * 4, ctx.stream>>>(
                  in, n, ranks, swap ? 1 : 0, cnt));
    std::vector<unsigned long long> h(ranks), off(ranks);
    DL_CUDA(cudaMemcpyAsync(h.data(), cnt, ranks * 8, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    unsigned long long s = 0;
    for (u32 r = 0; r < ranks; ++r) {
        off[r] = s;
        s += h[r];
        counts[r] = (i64) h[r];
    }
    DL_CUDA(cudaMemcpyAsync(cur, off.data(), ranks * 8, cudaMemcpyHostToDevice, ctx.stream));
    const u64 tiles = (n + (u64) PT_THREADS * PT_ROWS - 1) / ((u64) PT_THREADS * PT_ROWS);
    DL_LAUNCH(ctx, K_PREP, 16.0 * n,
              partition_scatter_kernel<<<(unsigned) std::min<u64>(tiles, (u64) ctx.sm_count * 8), PT_THREADS,
                                         ranks * 12, ctx.stream>>>(in, n, ranks, swap ? 1 : 0, cur,
                                                                  reinterpret_cast<int2 *>(out)));
    ctx.sync();  // the host copy of the offsets must outlive its transfer
}

}  // namespace dl
