// Merge-path set operations on sorted 64-bit tuple words.
//
// * diff_merge: one kernel for the semi-naive step that the reference runs
//   as thrust::unique + thrust::set_difference + thrust::merge (tc.cu:250-279,
//   sg.cu:330-368). Over the merged order of full (sorted, unique) and J
//   (sorted, duplicates allowed) a J word is new iff it differs from the
//   word before it; full' = unique(merge) and delta = the new J words. Since
//   full is duplicate-free, the position of a word in full' is (full words
//   before it) + (new words before it), so one decoupled look-back counter
//   (the number of new words) places both outputs.
//   HBM traffic: 8 B x (|full| + |J|) read, 8 B x (|full'| + |delta|) written.
// * merge: thrust::merge(set_cmp) (wcc.cu:308-312), stable, duplicates kept.
//
// Each CTA takes 4096 consecutive positions of the merged order; its start in
// both inputs comes from a partition kernel (one merge-path binary search per
// tile boundary). Inputs are staged in shared memory, every thread merges 16
// words serially, outputs leave through shared memory in coalesced runs.
#include "dl_internal.h"

namespace dl {
namespace {

constexpr int MP_THREADS = 256;
constexpr int MP_VT = 16;
constexpr int MP_TILE = MP_THREADS * MP_VT;

template <bool ENC>
__device__ __forceinline__ u64 ld_enc(const u64 *p) {
    const u64 x = *p;
    return ENC ? entity_encode(x) : x;
}

// Number of `a` words among the first `diag` words of merge(a, b), ties
// taking `a` first.
template <bool ENC>
__device__ __forceinline__ u64 merge_path(const u64 *a, u64 na, const u64 *b, u64 nb, u64 diag) {
    u64 lo = diag > nb ? diag - nb : 0;
    u64 hi = diag < na ? diag : na;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (ld_enc<ENC>(a + mid) <= ld_enc<ENC>(b + diag - 1 - mid)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ u32 merge_path_smem(const u64 *a, u32 na, const u64 *b, u32 nb, u32 diag) {
    u32 lo = diag > nb ? diag - nb : 0;
    u32 hi = diag < na ? diag : na;
    while (lo < hi) {
        const u32 mid = (lo + hi) >> 1;
        if (a[mid] <= b[diag - 1 - mid]) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

template <bool ENC>
__global__ void merge_partition_kernel(const u64 *a, u64 na, const u64 *b, u64 nb, u64 n_splits, u64 *splits) {
    const u64 t = (u64) blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_splits) return;
    const u64 diag = min(t * (u64) MP_TILE, na + nb);
    splits[t] = merge_path<ENC>(a, na, b, nb, diag);
}

struct MpSmem {
    u64 in[MP_TILE];
    u64 out[MP_TILE];
    u32 scratch[MP_THREADS / 32 + 1];
    u32 tile;
    u64 excl;
};

// Loads the tile's slices of a and b into s.in ([0, la) then [la, la+lb)).
template <bool ENC>
__device__ __forceinline__ void load_tile(MpSmem &s, const u64 *a, u64 a0, u32 la, const u64 *b, u64 b0, u32 lb) {
    for (u32 i = threadIdx.x; i < la + lb; i += MP_THREADS)
        s.in[i] = (i < la) ? ld_enc<ENC>(a + a0 + i) : ld_enc<ENC>(b + b0 + (i - la));
}

template <bool ENC, bool WRITE_FULL, bool WRITE_DELTA>
__global__ void __launch_bounds__(MP_THREADS)
diff_merge_kernel(const u64 *__restrict__ full, u64 nfull, const u64 *__restrict__ jw, u64 nj,
                  const u64 *__restrict__ splits, u64 *__restrict__ full_out, u64 *__restrict__ delta_out,
                  u64 *lb, u32 *tile_ctr, u32 epoch, u32 *err, u64 *delta_count) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MpSmem &s = *reinterpret_cast<MpSmem *>(smem_raw);
    const int tid = threadIdx.x;
    if (tid == 0) s.tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const u32 tile = s.tile;
    const u64 total = nfull + nj;
    const u64 d0 = (u64) tile * MP_TILE;
    const u64 d1 = min(d0 + MP_TILE, total);
    const u64 a0 = splits[tile], a1 = splits[tile + 1];
    const u64 b0 = d0 - a0, b1 = d1 - a1;
    const u32 la = (u32) (a1 - a0), lbn = (u32) (b1 - b0);
    load_tile<ENC>(s, full, a0, la, jw, b0, lbn);
    __syncthreads();

    const u64 *sa = s.in;
    const u64 *sb = s.in + la;
    const u32 td = min((u32) tid * MP_VT, la + lbn);
    u32 ta = merge_path_smem(sa, la, sb, lbn, td);
    u32 tb = td - ta;
    bool hp = false;
    u64 prev = 0;
    if (ta > 0) { prev = sa[ta - 1]; hp = true; }
    else if (a0 > 0) { prev = ld_enc<ENC>(full + a0 - 1); hp = true; }
    if (tb > 0) { const u64 v = sb[tb - 1]; prev = hp ? max(prev, v) : v; hp = true; }
    else if (b0 > 0) { const u64 v = ld_enc<ENC>(jw + b0 - 1); prev = hp ? max(prev, v) : v; hp = true; }

    const u32 ta_start = ta;
    u64 val[MP_VT];
    u32 is_a = 0, is_new = 0;
#pragma unroll
    for (int k = 0; k < MP_VT; ++k) {
        val[k] = 0;
        if (ta + tb < la + lbn) {
            const bool take_a = ta < la && (tb >= lbn || sa[ta] <= sb[tb]);
            const u64 v = take_a ? sa[ta] : sb[tb];
            if (take_a) { ++ta; is_a |= 1u << k; }
            else {
                ++tb;
                if (!hp || v != prev) is_new |= 1u << k;
            }
            prev = v;
            hp = true;
            val[k] = v;
        }
    }
    u32 tile_new;
    const u32 new_before = block_exclusive_sum<MP_THREADS / 32>((u32) __popc(is_new), s.scratch, &tile_new);
    if (tid < 32) {
        u64 excl = 0;
        if (tile == 0) {
            if (tid == 0) st_relaxed_u64(lb, lb_word(kStatusInc, epoch, tile_new));
        } else {
            if (tid == 0) st_relaxed_u64(lb + tile, lb_word(kStatusAgg, epoch, tile_new));
            excl = lookback_warp(lb, tile, epoch, err);
            if (tid == 0) st_relaxed_u64(lb + tile, lb_word(kStatusInc, epoch, excl + tile_new));
        }
        if (tid == 0) s.excl = excl;
    }
    __syncthreads();  // inputs no longer read; s.excl published
    {
        u32 na_run = ta_start, nn_run = new_before;
#pragma unroll
        for (int k = 0; k < MP_VT; ++k) {
            const bool a = (is_a >> k) & 1u, nw = (is_new >> k) & 1u;
            if (WRITE_FULL && (a || nw)) s.out[na_run + nn_run] = val[k];
            if (WRITE_DELTA && nw) s.in[nn_run] = val[k];
            na_run += a;
            nn_run += nw;
        }
    }
    __syncthreads();
    const u64 excl = s.excl;
    if (WRITE_FULL) {
        const u32 nout = la + tile_new;
        u64 *dst = full_out + a0 + excl;
        for (u32 i = tid; i < nout; i += MP_THREADS) dst[i] = ENC ? entity_decode(s.out[i]) : s.out[i];
    }
    if (WRITE_DELTA) {
        u64 *dst = delta_out + excl;
        for (u32 i = tid; i < tile_new; i += MP_THREADS) dst[i] = ENC ? entity_decode(s.in[i]) : s.in[i];
    }
    if (d1 == total && tid == 0) *delta_count = excl + tile_new;
}

template <bool ENC>
__global__ void __launch_bounds__(MP_THREADS)
merge_kernel(const u64 *__restrict__ a, u64 na, const u64 *__restrict__ b, u64 nb, const u64 *__restrict__ splits,
             u64 *__restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MpSmem &s = *reinterpret_cast<MpSmem *>(smem_raw);
    const int tid = threadIdx.x;
    const u64 tile = blockIdx.x;
    const u64 total = na + nb;
    const u64 d0 = tile * MP_TILE;
    const u64 d1 = min(d0 + MP_TILE, total);
    const u64 a0 = splits[tile], a1 = splits[tile + 1];
    const u64 b0 = d0 - a0, b1 = d1 - a1;
    const u32 la = (u32) (a1 - a0), lbn = (u32) (b1 - b0);
    load_tile<ENC>(s, a, a0, la, b, b0, lbn);
    __syncthreads();
    const u64 *sa = s.in;
    const u64 *sb = s.in + la;
    const u32 td = min((u32) tid * MP_VT, la + lbn);
    u32 ta = merge_path_smem(sa, la, sb, lbn, td);
    u32 tb = td - ta;
#pragma unroll
    for (int k = 0; k < MP_VT; ++k) {
        if (ta + tb < la + lbn) {
            const bool take_a = ta < la && (tb >= lbn || sa[ta] <= sb[tb]);
            s.out[td + k] = take_a ? sa[ta++] : sb[tb++];
        }
    }
    __syncthreads();
    for (u32 i = tid; i < la + lbn; i += MP_THREADS) out[d0 + i] = ENC ? entity_decode(s.out[i]) : s.out[i];
}

u64 *partition(Context &ctx, const u64 *a, u64 na, const u64 *b, u64 nb, Codec codec, u64 &tiles) {
    tiles = (na + nb + MP_TILE - 1) / MP_TILE;
    // Look-back words of the launch occupy [0, tiles + 1) of the context's
    // look-back buffer; the split points follow them.
    u64 *splits = ctx.lookback_words(2 * (tiles + 1)) + (tiles + 1);
    const unsigned grid = (unsigned) ((tiles + 1 + 255) / 256);
    if (codec == Codec::Entity) DL_LAUNCH(ctx, K_MERGE_PARTITION, 0, merge_partition_kernel<true><<<grid, 256, 0, ctx.stream>>>(a, na, b, nb, tiles + 1, splits));
    else DL_LAUNCH(ctx, K_MERGE_PARTITION, 0, merge_partition_kernel<false><<<grid, 256, 0, ctx.stream>>>(a, na, b, nb, tiles + 1, splits));
    return splits;
}

template <bool ENC, bool WF, bool WD>
void launch_diff_merge(Context &ctx, const u64 *full, u64 nfull, const u64 *j, u64 nj, const u64 *splits, u64 tiles,
                       u64 *full_out, u64 *delta_out, u64 *lb, u32 *ctr, u64 *cnt) {
    auto kern = diff_merge_kernel<ENC, WF, WD>;
    DL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sizeof(MpSmem)));
    DL_LAUNCH(ctx, K_DIFF_MERGE, 8.0 * (2 * nfull + nj), kern<<<(unsigned) tiles, MP_THREADS, sizeof(MpSmem), ctx.stream>>>(full, nfull, j, nj, splits, full_out, delta_out,
                                                                       lb, ctr, ctx.next_epoch(), &ctx.ctrl->err, cnt));
}

}  // namespace

void merge_words(Context &ctx, const u64 *a, u64 na, const u64 *b, u64 nb, u64 *out, Codec codec) {
    if (na + nb == 0) return;
    u64 tiles;
    u64 *splits = partition(ctx, a, na, b, nb, codec, tiles);
    if (codec == Codec::Entity) {
        DL_CUDA(cudaFuncSetAttribute(merge_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sizeof(MpSmem)));
        DL_LAUNCH(ctx, K_MERGE, 16.0 * (na + nb), merge_kernel<true><<<(unsigned) tiles, MP_THREADS, sizeof(MpSmem), ctx.stream>>>(a, na, b, nb, splits, out));
    } else {
        DL_CUDA(cudaFuncSetAttribute(merge_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sizeof(MpSmem)));
        DL_LAUNCH(ctx, K_MERGE, 16.0 * (na + nb), merge_kernel<false><<<(unsigned) tiles, MP_THREADS, sizeof(MpSmem), ctx.stream>>>(a, na, b, nb, splits, out));
    }
    DL_CHECK_LAUNCH();
}

u64 diff_merge_words(Context &ctx, const u64 *full, u64 nfull, const u64 *j, u64 nj, u64 *full_out, u64 *delta_out,
                     Codec codec) {
    if (nfull + nj == 0) return 0;
    u64 tiles;
    u64 *splits = partition(ctx, full, nfull, j, nj, codec, tiles);
    u64 *lb = ctx.lookback.as<u64>();  // first tiles+1 words (reserved by partition)
    u32 *ctr = ctx.tile_counter(40);
    u64 *cnt = &ctx.ctrl->scalar[1];
    DL_CUDA(cudaMemsetAsync(ctr, 0, sizeof(u32), ctx.stream));
    const bool ent = codec == Codec::Entity;
    const bool wf = full_out != nullptr, wd = delta_out != nullptr;
#define DL_DM(E, F, D) launch_diff_merge<E, F, D>(ctx, full, nfull, j, nj, splits, tiles, full_out, delta_out, lb, ctr, cnt)
    if (ent) {
        if (wf && wd) DL_DM(true, true, true);
        else if (wf) DL_DM(true, true, false);
        else DL_DM(true, false, true);
    } else {
        if (wf && wd) DL_DM(false, true, true);
        else if (wf) DL_DM(false, true, false);
        else DL_DM(false, false, true);
    }
#undef DL_DM
    DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, cnt, sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    const u64 nd = ctx.host_scalars[0];
    ctx.prof_add_bytes(K_DIFF_MERGE, 8.0 * ((wf ? (double) nd : -(double) nfull) + (wd ? (double) nd : 0.0)));
    return nd;
}

}  // namespace dl
