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
// tile boundary). Inputs are staged in shared memory, every thread merges 8
// words serially, outputs leave through the same 32 KiB buffer in coalesced
// runs (3 CTAs of 16 warps per SM).
#include "dl_internal.h"

namespace dl {
namespace {

// 2048-word tiles of 256 threads: six tiles per SM overlap each other's
// load, search and store phases (the per-tile work between the loads and
// the stores otherwise leaves the memory pipe idle).
constexpr int MP_THREADS = 256;
constexpr int MP_VT = 8;
constexpr int MP_TILE = MP_THREADS * MP_VT;
constexpr int MP_BLOCKS_PER_SM = 1536 / MP_THREADS;

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

// One 32 KiB buffer: the tile's inputs, then (after the merge, values in
// registers) the staged outputs.
struct MpSmem {
    u64 buf[MP_TILE];
    u32 scratch[MP_THREADS / 32 + 1];
    u32 tile;
    u64 excl;
};

// Loads the tile's slices of a and b into s.buf ([0, la) then [la, la+lb)).
template <bool ENC>
__device__ __forceinline__ void load_tile(MpSmem &s, const u64 *a, u64 a0, u32 la, const u64 *b, u64 b0, u32 lb) {
#pragma unroll
    for (int k = 0; k < MP_VT; ++k) {
        const u32 i = k * MP_THREADS + threadIdx.x;
        if (i < la + lb) s.buf[i] = (i < la) ? ld_enc<ENC>(a + a0 + i) : ld_enc<ENC>(b + b0 + (i - la));
    }
}

// Shared memory of diff_merge: the tile's slices of full and J (then the
// tile's full' output) and the tile's new J words.
struct DmSmem {
    u64 buf[MP_TILE];
    u64 dst[MP_TILE];
    u32 scratch[MP_THREADS / 32 + 1];
    u32 tile;
    u32 has_prev;
    u64 prev;
    LookbackScratch lbs;
};

// The fused step as a balanced merge: every thread takes MP_VT consecutive
// positions of merge(full, J) (ties take the full word first), so a J word is
// a duplicate exactly when it equals the merged word before it. Kept words
// form full' = full u J, the J words among them form delta = J \ full
// deduplicated. One packed block scan gives both output offsets within the
// tile; only the delta count needs the decoupled look-back, since the tile's
// full' offset is its full offset plus the delta words before it.
template <bool ENC, bool WRITE_FULL, bool WRITE_DELTA>
__global__ void __launch_bounds__(MP_THREADS, MP_BLOCKS_PER_SM)
diff_merge_kernel(const u64 *__restrict__ full, u64 nfull, const u64 *__restrict__ jw, u64 nj,
                  const u64 *__restrict__ splits, u64 *__restrict__ full_out, u64 *__restrict__ delta_out,
                  u64 *lb, u32 *tile_ctr, u32 epoch, u32 *err, u64 *delta_count) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DmSmem &s = *reinterpret_cast<DmSmem *>(smem_raw);
    const int tid = threadIdx.x;
    if (tid == 0) s.tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const u32 tile = s.tile;
    const u64 total = nfull + nj;
    const u64 d0 = (u64) tile * MP_TILE;
    const u64 d1 = min(d0 + MP_TILE, total);
    const u64 a0 = splits[tile], a1 = splits[tile + 1];
    const u64 b0 = d0 - a0, b1 = d1 - a1;
    const u32 la = (u32) (a1 - a0), lbn = (u32) (b1 - b0), n = la + lbn;
#pragma unroll
    for (int k = 0; k < MP_VT; ++k) {
        const u32 i = k * MP_THREADS + tid;
        if (i < n) s.buf[i] = (i < la) ? ld_enc<ENC>(full + a0 + i) : ld_enc<ENC>(jw + b0 + (i - la));
    }
    if (tid == 0) {  // the merged word just before the tile: the larger of the two predecessors
        u64 p = 0;
        u32 hp = 0;
        if (a0 > 0) {
            p = ld_enc<ENC>(full + a0 - 1);
            hp = 1;
        }
        if (b0 > 0) {
            const u64 q = ld_enc<ENC>(jw + b0 - 1);
            if (!hp || q > p) p = q;
            hp = 1;
        }
        s.prev = p;
        s.has_prev = hp;
    }
    __syncthreads();
    const u64 *sa = s.buf, *sb = s.buf + la;
    const u32 diag = min((u32) tid * MP_VT, n);
    u32 ta = merge_path_smem(sa, la, sb, lbn, diag);
    u32 tb = diag - ta;
    u64 last;
    bool hl;
    if (diag == 0) {
        last = s.prev;
        hl = s.has_prev != 0;
    } else {
        const u64 xa = ta > 0 ? sa[ta - 1] : 0ull, xb = tb > 0 ? sb[tb - 1] : 0ull;
        last = (ta > 0 && (tb == 0 || xa >= xb)) ? xa : xb;
        hl = true;
    }
    u64 val[MP_VT];
    u32 keep = 0, isnew = 0;
#pragma unroll
    for (int k = 0; k < MP_VT; ++k) {
        val[k] = 0;
        if (diag + k < n) {
            const bool take_a = ta < la && (tb >= lbn || sa[ta] <= sb[tb]);
            const u64 v = take_a ? sa[ta] : sb[tb];
            if (take_a) {
                ++ta;
                keep |= 1u << k;
            } else {
                ++tb;
                if (!hl || v != last) {
                    keep |= 1u << k;
                    isnew |= 1u << k;
                }
            }
            val[k] = v;
            last = v;
            hl = true;
        }
    }
    u32 tot;
    const u32 ex = block_exclusive_sum<MP_THREADS / 32>((u32) __popc(keep) | ((u32) __popc(isnew) << 16), s.scratch,
                                                        &tot);
    const u32 tile_keep = tot & 0xFFFFu, tile_new = tot >> 16;
    u64 excl = 0;
    if (tile == 0) {
        if (tid == 0) st_relaxed_u64(lb, lb_word(kStatusInc, epoch, tile_new));
    } else {
        if (tid == 0) st_relaxed_u64(lb + tile, lb_word(kStatusAgg, epoch, tile_new));
        excl = lookback_block<MP_THREADS / 32>(lb, tile, epoch, err, s.lbs);
        if (tid == 0) st_relaxed_u64(lb + tile, lb_word(kStatusInc, epoch, excl + tile_new));
    }
    __syncthreads();  // every thread is done reading the input slices
    {
        u32 r = ex & 0xFFFFu, q = ex >> 16;
#pragma unroll
        for (int k = 0; k < MP_VT; ++k) {
            if (WRITE_FULL && ((keep >> k) & 1u)) s.buf[r++] = val[k];
            if (WRITE_DELTA && ((isnew >> k) & 1u)) s.dst[q++] = val[k];
        }
    }
    __syncthreads();
    if (WRITE_FULL) {
        u64 *out = full_out + a0 + excl;
        for (u32 i = tid; i < tile_keep; i += MP_THREADS) out[i] = ENC ? entity_decode(s.buf[i]) : s.buf[i];
    }
    if (WRITE_DELTA) {
        u64 *out = delta_out + excl;
        for (u32 i = tid; i < tile_new; i += MP_THREADS) out[i] = ENC ? entity_decode(s.dst[i]) : s.dst[i];
    }
    if (d1 == total && tid == 0) *delta_count = excl + tile_new;
}

template <bool ENC>
__global__ void __launch_bounds__(MP_THREADS, MP_BLOCKS_PER_SM)
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
    const u64 *sa = s.buf;
    const u64 *sb = s.buf + la;
    const u32 td = min((u32) tid * MP_VT, la + lbn);
    u32 ta = merge_path_smem(sa, la, sb, lbn, td);
    u32 tb = td - ta;
    u64 val[MP_VT];
#pragma unroll
    for (int k = 0; k < MP_VT; ++k) {
        if (ta + tb < la + lbn) {
            const bool take_a = ta < la && (tb >= lbn || sa[ta] <= sb[tb]);
            val[k] = take_a ? sa[ta++] : sb[tb++];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < MP_VT; ++k)
        if (td + k < la + lbn) s.buf[td + k] = val[k];
    __syncthreads();
    for (u32 i = tid; i < la + lbn; i += MP_THREADS) out[d0 + i] = ENC ? entity_decode(s.buf[i]) : s.buf[i];
}

// Every SAMPLE_STRIDE-th word of a sorted run: a small L2-resident index
// that narrows the binary search of a probe to one block of the run.
constexpr u64 SAMPLE_STRIDE = 4096;

__global__ void sample_kernel(const u64 *__restrict__ run, u64 n, u64 *__restrict__ sample, u64 ns) {
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += (u64) gridDim.x * blockDim.x)
        sample[i] = run[i * SAMPLE_STRIDE];
}

// Sparse set difference of sorted J (duplicates allowed) against a sorted
// duplicate-free run: out[i] = J[i] if J[i] differs from J[i-1] and is not in
// the run, else the all-ones word (never a compact tuple word). One thread per
// J word: binary search of the sample, then of one 4096-word block.
__global__ void sparse_mark_kernel(const u64 *__restrict__ j, u64 nj, const u64 *__restrict__ run, u64 nrun,
                                   const u64 *__restrict__ sample, u64 ns, u64 *__restrict__ out) {
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < nj; i += (u64) gridDim.x * blockDim.x) {
        const u64 b = j[i];
        bool keep = (i == 0) || j[i - 1] != b;
        if (keep && nrun) {
            u64 lo = 0, hi = ns;  // last sample <= b
            while (lo < hi) {
                const u64 mid = (lo + hi) >> 1;
                if (sample[mid] <= b) lo = mid + 1;
                else hi = mid;
            }
            if (lo > 0) {
                u64 l = (lo - 1) * SAMPLE_STRIDE, h = min(l + SAMPLE_STRIDE, nrun);
                while (l < h) {
                    const u64 mid = (l + h) >> 1;
                    if (run[mid] < b) l = mid + 1;
                    else h = mid;
                }
                keep = !(l < nrun && run[l] == b);
            }
        }
        out[i] = keep ? b : ~0ull;
    }
}

u64 *partition(Context &ctx, const u64 *a, u64 na, const u64 *b, u64 nb, Codec codec, u64 &tiles) {
    tiles = (na + nb + MP_TILE - 1) / MP_TILE;
    // The split points get their own buffer: the look-back buffer is cleared
    // whenever the launch epoch wraps, which may happen at the next launch.
    if ((tiles + 1) * sizeof(u64) > ctx.merge_splits.cap) {
        ctx.sync();
        ctx.merge_splits.reserve((tiles + 1) * sizeof(u64));
    }
    u64 *splits = ctx.merge_splits.as<u64>();
    const unsigned grid = (unsigned) ((tiles + 1 + 255) / 256);
    if (codec == Codec::Entity) DL_LAUNCH(ctx, K_MERGE_PARTITION, 0, merge_partition_kernel<true><<<grid, 256, 0, ctx.stream>>>(a, na, b, nb, tiles + 1, splits));
    else DL_LAUNCH(ctx, K_MERGE_PARTITION, 0, merge_partition_kernel<false><<<grid, 256, 0, ctx.stream>>>(a, na, b, nb, tiles + 1, splits));
    return splits;
}

template <bool ENC, bool WF, bool WD>
void launch_diff_merge(Context &ctx, const u64 *full, u64 nfull, const u64 *j, u64 nj, const u64 *splits, u64 tiles,
                       u64 *full_out, u64 *delta_out, u64 *lb, u32 *ctr, u64 *cnt) {
    auto kern = diff_merge_kernel<ENC, WF, WD>;
    DL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sizeof(DmSmem)));
    DL_LAUNCH(ctx, K_DIFF_MERGE, 8.0 * (2 * nfull + nj), kern<<<(unsigned) tiles, MP_THREADS, sizeof(DmSmem), ctx.stream>>>(full, nfull, j, nj, splits, full_out, delta_out,
                                                                       lb, ctr, ctx.next_epoch(), &ctx.ctrl->err, cnt));
}

}  // namespace

void run_sample(Context &ctx, const u64 *run, u64 n, DevBuf &sample, u64 &ns) {
    ns = (n + SAMPLE_STRIDE - 1) / SAMPLE_STRIDE;
    ctx.reserve(sample, std::max<u64>(ns, 1) * 8);
    if (ns)
        DL_LAUNCH(ctx, K_SPARSE_DIFF, 8.0 * ns,
                  sample_kernel<<<(unsigned) std::min<u64>((ns + 255) / 256, 4096), 256, 0, ctx.stream>>>(
                      run, n, sample.as<u64>(), ns));
}

u64 sparse_diff_words(Context &ctx, const u64 *run, u64 nrun, const u64 *sample, u64 ns, const u64 *j, u64 nj,
                      u64 *out) {
    if (nj == 0) return 0;
    const unsigned grid = (unsigned) std::min<u64>((nj + 255) / 256, (u64) ctx.sm_count * 16);
    // algorithmic bytes: J read + out written; the probes are counted as one
    // 32-byte sector per J word
    DL_LAUNCH(ctx, K_SPARSE_DIFF, 48.0 * nj,
              sparse_mark_kernel<<<grid, 256, 0, ctx.stream>>>(j, nj, run, nrun, sample, ns, out));
    return select_words(ctx, out, nj, out, 0);
}

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
    u64 *lb = ctx.lookback_words(tiles + 1);
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
