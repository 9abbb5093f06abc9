// LSD radix sort of 64-bit tuple words (the dedup step's sort).
//
// Replaces thrust::sort(set_cmp) on Entity arrays (tc.cu:250-253,
// sg.cu:282-287, wcc.cu:286-291), which dispatches to a comparison merge
// sort. Here every pass is one "onesweep" kernel: a tile of 6144 keys is
// ranked by 8-bit digit inside the CTA (warp ballots + per-warp counters,
// stable), the tile's digit counts are chained to earlier tiles by
// decoupled look-back, and the keys leave through shared memory so that the
// global writes of one digit run are contiguous. Only digits whose bits vary
// are sorted: the engine's compact words carry 2*B bits (B = bits per node
// index), the C-ABI path detects constant digits from the histogram.
//
// HBM traffic per pass: 8 B read + 8 B written per key (+ 8 B read once for
// the histogram unless a producer kernel accumulated it while writing).
#include "dl_internal.h"
#include "dl_scan.cuh"

namespace dl {
namespace {

constexpr int RADIX = 256;
constexpr int SORT_THREADS = 384;
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr int SORT_KPT_MAX = 16;
constexpr int HIST_THREADS = 512;

template <int KPT>
struct SortSmem {
    u64 keys[SORT_THREADS * KPT];
    u32 warp_cnt[SORT_WARPS][RADIX];
    u32 match[SORT_WARPS][RADIX];  // peer masks of the atomicOr ranking
    u64 gbase[RADIX];
    u32 tile_start[RADIX];
    u32 scratch[SORT_WARPS + 1];
    u32 tile;
};

template <bool ENC>
__global__ void __launch_bounds__(HIST_THREADS)
radix_hist_kernel(const u64 *__restrict__ keys, u64 n, int ndig, u64 *__restrict__ hist) {
    __shared__ u32 sh[8 * RADIX];
    for (int i = threadIdx.x; i < 8 * RADIX; i += HIST_THREADS) sh[i] = 0;
    __syncthreads();
    const u64 stride = (u64) gridDim.x * HIST_THREADS;
    for (u64 i = (u64) blockIdx.x * HIST_THREADS + threadIdx.x; i < n; i += stride) {
        u64 k = __ldcs(keys + i);
        if (ENC) k = entity_encode(k);
#pragma unroll
        for (int d = 0; d < 8; ++d)
            if (d < ndig) atomicAdd(&sh[d * RADIX + ((k >> (8 * d)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ndig * RADIX; i += HIST_THREADS) {
        u32 c = sh[i];
        if (c) atomicAdd((unsigned long long *) &hist[i], (unsigned long long) c);
    }
}

// One block per digit: bucket[d][b] = exclusive scan of hist[d][*]; marks the
// digits on which all keys agree (nothing to sort).
__global__ void __launch_bounds__(RADIX) radix_bucket_kernel(const u64 *__restrict__ hist, u64 *__restrict__ bucket,
                                                             u64 n, u32 *trivial_mask) {
    __shared__ u64 scratch[RADIX / 32 + 1];
    const int d = blockIdx.x;
    u64 c = hist[d * RADIX + threadIdx.x];
    u64 tot;
    u64 ex = block_exclusive_sum<RADIX / 32>(c, scratch, &tot);
    bucket[d * RADIX + threadIdx.x] = ex;
    if (c == n) atomicOr(trivial_mask, 1u << d);
}

// Ranking of a key's digit among the warp's lanes ("peers"):
//   RANK_BALLOT = 0: 8 warp ballots, one per digit bit;
//   RANK_ATOMIC = 1: every lane sets its bit in a per-(warp, digit) shared
//                    mask with atomicOr and reads the mask back.
constexpr int RANK_BALLOT = 0;
constexpr int RANK_ATOMIC = 1;

template <bool ENC, bool DEC, int RANK, int KPT, int MINB>
__global__ void __launch_bounds__(SORT_THREADS, MINB)
onesweep_kernel(const u64 *__restrict__ in, u64 *__restrict__ out, u64 n, int shift,
                const u64 *__restrict__ bucket, u64 *lb, u32 *tile_ctr, u32 epoch, u32 *err) {
    constexpr int SORT_KPT = KPT;
    constexpr int SORT_TILE = SORT_THREADS * KPT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem<KPT> &s = *reinterpret_cast<SortSmem<KPT> *>(smem_raw);
    const int tid = threadIdx.x;
    const u32 lane = tid & 31;
    const int w = tid >> 5;

    for (int i = tid; i < SORT_WARPS * RADIX; i += SORT_THREADS) {
        (&s.warp_cnt[0][0])[i] = 0;
        if (RANK == RANK_ATOMIC) (&s.match[0][0])[i] = 0;
    }
    if (tid == 0) s.tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const u32 tile = s.tile;
    const u64 tile_base = (u64) tile * SORT_TILE;
    const u32 n_valid = (u32) min((u64) SORT_TILE, n - tile_base);

    // Warp-contiguous blocks, lane-striped items: coalesced 256 B loads, and
    // (warp, item, lane) order equals input order, which keeps ranks stable.
    u64 k[SORT_KPT];
    const u64 wbase = tile_base + (u64) w * 32 * SORT_KPT + lane;
#pragma unroll
    for (int i = 0; i < SORT_KPT; ++i) {
        const u64 idx = wbase + (u64) i * 32;
        if (idx < n) {
            u64 x = __ldcs(in + idx);
            k[i] = ENC ? entity_encode(x) : x;
        } else {
            k[i] = ~0ull;  // ranks after every valid key of digit 255
        }
    }

    u32 rank[SORT_KPT];
    const u32 lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < SORT_KPT; ++i) {
        const u32 d = (u32) (k[i] >> shift) & 255u;
        u32 peers;
        if (RANK == RANK_BALLOT) {
            peers = 0xffffffffu;
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                const u32 bit = (d >> b) & 1u;
                const u32 bal = __ballot_sync(0xffffffffu, bit);
                peers &= bit ? bal : ~bal;
            }
        } else {
            atomicOr(&s.match[w][d], 1u << lane);
            __syncwarp();
            peers = *reinterpret_cast<volatile u32 *>(&s.match[w][d]);
            __syncwarp();
        }
        const u32 leader = __ffs(peers) - 1;
        u32 prev = 0;
        if (lane == leader) {
            prev = s.warp_cnt[w][d];
            s.warp_cnt[w][d] = prev + __popc(peers);
            if (RANK == RANK_ATOMIC) s.match[w][d] = 0;
        }
        __syncwarp();
        prev = __shfl_sync(0xffffffffu, prev, leader);
        rank[i] = prev + __popc(peers & lt);
    }
    __syncthreads();

    u32 cnt_all = 0, cnt_valid = 0;
    if (tid < RADIX) {
        u32 sum = 0;
#pragma unroll
        for (int ww = 0; ww < SORT_WARPS; ++ww) {
            const u32 c = s.warp_cnt[ww][tid];
            s.warp_cnt[ww][tid] = sum;
            sum += c;
        }
        cnt_all = sum;
        cnt_valid = (tid == RADIX - 1) ? sum - (SORT_TILE - n_valid) : sum;
        st_relaxed_u64(lb + (u64) tile * RADIX + tid, lb_word(tile == 0 ? kStatusInc : kStatusAgg, epoch, cnt_valid));
    }
    u32 total;
    const u32 start = block_exclusive_sum<SORT_WARPS>(tid < RADIX ? cnt_all : 0u, s.scratch, &total);
    if (tid < RADIX) {
        s.tile_start[tid] = start;
        u64 excl = 0;
        if (tile > 0) {
            excl = lookback_serial(lb + tid, tile, RADIX, epoch, err);
            st_relaxed_u64(lb + (u64) tile * RADIX + tid, lb_word(kStatusInc, epoch, excl + cnt_valid));
        }
        s.gbase[tid] = bucket[tid] + excl - start;
    }
    __syncthreads();

#pragma unroll
    for (int i = 0; i < SORT_KPT; ++i) {
        const u32 d = (u32) (k[i] >> shift) & 255u;
        s.keys[s.tile_start[d] + s.warp_cnt[w][d] + rank[i]] = k[i];
    }
    __syncthreads();

    for (u32 j = tid; j < n_valid; j += SORT_THREADS) {
        const u64 x = s.keys[j];
        const u32 d = (u32) (x >> shift) & 255u;
        out[s.gbase[d] + j] = DEC ? entity_decode(x) : x;
    }
}

}  // namespace

Tuning default_tuning() {
    static const Tuning t = [] {
        Tuning d;
        const char *e = getenv("DL_SORT_RANK");
        if (e && std::string(e) == "ballot") d.rank = RANK_BALLOT;
        e = getenv("DL_SORT_KPT");
        if (e && std::string(e) == "12") d.sort_kpt = 12;
        e = getenv("DL_SORT_ALGO");
        if (e && std::string(e) == "onesweep") d.sort_algo = 0;
        e = getenv("DL_SORT_TMA");
        if (e && std::string(e) == "0") d.sort_tma = 0;
        e = getenv("DL_JOIN_FIRST_PASS");
        if (e && std::string(e) == "0") d.join_first_pass = 0;
        return d;
    }();
    return t;
}

namespace {

template <bool ENC, bool DEC, int KPT, int MINB>
void launch_onesweep_k(Context &ctx, const u64 *in, u64 *out, u64 n, int shift, const u64 *bucket, u64 *lb, u32 *ctr) {
    auto kern = ctx.tune.rank == RANK_BALLOT ? onesweep_kernel<ENC, DEC, RANK_BALLOT, KPT, MINB>
                                             : onesweep_kernel<ENC, DEC, RANK_ATOMIC, KPT, MINB>;
    const int smem = (int) sizeof(SortSmem<KPT>);
    DL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const u64 tile = (u64) SORT_THREADS * KPT;
    const u64 tiles = (n + tile - 1) / tile;
    DL_LAUNCH(ctx, K_SORT_PASS, 16.0 * n,
              kern<<<(unsigned) tiles, SORT_THREADS, smem, ctx.stream>>>(in, out, n, shift, bucket, lb, ctr,
                                                                          ctx.next_epoch(), &ctx.ctrl->err));
}

u64 sort_tile_keys(const Context &ctx) { return (u64) SORT_THREADS * ctx.tune.sort_kpt; }

template <bool ENC, bool DEC>
void launch_onesweep(Context &ctx, const u64 *in, u64 *out, u64 n, int shift, const u64 *bucket, u64 *lb,
                     u32 *ctr) {
    if (ctx.tune.sort_kpt == 12) launch_onesweep_k<ENC, DEC, 12, 3>(ctx, in, out, n, shift, bucket, lb, ctr);
    else launch_onesweep_k<ENC, DEC, 16, 2>(ctx, in, out, n, shift, bucket, lb, ctr);
}

// ---- three-kernel LSD pass: upsweep / spine / downsweep ---------------------
// A pass without inter-CTA waits: CTA c owns a contiguous chunk of keys. The
// upsweep counts the chunk's digits, a scan over the digit-major [256][G]
// matrix gives every (digit, CTA) its first output position, and the
// downsweep streams the chunk tile by tile (TMA bulk loads, double-buffered
// behind an mbarrier) keeping a running offset per digit. Traffic per pass:
// 8 B (upsweep) + 16 B (downsweep) per key.
constexpr int DS_THREADS = 256;
constexpr int DS_WARPS = DS_THREADS / 32;
constexpr int DS_KPT = 16;
constexpr int DS_TILE = DS_THREADS * DS_KPT;  // 4096 keys, 32 KiB
constexpr int US_THREADS = 512;

struct DsSmem {
    u64 buf[2][DS_TILE];  // TMA landing buffers; the current one also stages the scatter
    u32 warp_cnt[DS_WARPS][RADIX];
    u32 match[DS_WARPS][RADIX];
    u64 run_off[RADIX];
    u64 gbase[RADIX];
    u32 scratch[DS_WARPS + 1];
    u64 bar[2];
};

template <bool ENC>
__global__ void __launch_bounds__(US_THREADS)
radix_upsweep_kernel(const u64 *__restrict__ in, u64 n, int shift, u64 chunk, u32 G, u64 *__restrict__ hist) {
    __shared__ u32 h[US_THREADS / 32][RADIX];
    const int tid = threadIdx.x, w = tid >> 5;
    for (int i = tid; i < (US_THREADS / 32) * RADIX; i += US_THREADS) (&h[0][0])[i] = 0;
    __syncthreads();
    const u64 b = (u64) blockIdx.x * chunk;
    const u64 e = min(b + chunk, n);
    u64 i = b + tid;
    for (; i + 3 * US_THREADS < e; i += 4 * US_THREADS) {
        u64 k0 = __ldcs(in + i), k1 = __ldcs(in + i + US_THREADS), k2 = __ldcs(in + i + 2 * US_THREADS),
            k3 = __ldcs(in + i + 3 * US_THREADS);
        if (ENC) {
            k0 = entity_encode(k0);
            k1 = entity_encode(k1);
            k2 = entity_encode(k2);
            k3 = entity_encode(k3);
        }
        atomicAdd(&h[w][(k0 >> shift) & 255u], 1u);
        atomicAdd(&h[w][(k1 >> shift) & 255u], 1u);
        atomicAdd(&h[w][(k2 >> shift) & 255u], 1u);
        atomicAdd(&h[w][(k3 >> shift) & 255u], 1u);
    }
    for (; i < e; i += US_THREADS) {
        u64 k = __ldcs(in + i);
        if (ENC) k = entity_encode(k);
        atomicAdd(&h[w][(k >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (tid < RADIX) {
        u32 sum = 0;
#pragma unroll
        for (int ww = 0; ww < US_THREADS / 32; ++ww) sum += h[ww][tid];
        hist[(u64) tid * G + blockIdx.x] = sum;
    }
}

struct WordValue {
    const u64 *v;
    __device__ __forceinline__ u64 operator()(u64 i) const { return v[i]; }
};

template <bool ENC, bool DEC, int RANK>
__global__ void __launch_bounds__(DS_THREADS, 2)
radix_downsweep_kernel(const u64 *__restrict__ in, u64 *__restrict__ out, u64 n, int shift, u64 chunk, u32 G,
                       const u64 *__restrict__ offsets, int use_tma, u32 *err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    DsSmem &s = *reinterpret_cast<DsSmem *>(smem_raw);
    const int tid = threadIdx.x;
    const u32 lane = tid & 31;
    const int w = tid >> 5;
    const u64 cb = (u64) blockIdx.x * chunk;
    if (cb >= n) return;
    const u64 ce = min(cb + chunk, n);
    const u32 ntiles = (u32) ((ce - cb + DS_TILE - 1) / DS_TILE);
    if (tid < RADIX) s.run_off[tid] = offsets[(u64) tid * G + blockIdx.x];
    for (int i = tid; i < DS_WARPS * RADIX; i += DS_THREADS) {
        (&s.warp_cnt[0][0])[i] = 0;
        (&s.match[0][0])[i] = 0;
    }
    auto issue = [&](u32 t, int slot) {  // thread 0 only
        const u64 tb = cb + (u64) t * DS_TILE;
        const u32 cnt = (u32) min((u64) DS_TILE, ce - tb);
        const u32 bytes = (cnt * 8u) & ~15u;
        mbar_expect_tx(&s.bar[slot], bytes ? bytes : 16u);
        if (bytes) tma_load_1d(s.buf[slot], in + tb, bytes, &s.bar[slot]);
        else mbar_complete_tx(&s.bar[slot], 16u);
    };
    if (use_tma && tid == 0) {
        mbar_init(&s.bar[0], 1);
        mbar_init(&s.bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (use_tma && tid == 0) {
        issue(0, 0);
        if (ntiles > 1) issue(1, 1);
    }
    u32 phase0 = 0, phase1 = 0;
    const u32 lt = lanemask_lt();
    for (u32 t = 0; t < ntiles; ++t) {
        const int slot = t & 1;
        u64 *buf = s.buf[slot];
        const u64 tb = cb + (u64) t * DS_TILE;
        const u32 cnt = (u32) min((u64) DS_TILE, ce - tb);
        u32 tma_words = 0;
        if (use_tma) {
            tma_words = ((cnt * 8u) & ~15u) / 8u;
            if (slot == 0) {
                mbar_wait(&s.bar[0], phase0, err);
                phase0 ^= 1;
            } else {
                mbar_wait(&s.bar[1], phase1, err);
                phase1 ^= 1;
            }
        }
        u64 k[DS_KPT];
        const u32 wb = (u32) w * 32 * DS_KPT + lane;
#pragma unroll
        for (int i = 0; i < DS_KPT; ++i) {
            const u32 li = wb + i * 32;
            if (li < cnt) {
                const u64 x = li < tma_words ? buf[li] : __ldcs(in + tb + li);
                k[i] = ENC ? entity_encode(x) : x;
            } else {
                k[i] = ~0ull;
            }
        }
        u32 rank[DS_KPT];
#pragma unroll
        for (int i = 0; i < DS_KPT; ++i) {
            const u32 d = (u32) (k[i] >> shift) & 255u;
            u32 peers;
            if (RANK == RANK_BALLOT) {  // lanes with the same digit: one ballot per digit bit
                peers = 0xffffffffu;
#pragma unroll
                for (int b = 0; b < 8; ++b) {
                    const u32 bit = (d >> b) & 1u;
                    const u32 bal = __ballot_sync(0xffffffffu, bit);
                    peers &= bit ? bal : ~bal;
                }
            } else {
                atomicOr(&s.match[w][d], 1u << lane);
                __syncwarp();
                peers = *reinterpret_cast<volatile u32 *>(&s.match[w][d]);
                __syncwarp();
            }
            const u32 leader = __ffs(peers) - 1;
            u32 prev = 0;
            if (lane == leader) {
                prev = s.warp_cnt[w][d];
                s.warp_cnt[w][d] = prev + __popc(peers);
                if (RANK == RANK_ATOMIC) s.match[w][d] = 0;
            }
            __syncwarp();
            prev = __shfl_sync(0xffffffffu, prev, leader);
            rank[i] = prev + __popc(peers & lt);
        }
        __syncthreads();  // ranks done; the landing buffer is no longer read
        u32 cnt_all = 0, cnt_valid = 0;
        if (tid < RADIX) {
            u32 sum = 0;
#pragma unroll
            for (int ww = 0; ww < DS_WARPS; ++ww) {
                const u32 c = s.warp_cnt[ww][tid];
                s.warp_cnt[ww][tid] = sum;
                sum += c;
            }
            cnt_all = sum;
            cnt_valid = (tid == RADIX - 1) ? sum - (DS_TILE - cnt) : sum;
        }
        u32 total;
        const u32 start = block_exclusive_sum<DS_WARPS>(tid < RADIX ? cnt_all : 0u, s.scratch, &total);
        if (tid < RADIX) {
            // warp_cnt[w][d] becomes the tile position of warp w's first key of digit d
#pragma unroll
            for (int ww = 0; ww < DS_WARPS; ++ww) s.warp_cnt[ww][tid] += start;
            s.gbase[tid] = s.run_off[tid] - start;
            s.run_off[tid] += cnt_valid;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < DS_KPT; ++i) {
            const u32 d = (u32) (k[i] >> shift) & 255u;
            buf[s.warp_cnt[w][d] + rank[i]] = k[i];
        }
        __syncthreads();
        if (tid < RADIX)
#pragma unroll
            for (int ww = 0; ww < DS_WARPS; ++ww) s.warp_cnt[ww][tid] = 0;
        for (u32 j = tid; j < cnt; j += DS_THREADS) {
            const u64 x = buf[j];
            const u32 d = (u32) (x >> shift) & 255u;
            out[s.gbase[d] + j] = DEC ? entity_decode(x) : x;
        }
        __syncthreads();  // buffer and counters free for the next tiles
        if (use_tma && tid == 0 && t + 2 < ntiles) issue(t + 2, slot);
    }
}

bool use_lsd3(const Context &ctx) { return ctx.tune.sort_algo == 1; }

template <bool ENC, bool DEC>
void lsd3_pass(Context &ctx, const u64 *in, u64 *out, u64 n, int shift, u32 G, u64 chunk, u64 *hist, u64 *offs) {
    DL_LAUNCH(ctx, K_SORT_HIST, 8.0 * n,
              radix_upsweep_kernel<ENC><<<G, US_THREADS, 0, ctx.stream>>>(in, n, shift, chunk, G, hist));
    const u64 m = (u64) RADIX * G;
    const u64 tiles = (m + SCAN_TILE - 1) / SCAN_TILE;
    u64 *lb = ctx.lookback_words(tiles);
    u32 *ctr = ctx.tile_counter(56);
    DL_CUDA(cudaMemsetAsync(ctr, 0, sizeof(u32), ctx.stream));
    DL_LAUNCH(ctx, K_SORT_BUCKET, 16.0 * m,
              scan_kernel<WordValue><<<(unsigned) tiles, SCAN_THREADS, 0, ctx.stream>>>(
                  WordValue{hist}, m, offs, lb, ctr, ctx.next_epoch(), &ctx.ctrl->err, &ctx.ctrl->scalar[12]));
    auto kern = ctx.tune.rank == RANK_BALLOT ? radix_downsweep_kernel<ENC, DEC, RANK_BALLOT>
                                             : radix_downsweep_kernel<ENC, DEC, RANK_ATOMIC>;
    const int smem = (int) sizeof(DsSmem);
    DL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int use_tma = (ctx.tune.sort_tma && (reinterpret_cast<uintptr_t>(in) & 15u) == 0) ? 1 : 0;
    DL_LAUNCH(ctx, K_SORT_PASS, 16.0 * n,
              kern<<<G, DS_THREADS, smem, ctx.stream>>>(in, out, n, shift, chunk, G, offs, use_tma, &ctx.ctrl->err));
}

// CTA count and chunk (a multiple of the tile) of a three-kernel pass over n
// keys; reserves the per-(digit, CTA) counts.
void lsd3_grid(Context &ctx, u64 n, u64 &G, u64 &chunk) {
    G = std::min<u64>((u64) ctx.sm_count * 2, (n + DS_TILE - 1) / DS_TILE);
    if (G == 0) G = 1;
    chunk = (n + G - 1) / G;
    chunk = (chunk + DS_TILE - 1) / DS_TILE * DS_TILE;
    G = (n + chunk - 1) / chunk;
    ctx.reserve(ctx.radix_part, 2 * RADIX * G * sizeof(u64));
}

}  // namespace

u64 *radix_sort_windows(Context &ctx, u64 *a, u64 *b, u64 n, const int *shifts, int nwin) {
    if (n <= 1 || nwin <= 0) return a;
    if (!use_lsd3(ctx)) return radix_sort(ctx, a, b, n, Codec::Raw, shifts[nwin - 1] + 8);
    u64 G, chunk;
    lsd3_grid(ctx, n, G, chunk);
    u64 *ph = ctx.radix_part.as<u64>();
    u64 *po = ph + RADIX * G;
    const u64 *src = a;
    u64 *dst = b;
    for (int p = 0; p < nwin; ++p) {
        lsd3_pass<false, false>(ctx, src, dst, n, shifts[p], (u32) G, chunk, ph, po);
        u64 *t = const_cast<u64 *>(src);
        src = dst;
        dst = t;
    }
    return const_cast<u64 *>(src);
}

int plan_windows(int field_bits, int used_bits, int *shifts) {
    const int B = field_bits, kb = std::max(1, std::min(used_bits, field_bits));
    const int per_field = (kb + 7) / 8;
    const int contiguous = (B + kb + 7) / 8;
    int n = 0;
    if (contiguous <= 2 * per_field) {
        for (int i = 0; i < contiguous; ++i) shifts[n++] = 8 * i;
    } else {
        for (int i = 0; i < per_field; ++i) shifts[n++] = 8 * i;
        for (int i = 0; i < per_field; ++i) shifts[n++] = B + 8 * i;
    }
    return n;
}

// Histogram bins [8][256] followed by bucket bases [8][256].
u64 *radix_hist_buffer(Context &ctx) {
    ctx.sort_hist.reserve(2 * 8 * RADIX * sizeof(u64));
    return ctx.sort_hist.as<u64>();
}

void radix_hist_clear(Context &ctx) {
    DL_CUDA(cudaMemsetAsync(radix_hist_buffer(ctx), 0, 8 * RADIX * sizeof(u64), ctx.stream));
}

u64 *radix_sort(Context &ctx, u64 *a, u64 *b, u64 n, Codec codec, int known_bits, u64 *hist_accumulated) {
    if (n <= 1) return a;
    const bool ent = codec == Codec::Entity;
    u64 *hist = radix_hist_buffer(ctx);
    u64 *bucket = hist + 8 * RADIX;
    u32 *ctr = ctx.tile_counter(0);
    u32 *mask = ctx.tile_counter(16);
    int digits[8];
    int nd = 0;
    DL_CUDA(cudaMemsetAsync(ctr, 0, 17 * sizeof(u32), ctx.stream));
    const int ndig = (known_bits > 0 && !ent) ? (known_bits + 7) / 8 : 8;
    const bool lsd3 = use_lsd3(ctx);
    if (known_bits > 0 && !ent) {
        for (int d = 0; d < ndig; ++d) digits[nd++] = d;
    }
    if (!(known_bits > 0 && !ent) || !lsd3) {
        const unsigned hgrid = (unsigned) std::min<u64>((n + HIST_THREADS * 8 - 1) / (HIST_THREADS * 8),
                                                        (u64) ctx.sm_count * 4);
        if (!hist_accumulated) {
            radix_hist_clear(ctx);
            if (ent)
                DL_LAUNCH(ctx, K_SORT_HIST, 8.0 * n,
                          radix_hist_kernel<true><<<hgrid, HIST_THREADS, 0, ctx.stream>>>(a, n, ndig, hist));
            else
                DL_LAUNCH(ctx, K_SORT_HIST, 8.0 * n,
                          radix_hist_kernel<false><<<hgrid, HIST_THREADS, 0, ctx.stream>>>(a, n, ndig, hist));
        }
        DL_LAUNCH(ctx, K_SORT_BUCKET, 0,
                  radix_bucket_kernel<<<ndig, RADIX, 0, ctx.stream>>>(hist, bucket, n, mask));
        if (!(known_bits > 0 && !ent)) {
            DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, mask, sizeof(u32), cudaMemcpyDeviceToHost, ctx.stream));
            ctx.sync();
            const u32 m = *reinterpret_cast<u32 *>(ctx.host_scalars);
            for (int d = 0; d < 8; ++d)
                if (!((m >> d) & 1u)) digits[nd++] = d;
        }
    }
    if (nd == 0) return a;
    const u64 *src = a;
    u64 *dst = b;
    if (lsd3) {
        u64 G, chunk;
        lsd3_grid(ctx, n, G, chunk);
        u64 *ph = ctx.radix_part.as<u64>();
        u64 *po = ph + RADIX * G;
        for (int p = 0; p < nd; ++p) {
            const bool enc = ent && p == 0, dec = ent && p == nd - 1;
            const int sh = 8 * digits[p];
            if (enc && dec) lsd3_pass<true, true>(ctx, src, dst, n, sh, (u32) G, chunk, ph, po);
            else if (enc) lsd3_pass<true, false>(ctx, src, dst, n, sh, (u32) G, chunk, ph, po);
            else if (dec) lsd3_pass<false, true>(ctx, src, dst, n, sh, (u32) G, chunk, ph, po);
            else lsd3_pass<false, false>(ctx, src, dst, n, sh, (u32) G, chunk, ph, po);
            u64 *t = const_cast<u64 *>(src);
            src = dst;
            dst = t;
        }
        return const_cast<u64 *>(src);
    }
    const u64 tiles = (n + sort_tile_keys(ctx) - 1) / sort_tile_keys(ctx);
    u64 *lb = ctx.lookback_words(tiles * RADIX);
    for (int p = 0; p < nd; ++p) {
        const bool enc = ent && p == 0, dec = ent && p == nd - 1;
        const u64 *bk = bucket + digits[p] * RADIX;
        const int sh = 8 * digits[p];
        if (enc && dec) launch_onesweep<true, true>(ctx, src, dst, n, sh, bk, lb, ctr + p);
        else if (enc) launch_onesweep<true, false>(ctx, src, dst, n, sh, bk, lb, ctr + p);
        else if (dec) launch_onesweep<false, true>(ctx, src, dst, n, sh, bk, lb, ctr + p);
        else launch_onesweep<false, false>(ctx, src, dst, n, sh, bk, lb, ctr + p);
        u64 *t = const_cast<u64 *>(src);
        src = dst;
        dst = t;
    }
    return const_cast<u64 *>(src);
}

bool radix_wants_histogram(const Context &ctx) { return !use_lsd3(ctx); }

}  // namespace dl
