// TC with the full relation held as a bit matrix over node ranks.
//
// The reference deduplicates each iteration's join output by sorting it,
// subtracting the sorted full relation and merging the difference back in
// (tc.cu:250-286). Here, when n x n bits fit in device memory (n = distinct
// node ids; 12.6 GB for 317K nodes), full is a bit matrix M with one row per
// path source x and one column per path target w, and one semi-naive step is
// a single pass over the join output: every join word (x, w) sets its bit with
// atomicOr, and it is a new tuple exactly when the bit was clear before. That
// is dedup(J) \ full and full u J at once, without materialising J: the
// delta is the same set as the reference's (each tuple is claimed by exactly
// one atomic), so per-iteration |delta| and the fixpoint are identical. The
// result leaves as sorted (target, source) words -- the reference's output
// order (tc.cu:345-366) -- through a bit-matrix transpose, row popcounts, a
// scan and an extraction pass.
//
// Locality: the first delta is the edge list in source-major order and every
// later delta is appended tile by tile in probe order, so the probe rows of
// one source stay close together and its matrix row (n / 8 bytes) stays in L2
// while their join outputs land in it.
#include "dl_engine_detail.h"
#include "dl_join.cuh"

namespace dl {
namespace detail {
namespace {

constexpr int TR_ROWS = 256;  // source rows per transpose tile
constexpr int TR_WORDS = 16;  // source words (512 columns) per transpose tile

// Word (w << bits) | x of a delta -> bit (x, w) of the matrix.
__global__ void bitmat_set_kernel(const u64 *__restrict__ words, u64 n, int bits, u32 *__restrict__ m, u64 stride) {
    const u64 mask = (1ull << bits) - 1;
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64) gridDim.x * blockDim.x) {
        const u64 v = words[i];
        const u64 w = v >> bits, x = v & mask;
        atomicOr(&m[x * stride + (w >> 5)], 1u << (w & 31));
    }
}

// Sorted (x << bits) | y edge words -> probe words (y << bits) | x in the
// same (source-major) order.
__global__ void swap_fields_kernel(const u64 *__restrict__ in, u64 n, int bits, u64 *__restrict__ out) {
    const u64 mask = (1ull << bits) - 1;
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64) gridDim.x * blockDim.x) {
        const u64 v = in[i];
        out[i] = ((v & mask) << bits) | (v >> bits);
    }
}

struct StepSmem {
    u64 obeg[JN_TILE + 1];    // first output of each loaded row; then the staged words' next offsets
    u64 begin[JN_TILE + 1];   // first match of each loaded row; then the staged new words
    u32 payload[JN_TILE + 1]; // probe value of each loaded row; then the staged words' degrees
    u64 scratch64[JN_THREADS / 32 + 1];
    u32 flags[(JN_TILE / JN_THREADS) * (JN_THREADS / 32)];  // new-word ballots, slot order
    u32 fbase[(JN_TILE / JN_THREADS) * (JN_THREADS / 32)];
    u32 nfresh;
    u64 base_cnt, base_deg;
    u32 tile;
};

// One semi-naive TC step over a delta: for probe row (y << bits) | x and
// every edge y -> w, test-and-set bit (x, w); the new tuples form the next
// delta as words (w << bits) | x, in tile order, together with the next
// step's join offsets (exclusive prefix of the new words' out-degrees) --
// so the next step needs no count pass. Tiles take their positions in the
// next delta by decoupled look-back on two columns (new words, their
// degrees); `totals` gets |next delta| and its join size. The tile/owner
// layout is the join emit's (rows and outputs merged along a merge path,
// `splits` from the same partition); the loads and atomics of a thread's
// items are issued in separate unrolled phases so that they overlap.
__global__ void __launch_bounds__(JN_THREADS, 4)
bitmat_step_kernel(CsrSrc<EmitKind::ZV> src, u64 n_probe, const u64 *__restrict__ offsets, u64 total,
                   const u64 *__restrict__ splits, u32 *__restrict__ m, u64 stride, u64 *__restrict__ out,
                   u64 *__restrict__ out_offsets, u64 capacity, u64 *lb_cnt, u64 *lb_deg, u32 *tile_ctr, u32 epoch,
                   u32 ntiles, u32 *err, u64 *totals) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StepSmem &s = *reinterpret_cast<StepSmem *>(smem_raw);
    constexpr u32 VT = JN_TILE / JN_THREADS;
    const int tid = threadIdx.x;
    if (tid == 0) s.tile = atomicAdd(tile_ctr, 1u);  // launch order: look-back always progresses
    __syncthreads();
    const u32 tile = s.tile;
    const u64 d0 = (u64) tile * JN_TILE;
    const u64 d1 = min(d0 + JN_TILE, n_probe + total);
    const u64 i0 = splits[tile], i1 = splits[tile + 1];
    const u64 o0 = d0 - i0, o1 = d1 - i1;
    const u64 istart = i0 > 0 ? i0 - 1 : 0;
    const u32 ni = (u32) (i1 - istart);
    {
        // rows: probe words and offsets first, then their index entries, so
        // that a thread's row loads are in flight together
        constexpr u32 RV = (JN_TILE + 1 + JN_THREADS - 1) / JN_THREADS;
        const u64 pmask = (1ull << src.bits) - 1;
        u64 pw[RV];
#pragma unroll
        for (u32 r = 0; r < RV; ++r) {
            const u32 j = tid + r * JN_THREADS;
            pw[r] = 0;
            if (j < ni) {
                pw[r] = src.probe[istart + j];
                s.obeg[j] = offsets[istart + j];
            }
        }
#pragma unroll
        for (u32 r = 0; r < RV; ++r) {
            const u32 j = tid + r * JN_THREADS;
            if (j < ni) {
                s.begin[j] = __ldg(src.off + (pw[r] >> src.bits));
                s.payload[j] = (u32) (pw[r] & pmask);
            }
        }
    }
    __syncthreads();
    // phase 1: owner row of every item (shared memory only)
    u64 idx[VT];
    u32 xs[VT];
    u32 valid = 0;
    u32 j = 0;
#pragma unroll
    for (u32 k = 0; k < VT; ++k) {
        idx[k] = 0;
        xs[k] = 0;
        const u64 o = o0 + tid + (u64) k * JN_THREADS;
        if (o < o1) {
            u32 lo = j, hi = ni;  // last loaded row whose first output is <= o
            while (lo < hi) {
                const u32 mid = (lo + hi) >> 1;
                if (s.obeg[mid] <= o) lo = mid + 1;
                else hi = mid;
            }
            j = lo - 1;
            idx[k] = s.begin[j] + (o - s.obeg[j]);
            xs[k] = s.payload[j];
            valid |= 1u << k;
        }
    }
    // phase 2: edge targets
    u32 wt[VT];
#pragma unroll
    for (u32 k = 0; k < VT; ++k) wt[k] = (valid >> k) & 1u ? __ldg(src.val + idx[k]) : 0u;
    // phase 3: test-and-set (all atomics issued before any result is used)
    u32 old[VT];
#pragma unroll
    for (u32 k = 0; k < VT; ++k)
        old[k] = (valid >> k) & 1u ? atomicOr(&m[(u64) xs[k] * stride + (wt[k] >> 5)], 1u << (wt[k] & 31)) : ~0u;
    u32 fresh = 0;
#pragma unroll
    for (u32 k = 0; k < VT; ++k)
        if (!((old[k] >> (wt[k] & 31)) & 1u)) fresh |= 1u << k;
    // phase 4: out-degrees of the new words (their join size next step)
    u32 dg[VT];
#pragma unroll
    for (u32 k = 0; k < VT; ++k) dg[k] = (fresh >> k) & 1u ? __ldg(src.off + wt[k] + 1) - __ldg(src.off + wt[k]) : 0u;
    // Compaction in join-output order (item k of thread t is slot t + k * JN_THREADS),
    // so the next delta keeps the probe order: grouped by source x.
    const u32 lane = tid & 31, warp = tid >> 5;
    u32 bal[VT];
#pragma unroll
    for (u32 k = 0; k < VT; ++k) {
        bal[k] = __ballot_sync(0xffffffffu, (fresh >> k) & 1u);
        if (lane == 0) s.flags[k * (JN_THREADS / 32) + warp] = bal[k];
    }
    __syncthreads();
    if (warp == 0) {  // exclusive prefix of the 64 flag words' popcounts, in slot order
        constexpr u32 NF = VT * (JN_THREADS / 32);
        static_assert(NF == 64, "two flag words per lane");
        const u32 c0 = __popc(s.flags[2 * lane]), c1 = __popc(s.flags[2 * lane + 1]);
        const u32 incl = warp_inclusive_sum(c0 + c1);
        s.fbase[2 * lane] = incl - c0 - c1;
        s.fbase[2 * lane + 1] = incl - c1;
        if (lane == 31) s.nfresh = incl;
    }
    __syncthreads();  // rows no longer read: obeg/begin/payload take the staged words
    const u32 lt = lanemask_lt();
#pragma unroll
    for (u32 k = 0; k < VT; ++k) {
        if ((fresh >> k) & 1u) {
            const u32 p = s.fbase[k * (JN_THREADS / 32) + warp] + __popc(bal[k] & lt);
            s.begin[p] = ((u64) wt[k] << src.bits) | xs[k];
            s.payload[p] = dg[k];
        }
    }
    __syncthreads();
    const u32 tot_cnt = s.nfresh;
    // degree prefix over the staged words (blocked: thread t owns VT consecutive)
    u64 mine = 0;
#pragma unroll
    for (u32 k = 0; k < VT; ++k) {
        const u32 p = tid * VT + k;
        mine += p < tot_cnt ? s.payload[p] : 0u;
    }
    u64 tot_deg;
    u64 dpos = block_exclusive_sum<JN_THREADS / 32>(mine, s.scratch64, &tot_deg);
#pragma unroll
    for (u32 k = 0; k < VT; ++k) {
        const u32 p = tid * VT + k;
        if (p < tot_cnt) {
            s.obeg[p] = dpos;
            dpos += s.payload[p];
        }
    }
    // positions in the next delta: look-back on both columns, one warp each
    if (tile == 0) {
        if (tid == 0) {
            st_relaxed_u64(lb_cnt, lb_word(kStatusInc, epoch, tot_cnt));
            st_relaxed_u64(lb_deg, lb_word(kStatusInc, epoch, tot_deg));
            s.base_cnt = 0;
            s.base_deg = 0;
        }
    } else {
        if (tid == 0) {
            st_relaxed_u64(lb_cnt + tile, lb_word(kStatusAgg, epoch, tot_cnt));
            st_relaxed_u64(lb_deg + tile, lb_word(kStatusAgg, epoch, tot_deg));
        }
        if (warp < 2) {
            u64 *lb = warp == 0 ? lb_cnt : lb_deg;
            const u64 mytot = warp == 0 ? (u64) tot_cnt : tot_deg;
            const u64 ex = lookback_warp(lb, tile, epoch, err);
            if (lane == 0) {
                st_relaxed_u64(lb + tile, lb_word(kStatusInc, epoch, ex + mytot));
                if (warp == 0) s.base_cnt = ex;
                else s.base_deg = ex;
            }
        }
    }
    __syncthreads();
    const u64 bc = s.base_cnt, bd = s.base_deg;
    if (tile == ntiles - 1 && tid == 0) {
        totals[0] = bc + tot_cnt;
        totals[1] = bd + tot_deg;
    }
    for (u32 i = tid; i < tot_cnt; i += JN_THREADS) {
        if (bc + i < capacity) {
            out[bc + i] = s.begin[i];
            out_offsets[bc + i] = bd + s.obeg[i];
        } else {
            atomicOr(err, DL_DEVERR_CAPACITY);  // more new tuples than join outputs: reported, never written
        }
    }
}

// Lane l gets the word whose bit b is bit l of lane b's word (32 x 32 bit
// transpose by recursive block swaps: each stage exchanges bit j of the row
// index with bit j of the column index).
__device__ __forceinline__ u32 transpose32(u32 v, u32 lane) {
    const u32 masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const int j = 16 >> s;
        const u32 mk = masks[s];
        const u32 u = __shfl_xor_sync(0xffffffffu, v, j);
        v = (lane & j) ? ((v & ~mk) | ((u >> j) & mk)) : ((v & mk) | ((u & mk) << j));
    }
    return v;
}

// t = transpose of a (both n rows of `stride` words). A tile is 256 source
// rows x 512 columns; the 512 target rows each receive 8 words (32 bytes).
__global__ void __launch_bounds__(256) bitmat_transpose_kernel(const u32 *__restrict__ a, u32 *__restrict__ t, u64 n,
                                                               u64 stride) {
    __shared__ u32 in[TR_ROWS][TR_WORDS + 1];
    __shared__ u32 outw[TR_WORDS * 32][TR_ROWS / 32 + 1];
    const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const u64 x0 = (u64) blockIdx.y * TR_ROWS;
    const u64 c0 = (u64) blockIdx.x * TR_WORDS;
    for (u32 i = tid; i < TR_ROWS * TR_WORDS; i += 256) {
        const u32 r = i / TR_WORDS, c = i % TR_WORDS;
        const u64 x = x0 + r, col = c0 + c;
        in[r][c] = (x < n && col < stride) ? a[x * stride + col] : 0u;
    }
    __syncthreads();
    // warp w transposes source rows w*32 .. w*32+31 (target word w of the tile)
#pragma unroll 4
    for (u32 c = 0; c < TR_WORDS; ++c) outw[c * 32 + lane][warp] = transpose32(in[warp * 32 + lane][c], lane);
    __syncthreads();
    for (u32 i = tid; i < TR_WORDS * 32 * (TR_ROWS / 32); i += 256) {
        const u32 r = i / (TR_ROWS / 32), xw = i % (TR_ROWS / 32);
        const u64 w = c0 * 32 + r, col = x0 / 32 + xw;
        if (w < n && col < stride) t[w * stride + col] = outw[r][xw];
    }
}

// counts[w] = set bits among the first `words` words of row w (warp per row).
__global__ void bitmat_row_count_kernel(const u32 *__restrict__ t, u64 n, u64 stride, u64 words, u64 *__restrict__ counts) {
    const u32 lane = threadIdx.x & 31;
    const u64 warps = (u64) gridDim.x * (blockDim.x / 32);
    for (u64 w = ((u64) blockIdx.x * blockDim.x + threadIdx.x) / 32; w < n; w += warps) {
        const u32 *row = t + w * stride;
        u32 c = 0;
        for (u64 k = lane; k < words; k += 32) c += __popc(__ldcs(row + k));
        c = warp_sum(c);
        if (lane == 0) counts[w] = c;
    }
}

// Row w of t -> words (w << bits) | x for its set bits x, ascending, from
// out[first[w]] on (warp per row).
__global__ void bitmat_extract_kernel(const u32 *__restrict__ t, u64 n, u64 stride, u64 words, int bits,
                                      const u64 *__restrict__ first, u64 *__restrict__ out) {
    const u32 lane = threadIdx.x & 31;
    const u64 warps = (u64) gridDim.x * (blockDim.x / 32);
    for (u64 w = ((u64) blockIdx.x * blockDim.x + threadIdx.x) / 32; w < n; w += warps) {
        const u32 *row = t + w * stride;
        u64 pos = first[w];
        const u64 hi = w << bits;
        for (u64 k0 = 0; k0 < words; k0 += 32) {
            const u64 k = k0 + lane;
            u32 v = k < words ? __ldcs(row + k) : 0u;
            const u32 c = __popc(v);
            // exclusive prefix of the lanes' counts
            u32 incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const u32 y = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= (u32) d) incl += y;
            }
            const u32 sum = __shfl_sync(0xffffffffu, incl, 31);
            u64 p = pos + (incl - c);
            while (v) {
                const int b = __ffs(v) - 1;
                v &= v - 1;
                out[p++] = hi | (k * 32 + (u64) b);
            }
            pos += sum;
        }
    }
}

struct CountValue {
    const u64 *v;
    __device__ __forceinline__ u64 operator()(u64 i) const { return v[i]; }
};

// out[i] = sum of in[0..i); returns the total.
u64 exclusive_scan(Context &ctx, const u64 *in, u64 n, u64 *out) {
    if (n == 0) return 0;
    const u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    u64 *lb = ctx.lookback_words(tiles);
    u32 *ctr = ctx.tile_counter(62);
    u64 *tot = &ctx.ctrl->scalar[49];
    DL_CUDA(cudaMemsetAsync(ctr, 0, sizeof(u32), ctx.stream));
    DL_LAUNCH(ctx, K_BITMAP_EXTRACT, 16.0 * n,
              scan_kernel<CountValue><<<(unsigned) tiles, SCAN_THREADS, 0, ctx.stream>>>(
                  CountValue{in}, n, out, lb, ctr, ctx.next_epoch(), &ctx.ctrl->err, tot));
    DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, tot, sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    return ctx.host_scalars[0];
}

}  // namespace

u64 bitmat_stride(u64 n) { return ((n + 31) / 32 + 31) / 32 * 32; }
u64 bitmat_bytes(u64 n) { return n * bitmat_stride(n) * 4; }

bool bitmat_choose(Context &ctx, const dl_options &opt, u64 n) {
    if (opt.dedup != DL_DEDUP_AUTO && opt.dedup != DL_DEDUP_BITMAP) return false;
    const u64 need = 2 * bitmat_bytes(n);
    size_t free_b = 0, total_b = 0;
    DL_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const u64 held = ctx.ws.bitmat[0].cap + ctx.ws.bitmat[1].cap;
    const u64 avail = (u64) free_b + held;
    if (opt.dedup == DL_DEDUP_BITMAP) {
        if (need > avail)
            throw Error(DL_ERR_OUT_OF_MEMORY, "bitmap dedup needs " + std::to_string(need) + " bytes for " +
                                                  std::to_string(n) + " nodes; " + std::to_string(avail) +
                                                  " available");
        return true;
    }
    return need <= ((u64) ctx.tune.bitmap_max_gib << 30) && need <= avail / 2;
}

u64 tc_bitmap_fixpoint(Context &ctx, Run &r, const Graph &g, const u64 *edges, u64 ne, const dl_options &opt,
                       PhaseTimer &pt) {
    Workspace &ws = ctx.ws;
    const u64 n = g.n_ids;
    const u64 stride = bitmat_stride(n);
    const u64 words_used = (n + 31) / 32;
    DevBuf &M = ws.bitmat[0];
    ctx.reserve(M, std::max<u64>(bitmat_bytes(n), 4));
    DL_CUDA(cudaMemsetAsync(M.p, 0, bitmat_bytes(n), ctx.stream));
    u32 *m = M.as<u32>();
    // delta_0 = the edges, source-major
    ctx.reserve(ws.jbuf[0], std::max<u64>(ne, 1) * 8);
    u64 *delta = ws.jbuf[0].as<u64>();
    u64 ndelta = ne;
    if (ne) {
        DL_LAUNCH(ctx, K_PREP, 16.0 * ne,
                  swap_fields_kernel<<<grid_for(ne, T256, ctx), T256, 0, ctx.stream>>>(edges, ne, g.bits, delta));
        DL_LAUNCH(ctx, K_BITMAP_EXPAND, 16.0 * ne,
                  bitmat_set_kernel<<<grid_for(ne, T256, ctx), T256, 0, ctx.stream>>>(delta, ne, g.bits, m, stride));
    }
    u64 nfull = ne;
    // join offsets of delta_0; later deltas get theirs from the step kernel
    pt.mark(PH_JOIN);
    ctx.reserve(ws.offsets, std::max<u64>(ndelta, 1) * 8);
    u64 total = ne ? join_count(ctx, g.csr, delta, ndelta, g.bits, ws.offsets.as<u64>()) : 0;
    u64 *totals = &ctx.ctrl->scalar[50];
    const CsrSrc<EmitKind::ZV> src{g.csr.off, g.csr.val, nullptr, g.bits};
    auto kern = bitmat_step_kernel;
    DL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sizeof(StepSmem)));
    for (int it = 0; ne > 0; ++it) {  // tc.cu:216-314
        pt.mark(PH_JOIN);
        ctx.run_join_total += total;
        ctx.run_join_max = std::max(ctx.run_join_max, total);
        DevBuf &nbuf = other(ws, delta);
        ctx.reserve(nbuf, std::max<u64>(total, 1) * 8);
        ctx.reserve(ws.offsets_next, std::max<u64>(total, 1) * 8);
        u64 nnew = 0, next_total = 0;
        if (total) {
            pt.mark(PH_DEDUP);
            const u64 tiles = (ndelta + total + JN_TILE - 1) / JN_TILE;
            ctx.lbs_splits.reserve((tiles + 1) * sizeof(u64));
            u64 *splits = ctx.lbs_splits.as<u64>();
            DL_LAUNCH(ctx, K_JOIN_PARTITION, 0,
                      lbs_partition_kernel<<<(unsigned) ((tiles + 1 + 255) / 256), 256, 0, ctx.stream>>>(
                          ws.offsets.as<u64>(), ndelta, total, tiles + 1, splits));
            u64 *lb = ctx.lookback_words(2 * tiles);
            u32 *ctr = ctx.tile_counter(63);
            DL_CUDA(cudaMemsetAsync(ctr, 0, sizeof(u32), ctx.stream));
            CsrSrc<EmitKind::ZV> sv = src;
            sv.probe = delta;
            DL_LAUNCH(ctx, K_BITMAP_EXPAND, 16.0 * ndelta + 12.0 * total,
                      kern<<<(unsigned) tiles, JN_THREADS, sizeof(StepSmem), ctx.stream>>>(
                          sv, ndelta, ws.offsets.as<u64>(), total, splits, m, stride, nbuf.as<u64>(),
                          ws.offsets_next.as<u64>(), total, lb, lb + tiles, ctr, ctx.next_epoch(), (u32) tiles,
                          &ctx.ctrl->err, totals));
            DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, totals, 2 * sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
            ctx.sync();
            nnew = ctx.host_scalars[0];
            next_total = ctx.host_scalars[1];
            ctx.prof_add_bytes(K_BITMAP_EXPAND, 16.0 * nnew);
        }
        pt.mark(PH_MERGE);
        nfull += nnew;
        r.deltas.push_back((i64) nnew);
        r.joins.push_back((i64) total);
        r.fulls.push_back((i64) nfull);
        delta = nbuf.as<u64>();
        ndelta = nnew;
        total = next_total;
        std::swap(ws.offsets, ws.offsets_next);
        if (nnew == 0) break;  // |full| unchanged
        if (opt.max_iterations > 0 && it + 1 >= opt.max_iterations) break;
    }
    pt.mark(PH_FINAL);
    // full -> sorted (w << bits) | x words in ws.full[0]
    ctx.reserve(ws.full[0], std::max<u64>(nfull, 1) * 8);
    if (nfull) {
        DevBuf &T = ws.bitmat[1];
        ctx.reserve(T, bitmat_bytes(n));
        const dim3 tg((unsigned) (stride / TR_WORDS), (unsigned) ((n + TR_ROWS - 1) / TR_ROWS));
        DL_LAUNCH(ctx, K_BITMAP_EXTRACT, 2.0 * bitmat_bytes(n),
                  bitmat_transpose_kernel<<<tg, 256, 0, ctx.stream>>>(m, T.as<u32>(), n, stride));
        ctx.reserve(ws.offsets, (n + 1) * 8);
        u64 *counts = ws.offsets.as<u64>();
        ctx.reserve(ws.w0, (n + 1) * 8);
        u64 *first = ws.w0.as<u64>();
        const unsigned rg = grid_for(n * 32, T256, ctx, 8);
        DL_LAUNCH(ctx, K_BITMAP_EXTRACT, 4.0 * n * words_used,
                  bitmat_row_count_kernel<<<rg, T256, 0, ctx.stream>>>(T.as<u32>(), n, stride, words_used, counts));
        const u64 total = exclusive_scan(ctx, counts, n, first);
        if (total != nfull)
            throw Error(DL_ERR_INTERNAL, "bit matrix holds " + std::to_string(total) + " tuples, expected " +
                                             std::to_string(nfull));
        DL_LAUNCH(ctx, K_BITMAP_EXTRACT, 4.0 * n * words_used + 8.0 * nfull,
                  bitmat_extract_kernel<<<rg, T256, 0, ctx.stream>>>(T.as<u32>(), n, stride, words_used, g.bits, first,
                                                                     ws.full[0].as<u64>()));
    }
    return nfull;
}

}  // namespace detail
}  // namespace dl
