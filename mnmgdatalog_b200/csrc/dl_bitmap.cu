// TC with the full relation held as a bit matrix over node ranks.
//
// The reference deduplicates each iteration's join output by sorting it,
// subtracting the sorted full relation and merging the difference back in
// (tc.cu:250-286). Here, when n x n bits fit in device memory (n = distinct
// node ids; 12.6 GB for 317K nodes), full is a bit matrix M with one row per
// path source x and one column per path target w, and dedup(J) \ full and
// full u J are one operation: a join tuple (x, w) is new exactly when its bit
// goes from 0 to 1. The delta is the same set as the reference's (every new
// bit is claimed by exactly one atomic on M), so per-iteration |delta| and the
// fixpoint are identical. The result leaves as sorted (target, source) words
// -- the reference's output order (tc.cu:345-366) -- through a bit-matrix
// transpose, row popcounts, a scan and an extraction pass.
//
// A delta is kept as units: one source x and a run of path targets y (u32,
// at most `unit_rows` of them; Tuning::bitmap_unit_rows, default 65,536: a
// unit costs one fold of the whole row, so fewer, larger units are cheaper).
// Almost all join output of a TC iteration belongs to a few heavy
// (x, iteration) pairs, so a CTA takes a unit, ORs
// the join words (x, w) for every edge y -> w into a shared-memory copy of
// row x, and then folds that row into M with one atomicOr per touched word
// (consecutive words: coalesced), instead of one global atomic per join word.
// The new bits of the unit are its part of the next delta: all of them count
// in |delta|, and those whose target has out-edges (the only ones that can
// join next step) become its rows.
#include "dl_engine_detail.h"
#include "dl_join.cuh"

namespace dl {
namespace detail {
namespace {

constexpr int TR_ROWS = 512;  // source rows per transpose tile
constexpr int TR_WORDS = 16;  // source words (512 columns) per transpose tile
constexpr int UT = 512;       // threads of the unit kernel

// One source x and delta rows rows[start, start + len): paths x -> rows[i].
struct Unit {
    u32 x;
    u32 len;
    u64 start;
};

// Sorted (x << bits) | y edge words -> bit (x, y) of the matrix.
__global__ void bitmat_set_edges_kernel(const u64 *__restrict__ words, u64 n, int bits, u32 *__restrict__ m,
                                        u64 stride) {
    const u64 mask = (1ull << bits) - 1;
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64) gridDim.x * blockDim.x) {
        const u64 v = words[i];
        const u64 x = v >> bits, y = v & mask;
        atomicOr(&m[x * stride + (y >> 5)], 1u << (y & 31));
    }
}

// Units of the first delta (the edges, from the CSR): per[x] = units of x.
__global__ void units_per_source_kernel(const u32 *__restrict__ off, u64 n, u64 unit_rows, u64 *__restrict__ per) {
    for (u64 x = (u64) blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (u64) gridDim.x * blockDim.x)
        per[x] = ((u64) (off[x + 1] - off[x]) + unit_rows - 1) / unit_rows;
}

__global__ void units_fill_kernel(const u32 *__restrict__ off, u64 n, u64 unit_rows, const u64 *__restrict__ first,
                                  Unit *__restrict__ units) {
    for (u64 x = (u64) blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (u64) gridDim.x * blockDim.x) {
        const u64 b = off[x], e = off[x + 1];
        u64 k = first[x];
        for (u64 s = b; s < e; s += unit_rows) units[k++] = Unit{(u32) x, (u32) min(unit_rows, e - s), s};
    }
}

// sum over edges of the target's out-degree: the first join's size.
__global__ void edge_degree_sum_kernel(const u32 *__restrict__ off, const u32 *__restrict__ val, u64 ne,
                                       unsigned long long *__restrict__ sum) {
    u64 s = 0;
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += (u64) gridDim.x * blockDim.x) {
        const u32 y = val[i];
        s += off[y + 1] - off[y];
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(sum, (unsigned long long) s);
}

constexpr int UW = UT / 32;   // warps of the unit kernel
constexpr u32 SCHUNK = 8;     // summary words per warp chunk in the fold and emit phases

struct UnitSmem {
    u32 wbeg[UW][32];   // per-warp compacted rows: first edge
    u32 wdeg[UW][32];   // and degree
    u32 wrows[UW];      // per-warp new rows of the unit (fold phase)
    u32 wbits[UW];      // per-warp new bits of the unit
    u32 unit;
    u32 next_group;
    unsigned long long obase;
    // followed by: u32 row[words], u32 summ[swords]
};

// Counters of one step (device, zeroed before the launch).
struct StepCounters {
    unsigned long long fetch;   // next unit to take
    unsigned long long words;   // new tuples (next delta rows)
    unsigned long long join;    // join size of the next step
    unsigned long long units;   // units of the next delta
    unsigned long long fresh;   // new tuples (|delta|; rows are written only for targets with out-edges)
};

// hasout[k] bit b = node 32 k + b has out-edges (only those can join next step).
__global__ void hasout_kernel(const u32 *__restrict__ off, u64 n, u64 words, u32 *__restrict__ hasout) {
    for (u64 k = (u64) blockIdx.x * blockDim.x + threadIdx.x; k < words; k += (u64) gridDim.x * blockDim.x) {
        u32 v = 0;
        for (u32 b = 0; b < 32; ++b) {
            const u64 x = k * 32 + b;
            if (x < n && off[x + 1] > off[x]) v |= 1u << b;
        }
        hasout[k] = v;
    }
}

// Next row group of the unit for this warp (lane 0 takes it, all lanes get it).
__device__ __forceinline__ u32 take_group(UnitSmem &s, u32 lane) {
    u32 g = 0;
    if (lane == 0) g = atomicAdd(&s.next_group, 1u);
    return __shfl_sync(0xffffffffu, g, 0);
}

// One semi-naive TC step over the units of a delta (persistent CTAs).
//
// Per unit (source x, delta rows y): every join word (x, w), w an edge target
// of a row y, is ORed into a shared-memory copy of row x; a summary bit per
// 32 row words records which words were touched (set by the lane that first
// touches a word). The fold then visits only touched words: one atomicOr
// (with return) on the matrix per word, coalesced over 32 consecutive words;
// new bits = row & ~old, and those whose target has out-edges become rows of
// the next delta. The emit visits only words with such rows and writes them
// warp-cooperatively (one ballot per non-zero word, consecutive positions).
// Phases are separated by four CTA barriers per unit.
__global__ void __launch_bounds__(UT, 4)
bitmat_unit_step_kernel(const u32 *__restrict__ off, const u32 *__restrict__ val, const u32 *__restrict__ rows,
                        const Unit *__restrict__ units, u64 nunits, u32 *__restrict__ m, u64 stride, u32 words,
                        u32 *__restrict__ out, u64 out_cap, Unit *__restrict__ uout, u64 uout_cap, u64 unit_rows,
                        const u32 *__restrict__ hasout, StepCounters *__restrict__ ctr, u32 *err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    UnitSmem &s = *reinterpret_cast<UnitSmem *>(smem_raw);
    u32 *row = reinterpret_cast<u32 *>(smem_raw + sizeof(UnitSmem));
    const u32 swords = (words + 31) / 32;
    u32 *summ = row + words;
    const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const u32 lt = lanemask_lt();
    const u32 le = lane == 31 ? ~0u : (2u << lane) - 1;  // lanes <= lane
    const u32 nchunks = (swords + SCHUNK - 1) / SCHUNK;
    for (u32 k = tid; k < words + swords; k += UT) row[k] = 0;
    if (tid == 0) s.next_group = 0;
    for (;;) {
        if (tid == 0) s.unit = (u32) min((unsigned long long) nunits, atomicAdd(&ctr->fetch, 1ull));
        __syncthreads();  // (1) unit taken; row, summary and group counter are clear
        const u64 ui = s.unit;
        if (ui >= nunits) break;
        const Unit U = units[ui];
        // ---- join words (x, w) of the unit into the shared row ----
        // Warps take groups of 32 rows; the next group's rows are loaded while
        // the current one is expanded, 32 join words at a time (the rows
        // starting in a window are a bit mask; a word's row is the number of
        // rows started up to its position), with the next window's edge-target
        // load in flight before the current window's shared-memory atomics.
        u32 grp = take_group(s, lane);
        u32 ny = 0;
        if (grp * 32 + lane < U.len) ny = rows[U.start + grp * 32 + lane];
        while (grp * 32 < U.len) {
            const u32 r = grp * 32 + lane;
            u32 beg = 0, deg = 0;
            if (r < U.len) {
                beg = __ldg(off + ny);
                deg = __ldg(off + ny + 1) - beg;
            }
            const u32 ngrp = take_group(s, lane);
            if (ngrp * 32 + lane < U.len) ny = rows[U.start + ngrp * 32 + lane];
            const u32 nz = __ballot_sync(0xffffffffu, deg != 0);
            if (nz) {
                if (deg) {
                    const u32 rk = __popc(nz & lt);
                    s.wbeg[warp][rk] = beg;
                    s.wdeg[warp][rk] = deg;
                }
                __syncwarp();
                const u32 nrows = __popc(nz);
                beg = lane < nrows ? s.wbeg[warp][lane] : 0u;
                deg = lane < nrows ? s.wdeg[warp][lane] : 0u;
                __syncwarp();
                const u32 incl = warp_inclusive_sum(deg);
                const u32 pre = incl - deg;
                const u32 total = __shfl_sync(0xffffffffu, incl, 31);
                int base = -1;  // last row started before the window
                // edge-target address of this lane's word of window i0
                auto addr = [&](u32 i0) -> u32 {
                    const u32 st = (deg && pre >= i0 && pre < i0 + 32) ? 1u << (pre - i0) : 0u;
                    const u32 starts = __reduce_or_sync(0xffffffffu, st);
                    const int o = base + __popc(starts & le);
                    base += __popc(starts);
                    const u32 ob = __shfl_sync(0xffffffffu, beg, o);
                    const u32 op = __shfl_sync(0xffffffffu, pre, o);
                    return ob + (i0 + lane - op);
                };
                const u32 a0 = addr(0);  // warp-collective: every lane calls it
                u32 w = lane < total ? __ldg(val + a0) : 0u;
                for (u32 i0 = 0; i0 < total; i0 += 32) {
                    const bool have = i0 + lane < total;
                    u32 wn = 0;
                    if (i0 + 32 < total) {
                        const u32 a = addr(i0 + 32);
                        if (i0 + 32 + lane < total) wn = __ldg(val + a);
                    }
                    if (have) {
                        const u32 old = atomicOr(&row[w >> 5], 1u << (w & 31));
                        if (old == 0) atomicOr(&summ[w >> 10], 1u << ((w >> 5) & 31));
                    }
                    w = wn;
                }
            }
            grp = ngrp;
        }
        __syncthreads();  // (2) the row is complete
        // ---- fold the touched words into M: new bits = row & ~M ----
        // Every new bit counts in |delta|; only targets with out-edges become
        // rows of the next delta. Warp w takes summary chunks w, w + UW, ...
        const u64 mrow = (u64) U.x * stride;
        u32 nrows_w = 0, nbits_w = 0;
        for (u32 c = warp; c < nchunks; c += UW) {
            const u32 sw0 = c * SCHUNK;
            const u32 sv = (lane < SCHUNK && sw0 + lane < swords) ? summ[sw0 + lane] : 0u;
            u32 todo = __ballot_sync(0xffffffffu, sv != 0);
            while (todo) {
                // up to two summary words at once: both matrix atomics in flight
                const u32 j0 = __ffs(todo) - 1;
                todo &= todo - 1;
                const u32 j1 = todo ? __ffs(todo) - 1 : 32u;
                if (todo) todo &= todo - 1;
                const u32 s0 = __shfl_sync(0xffffffffu, sv, j0);
                const u32 s1 = __shfl_sync(0xffffffffu, sv, j1 & 31);
                const bool a0 = (s0 >> lane) & 1, a1 = j1 < 32 && ((s1 >> lane) & 1);
                const u32 k0 = (sw0 + j0) * 32 + lane, k1 = (sw0 + (j1 & 31)) * 32 + lane;
                const u32 v0 = a0 ? row[k0] : 0u, v1 = a1 ? row[k1] : 0u;
                const u32 o0 = a0 ? atomicOr(&m[mrow + k0], v0) : ~0u;
                const u32 o1 = a1 ? atomicOr(&m[mrow + k1], v1) : ~0u;
                const u32 h0 = a0 ? __ldg(hasout + k0) : 0u, h1 = a1 ? __ldg(hasout + k1) : 0u;
                const u32 f0 = v0 & ~o0, f1 = v1 & ~o1;
                const u32 r0 = f0 & h0, r1 = f1 & h1;
                if (a0) row[k0] = r0;
                if (a1) row[k1] = r1;
                nbits_w += __popc(f0) + __popc(f1);
                nrows_w += __popc(r0) + __popc(r1);
                const u32 m0 = __ballot_sync(0xffffffffu, r0 != 0);
                const u32 m1 = __ballot_sync(0xffffffffu, r1 != 0);
                if (lane == 0) {
                    summ[sw0 + j0] = m0;  // summary now marks words with new rows
                    if (j1 < 32) summ[sw0 + j1] = m1;
                }
            }
        }
        nrows_w = warp_sum(nrows_w);
        nbits_w = warp_sum(nbits_w);
        if (lane == 0) {
            s.wrows[warp] = nrows_w;
            s.wbits[warp] = nbits_w;
        }
        __syncthreads();  // (3) per-warp counts
        const u32 cw = lane < UW ? s.wrows[lane] : 0u;
        const u32 bw = lane < UW ? s.wbits[lane] : 0u;
        const u32 cinc = warp_inclusive_sum(cw);
        const u32 total = __shfl_sync(0xffffffffu, cinc, 31);
        const u32 before = __shfl_sync(0xffffffffu, cinc - cw, warp);  // new rows of lower warps
        const u32 fresh = warp_sum(bw);
        if (tid == 0) {
            s.obase = total ? atomicAdd(&ctr->words, (unsigned long long) total) : 0ull;
            if (fresh) atomicAdd(&ctr->fresh, (unsigned long long) fresh);
        }
        __syncthreads();  // (4) the unit's place in the next delta
        const u64 obase = s.obase;
        // ---- emit the new rows (targets of x) and clear the row ----
        // New bits are sparse within a word, so each lane walks its own word.
        u64 p = obase + before;
        u64 dsum = 0;
        for (u32 c = warp; c < nchunks; c += UW) {
            const u32 sw0 = c * SCHUNK;
            const u32 sv = (lane < SCHUNK && sw0 + lane < swords) ? summ[sw0 + lane] : 0u;
            if (lane < SCHUNK && sw0 + lane < swords && sv) summ[sw0 + lane] = 0;
            u32 todo = __ballot_sync(0xffffffffu, sv != 0);
            while (todo) {
                const u32 j = __ffs(todo) - 1;
                todo &= todo - 1;
                const u32 sj = __shfl_sync(0xffffffffu, sv, j);
                const u32 kb = (sw0 + j) * 32;
                u32 fr = 0;
                if ((sj >> lane) & 1) {
                    fr = row[kb + lane];
                    row[kb + lane] = 0;
                }
                const u32 cnt = __popc(fr);
                const u32 incl = warp_inclusive_sum(cnt);
                u64 q = p + (incl - cnt);
                while (fr) {
                    const u32 t = (kb + lane) * 32 + (__ffs(fr) - 1);
                    fr &= fr - 1;
                    if (q < out_cap) out[q] = t;
                    else atomicOr(err, DL_DEVERR_CAPACITY);  // more new tuples than join words: reported
                    ++q;
                    dsum += __ldg(off + t + 1) - __ldg(off + t);
                }
                p += __shfl_sync(0xffffffffu, incl, 31);
            }
        }
        // rows of the row words untouched by the fold are already zero; the
        // touched ones were zeroed in the fold (no new rows) or just now
        dsum = warp_sum(dsum);
        if (lane == 0 && dsum) atomicAdd(&ctr->join, (unsigned long long) dsum);
        if (warp == 0 && total) {
            const u64 nsub = (total + unit_rows - 1) / unit_rows;
            u64 ub = 0;
            if (lane == 0) ub = atomicAdd(&ctr->units, (unsigned long long) nsub);
            ub = __shfl_sync(0xffffffffu, ub, 0);
            for (u64 i = lane; i < nsub; i += 32) {
                if (ub + i < uout_cap)
                    uout[ub + i] = Unit{U.x, (u32) min(unit_rows, total - i * unit_rows), obase + i * unit_rows};
                else
                    atomicOr(err, DL_DEVERR_CAPACITY);
            }
        }
        if (tid == 0) s.next_group = 0;  // read again only after barrier (1)
    }
}

// Lane l gets the word whose bit b is bit l of lane b's word (32 x 32 bit
// transpose by recursive block swaps: each stage exchanges bit j of the row
// index with bit j of the column index). The 16- and 8-bit stages move whole
// bytes, so one byte permute does each.
__device__ __forceinline__ u32 transpose32(u32 v, u32 lane) {
    u32 u = __shfl_xor_sync(0xffffffffu, v, 16);
    v = __byte_perm(v, u, (lane & 16) ? 0x3276 : 0x5410);
    u = __shfl_xor_sync(0xffffffffu, v, 8);
    v = __byte_perm(v, u, (lane & 8) ? 0x3715 : 0x6240);
    const u32 masks[3] = {0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        const int j = 4 >> s;
        const u32 mk = masks[s];
        u = __shfl_xor_sync(0xffffffffu, v, j);
        v = (lane & j) ? ((v & ~mk) | ((u >> j) & mk)) : ((v & mk) | ((u & mk) << j));
    }
    return v;
}

__device__ __forceinline__ void cp_async4(u32 *dst, const u32 *src) {
    const unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// t = transpose of a (both n rows of `stride` words), and counts[w] += set
// bits of target row w. A tile is 512 source rows x 512 columns: 64 bytes
// read from every source row and 64 bytes written to every target row. CTA
// (c, g) walks the tiles of column block c (targets 512 c ...) for source
// blocks g, g + G, ...; the next tile is copied into shared memory (cp.async,
// two buffers) while the current one is transposed and stored. Thread i keeps
// the popcount of target row 512 c + i over its tiles and adds it to counts
// once at the end (G atomics per row).
constexpr int TR_PAD = TR_WORDS + 1;
constexpr int TR_SMEM = 3 * TR_ROWS * TR_PAD * 4;  // two input tiles + the transposed tile
__global__ void __launch_bounds__(TR_ROWS, 2) bitmat_transpose_count_kernel(const u32 *__restrict__ a,
                                                                            u32 *__restrict__ t, u64 n, u64 stride,
                                                                            unsigned long long *__restrict__ counts) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u32(*in)[TR_ROWS][TR_PAD] = reinterpret_cast<u32(*)[TR_ROWS][TR_PAD]>(smem_raw);
    u32(*outw)[TR_ROWS / 32 + 1] = reinterpret_cast<u32(*)[TR_ROWS / 32 + 1]>(smem_raw + 2 * TR_ROWS * TR_PAD * 4);
    static_assert(TR_WORDS * 32 == TR_ROWS && TR_ROWS / 32 == TR_WORDS, "square tile: 512 x 512 bits");
    const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const u64 c0 = (u64) blockIdx.x * TR_WORDS;  // first column word of the block
    const u64 nblocks = (n + TR_ROWS - 1) / TR_ROWS;
    auto issue = [&](u64 b, int buf) {  // tile (b, c) -> in[buf]
        const u64 x0 = b * TR_ROWS;
#pragma unroll
        for (u32 j = 0; j < TR_WORDS; ++j) {
            const u32 i = tid + j * TR_ROWS, r = i / TR_WORDS, c = i % TR_WORDS;
            const u64 x = x0 + r, col = c0 + c;
            if (x < n && col < stride) cp_async4(&in[buf][r][c], a + x * stride + col);
            else in[buf][r][c] = 0u;
        }
    };
    u32 cnt = 0;  // set bits of target row c0 * 32 + tid in this CTA's tiles
    u64 b = blockIdx.y;
    int buf = 0;
    if (b < nblocks) issue(b, 0);
    cp_async_commit();
    for (; b < nblocks; b += gridDim.y, buf ^= 1) {
        // in[buf ^ 1] was last read by the previous tile's transpose, which
        // every thread finished before the barrier ahead of its stores
        if (b + gridDim.y < nblocks) issue(b + gridDim.y, buf ^ 1);
        cp_async_commit();
        cp_async_wait_prev();  // this thread's copies of tile b have landed
        __syncthreads();       // everyone's have
#pragma unroll 4
        for (u32 c = 0; c < TR_WORDS; ++c)
            outw[c * 32 + lane][warp] = transpose32(in[buf][warp * 32 + lane][c], lane);
        __syncthreads();
#pragma unroll
        for (u32 xw = 0; xw < TR_ROWS / 32; ++xw) cnt += __popc(outw[tid][xw]);
        const u64 x0 = b * TR_ROWS;
#pragma unroll 4
        for (u32 j = 0; j < TR_WORDS; ++j) {
            const u32 i = tid + j * TR_ROWS;
            const u32 r = i / (TR_ROWS / 32), xw = i % (TR_ROWS / 32);
            const u64 w = c0 * 32 + r, col = x0 / 32 + xw;
            if (w < n && col < stride) t[w * stride + col] = outw[r][xw];
        }
        // outw is rewritten only after the next iteration's first barrier
    }
    const u64 w = c0 * 32 + tid;
    if (w < n && cnt) atomicAdd(counts + w, (unsigned long long) cnt);
}

// Row w of t -> result rows (ids[x], ids[w]) for its set bits x, ascending,
// from out[first[w]] on: the reference's TC file order (x, z) sorted by
// (z, x). One warp per row; a lane takes 4 consecutive words per step (one
// 16-byte load, the next one in flight); a step's rows are staged in shared
// memory and leave with consecutive stores unless there are more than
// EX_STAGE of them. (Result words are sparse -- C1 averages well under one
// set bit per non-zero word -- so each lane walks its own words' bits.)
constexpr int EX_THREADS = 256;
constexpr int EX_STAGE = 256;
__global__ void __launch_bounds__(EX_THREADS) bitmat_extract_rows_kernel(const u32 *__restrict__ t, u64 n,
                                                                         u64 stride, u64 words,
                                                                         const u64 *__restrict__ first,
                                                                         const int32_t *__restrict__ ids,
                                                                         u64 *__restrict__ out) {
    __shared__ u64 stage[EX_THREADS / 32][EX_STAGE];
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u64 *st = stage[warp];
    const u64 warps = (u64) gridDim.x * (EX_THREADS / 32);
    for (u64 w = (u64) blockIdx.x * (EX_THREADS / 32) + warp; w < n; w += warps) {
        const u32 *row = t + w * stride;
        u64 pos = first[w];
        const u64 hi = (u64) (u32) ids[w] << 32;  // (x id, z id) as one little-endian 8-byte row
        // stride is a multiple of 32 words: a lane's vector stays in the row
        uint4 nxt = make_uint4(0, 0, 0, 0);
        if ((u64) lane * 4 < words) nxt = __ldcs(reinterpret_cast<const uint4 *>(row + lane * 4));
        for (u64 k0 = 0; k0 < words; k0 += 128) {
            const u64 k = k0 + lane * 4;
            const uint4 q = nxt;  // this step's words; the next step's load is in flight meanwhile
            nxt = make_uint4(0, 0, 0, 0);
            if (k + 128 < words) nxt = __ldcs(reinterpret_cast<const uint4 *>(row + k + 128));
            u32 v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (k + c >= words) v[c] = 0;  // past the used columns
            const u32 cnt = __popc(v[0]) + __popc(v[1]) + __popc(v[2]) + __popc(v[3]);
            const u32 incl = warp_inclusive_sum(cnt);
            const u32 sum = __shfl_sync(0xffffffffu, incl, 31);
            if (sum == 0) continue;
            u32 p = incl - cnt;
            if (sum <= EX_STAGE) {
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    for (u32 b = v[c]; b; b &= b - 1)
                        st[p++] = hi | (u32) __ldg(ids + (k + c) * 32 + (__ffs(b) - 1));
                __syncwarp();
                for (u32 i = lane; i < sum; i += 32) out[pos + i] = st[i];
                __syncwarp();
            } else {
                u64 q2 = pos + p;
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    for (u32 b = v[c]; b; b &= b - 1)
                        out[q2++] = hi | (u32) __ldg(ids + (k + c) * 32 + (__ffs(b) - 1));
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
    const u64 unit_rows = std::max<u64>(1, ctx.tune.bitmap_unit_rows);
    const u64 words_used = (n + 31) / 32;
    const size_t smem = sizeof(UnitSmem) + (words_used + (words_used + 31) / 32) * 4 + 16;
    if (smem > 227 * 1024) throw Error(DL_ERR_OUT_OF_MEMORY, "bit-matrix rows of " + std::to_string(n) +
                                                              " nodes do not fit in shared memory");
    DevBuf &M = ws.bitmat[0];
    ctx.reserve(M, std::max<u64>(bitmat_bytes(n), 4));
    DL_CUDA(cudaMemsetAsync(M.p, 0, bitmat_bytes(n), ctx.stream));
    u32 *m = M.as<u32>();
    StepCounters *ctr = reinterpret_cast<StepCounters *>(&ctx.ctrl->scalar[52]);
    // delta_0 = the edges: rows are the CSR's values, units from its offsets
    const u32 *rows = g.csr.val;
    u64 nunits = 0, join = 0;
    DevBuf *ubuf = &ws.offsets, *ubuf_next = &ws.offsets_next;
    if (ne) {
        DL_LAUNCH(ctx, K_BITMAP_EXPAND, 16.0 * ne,
                  bitmat_set_edges_kernel<<<grid_for(ne, T256, ctx), T256, 0, ctx.stream>>>(edges, ne, g.bits, m,
                                                                                            stride));
        ctx.reserve(ws.w0, (n + 1) * 8);
        ctx.reserve(ws.w1, (n + 1) * 8);
        DL_LAUNCH(ctx, K_PREP, 12.0 * n,
                  units_per_source_kernel<<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(g.csr.off, n, unit_rows,
                                                                                           ws.w0.as<u64>()));
        nunits = exclusive_scan(ctx, ws.w0.as<u64>(), n, ws.w1.as<u64>());
        ctx.reserve(*ubuf, std::max<u64>(nunits, 1) * sizeof(Unit));
        DL_LAUNCH(ctx, K_PREP, 16.0 * nunits,
                  units_fill_kernel<<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(g.csr.off, n, unit_rows, ws.w1.as<u64>(),
                                                                                     ubuf->as<Unit>()));
        DL_CUDA(cudaMemsetAsync(&ctr->join, 0, sizeof(u64), ctx.stream));
        DL_LAUNCH(ctx, K_PREP, 8.0 * ne,
                  edge_degree_sum_kernel<<<grid_for(ne, T256, ctx), T256, 0, ctx.stream>>>(g.csr.off, g.csr.val, ne,
                                                                                           &ctr->join));
        DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, &ctr->join, sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
        join = ctx.host_scalars[0];
    }
    ctx.reserve(ws.bit_hasout, std::max<u64>(words_used, 1) * 4);
    DL_LAUNCH(ctx, K_PREP, 4.0 * n + 4.0 * words_used,
              hasout_kernel<<<grid_for(words_used, T256, ctx), T256, 0, ctx.stream>>>(g.csr.off, n, words_used,
                                                                                      ws.bit_hasout.as<u32>()));
    u64 nfull = ne;
    u64 nrows = ne;  // rows of the current delta
    auto kern = bitmat_unit_step_kernel;
    DL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    int per_sm = 0;
    DL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, UT, smem));
    const u64 resident = (u64) ctx.sm_count * std::max(per_sm, 1);
    int slot = 0;
    for (int it = 0; ne > 0; ++it) {  // tc.cu:216-314
        pt.mark(PH_JOIN);
        ctx.run_join_total += join;
        ctx.run_join_max = std::max(ctx.run_join_max, join);
        u64 nnew = 0, next_join = 0, next_units = 0;
        if (join) {
            pt.mark(PH_DEDUP);
            DevBuf &obuf = ws.jbuf[slot];
            ctx.reserve(obuf, join * 4);
            const u64 ucap = nunits + join / unit_rows + 1;
            ctx.reserve(*ubuf_next, ucap * sizeof(Unit));
            DL_CUDA(cudaMemsetAsync(ctr, 0, sizeof(StepCounters), ctx.stream));
            const unsigned grid = (unsigned) std::min<u64>(nunits, resident);
            // algorithmic bytes: delta rows and units in, one edge target per join word, new rows and units out
            DL_LAUNCH(ctx, K_BITMAP_EXPAND, 4.0 * nrows + 16.0 * nunits + 4.0 * join,
                      kern<<<grid, UT, smem, ctx.stream>>>(g.csr.off, g.csr.val, rows, ubuf->as<Unit>(), nunits, m,
                                                           stride, (u32) words_used, obuf.as<u32>(), join,
                                                           ubuf_next->as<Unit>(), ucap, unit_rows,
                                                           ws.bit_hasout.as<u32>(), ctr, &ctx.ctrl->err));
            DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, ctr, sizeof(StepCounters), cudaMemcpyDeviceToHost, ctx.stream));
            ctx.sync();
            const u64 next_rows = ctx.host_scalars[1];
            next_join = ctx.host_scalars[2];
            next_units = ctx.host_scalars[3];
            nnew = ctx.host_scalars[4];
            ctx.prof_add_bytes(K_BITMAP_EXPAND, 4.0 * next_rows + 16.0 * next_units);
            rows = obuf.as<u32>();
            nrows = next_rows;
            slot ^= 1;
            std::swap(ubuf, ubuf_next);
        }
        pt.mark(PH_MERGE);
        nfull += nnew;
        r.deltas.push_back((i64) nnew);
        r.joins.push_back((i64) join);
        r.fulls.push_back((i64) nfull);
        nunits = next_units;
        join = next_join;
        if (nnew == 0) break;  // |full| unchanged
        if (opt.max_iterations > 0 && it + 1 >= opt.max_iterations) break;
    }
    pt.mark(PH_FINAL);
    // full -> its transpose (row = target) and per-target counts; the result
    // rows are extracted from it when they are copied out (bitmat_extract_rows)
    if (nfull) {
        DevBuf &T = ws.bitmat[1];
        ctx.reserve(T, bitmat_bytes(n));
        ctx.reserve(ws.offsets, (n + 1) * 8);
        u64 *counts = ws.offsets.as<u64>();
        DL_CUDA(cudaMemsetAsync(counts, 0, n * 8, ctx.stream));
        DL_CUDA(cudaFuncSetAttribute(bitmat_transpose_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TR_SMEM));
        int tr_per_sm = 0;
        DL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tr_per_sm, bitmat_transpose_count_kernel, TR_ROWS,
                                                              TR_SMEM));
        const u64 xblocks = stride / TR_WORDS, nblocks = (n + TR_ROWS - 1) / TR_ROWS;
        const u64 resident_tr = (u64) ctx.sm_count * std::max(tr_per_sm, 1);
        const u64 gy = std::min<u64>(nblocks, std::max<u64>(1, (8 * resident_tr + xblocks - 1) / xblocks));
        const dim3 tg((unsigned) xblocks, (unsigned) gy);
        DL_LAUNCH(ctx, K_BITMAP_TRANSPOSE, 2.0 * bitmat_bytes(n),
                  bitmat_transpose_count_kernel<<<tg, TR_ROWS, TR_SMEM, ctx.stream>>>(
                      m, T.as<u32>(), n, stride, reinterpret_cast<unsigned long long *>(counts)));
        ctx.reserve(ws.w0, (n + 1) * 8);
        u64 *first = ws.w0.as<u64>();
        const u64 total = exclusive_scan(ctx, counts, n, first);
        if (total != nfull)
            throw Error(DL_ERR_INTERNAL, "bit matrix holds " + std::to_string(total) + " tuples, expected " +
                                             std::to_string(nfull));
        r.bm_t = T;
        T = DevBuf();
        r.bm_first = ws.w0;
        ws.w0 = DevBuf();
        r.bm_n = n;
        r.bm_stride = stride;
        r.bm_words = words_used;
    }
    r.from_bitmat = true;
    return nfull;
}

}  // namespace detail

// The result rows of a bit-matrix TC run, written straight from the stored
// transpose into `out` (device memory): (x, z) rows ordered by (z, x).
void bitmat_extract_rows(Context &ctx, const Run &r, int32_t *out) {
    using namespace detail;
    if (r.info.output_rows == 0) return;
    const u64 n = r.bm_n;
    DL_LAUNCH(ctx, K_BITMAP_EXTRACT, 4.0 * n * r.bm_words + 8.0 * (double) r.info.output_rows,
              bitmat_extract_rows_kernel<<<grid_for(n * 32, EX_THREADS, ctx, 8), EX_THREADS, 0, ctx.stream>>>(
                  r.bm_t.as<u32>(), n, r.bm_stride, r.bm_words, r.bm_first.as<u64>(), r.ids.as<int32_t>(),
                  reinterpret_cast<u64 *>(out)));
}

}  // namespace dl
