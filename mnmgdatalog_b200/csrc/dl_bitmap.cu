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
// fixpoint are identical. The result rows leave in the reference's output
// order (tc.cu:345-366: by target, then source) from M's transpose, made by
// one pass over M that transposes 32 x 32 bit blocks in registers, or --
// when a second matrix does not fit -- straight from M's columns by a
// counting pass and a rows pass of the same kind.
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

constexpr int UT = 512;       // threads of the unit kernel

// One source x and delta rows rows[start, start + len): paths x -> y for
// the rows' targets y. A delta row holds the target's edge range (first edge,
// out-degree) rather than the target itself: that is all a join needs.
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

// Delta_0 rows: edge i (x -> y) as (off[y], deg y).
__global__ void edge_rows_kernel(const u32 *__restrict__ off, const u32 *__restrict__ val, u64 ne,
                                 uint2 *__restrict__ rows) {
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += (u64) gridDim.x * blockDim.x) {
        const u32 y = val[i];
        const u32 b = off[y];
        rows[i] = make_uint2(b, off[y + 1] - b);
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

constexpr int UW = UT / 32;      // warps of the unit kernel
constexpr u32 SCHUNK = 8;        // summary words per warp chunk in the fold and emit phases
constexpr u64 OCHUNK = 1 << 18;  // next-delta rows a CTA reserves at a time (a unit crossing the end of one is split)
constexpr u64 UCHUNK = 16;       // next-delta unit slots a CTA reserves at a time

// Shared memory of the expansion of a unit's rows into a shared row (NW warps).
template <int NW>
struct ExpandSmemT {
    u32 wbeg[NW][32];   // per-warp compacted rows: first edge
    u32 wdeg[NW][32];   // and degree
    u32 next_group;     // next row group to take
};
using ExpandSmem = ExpandSmemT<UW>;

struct UnitSmem {
    ExpandSmem e;
    u32 wrows[UW];      // per-warp new rows of the unit (fold phase)
    Unit cur;           // the unit being processed (len 0: none left)
    Unit next;          // the next one, fetched while the current one runs
    u64 ocur, oend;     // the CTA's reserved next-delta rows [ocur, oend)
    u64 ucur, uend;     // and unit slots
    u64 nbase;          // a fresh row reservation (when the unit does not fit the current one)
    u64 pend_ocur, pend_oend;  // thread 0: the row reservation after the current unit
    unsigned long long acc[UW][3];  // per warp: new tuples, next join size, rows written
    // followed by: u32 row[words], u32 summ[swords]
};

// Counters of one step (device, zeroed before the launch).
struct StepCounters {
    unsigned long long fetch;   // next unit slot to take
    unsigned long long words;   // next-delta rows reserved (rows + unused tails of CTA reservations)
    unsigned long long join;    // join size of the next step
    unsigned long long units;   // next-delta unit slots reserved (unused ones hold len = 0)
    unsigned long long fresh;   // new tuples (|delta|; rows are written only for targets with out-edges)
    unsigned long long rows;    // next-delta rows written
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
template <int NW>
__device__ __forceinline__ u32 take_group(ExpandSmemT<NW> &s, u32 lane) {
    u32 g = 0;
    if (lane == 0) g = atomicAdd(&s.next_group, 1u);
    return __shfl_sync(0xffffffffu, g, 0);
}

// Join words of unit U into the shared row: for every delta row (an edge
// range: first edge, degree), OR bit w into row[] for each edge target w, and
// when the word w / 32 goes from zero to non-zero, set summary bit w / 1024
// (LIST false) or append w / 32 to the touched-word list lk[*nlist] (LIST
// true; one shared-memory atomic per warp and window).
// Warps take groups of 32 rows; the next group's rows are loaded while the
// current one is expanded, 32 join words at a time (the rows starting in a
// window are a bit mask; a word's row is the number of rows started up to
// its position), with the next window's edge-target load in flight before
// the current window's shared-memory atomics. Called by every thread of the
// CTA; s.next_group must be zero.
template <bool LIST = false, int NW>
__device__ __forceinline__ void expand_unit(ExpandSmemT<NW> &s, u32 *row, u32 *summ, const uint2 *__restrict__ rows,
                                            const u32 *__restrict__ val, const Unit &U, u32 lane, u32 warp, u32 lt,
                                            u32 le, u32 *lk = nullptr, u32 *nlist = nullptr) {
    u32 grp = take_group(s, lane);
    uint2 cur = make_uint2(0, 0);
    if (grp * 32 + lane < U.len) cur = rows[U.start + grp * 32 + lane];
    while (grp * 32 < U.len) {
        const u32 grp1 = take_group(s, lane);
        uint2 nxt = make_uint2(0, 0);
        if (grp1 * 32 + lane < U.len) nxt = rows[U.start + grp1 * 32 + lane];
        const u32 beg = cur.x, deg = cur.y;
        const u32 nz = __ballot_sync(0xffffffffu, deg != 0);
        if (nz) {
            if (deg) {
                const u32 rk = __popc(nz & lt);
                s.wbeg[warp][rk] = beg;
                s.wdeg[warp][rk] = deg;
            }
            __syncwarp();
            const u32 nrows = __popc(nz);
            const u32 cb = lane < nrows ? s.wbeg[warp][lane] : 0u;
            const u32 cd = lane < nrows ? s.wdeg[warp][lane] : 0u;
            __syncwarp();
            const u32 incl = warp_inclusive_sum(cd);
            const u32 pre = incl - cd;
            const u32 total = __shfl_sync(0xffffffffu, incl, 31);
            int base = -1;  // last row started before the window
            // edge-target address of this lane's word of window i0
            auto addr = [&](u32 i0) -> u32 {
                const u32 st = (cd && pre >= i0 && pre < i0 + 32) ? 1u << (pre - i0) : 0u;
                const u32 starts = __reduce_or_sync(0xffffffffu, st);
                const int o = base + __popc(starts & le);
                base += __popc(starts);
                const u32 ob = __shfl_sync(0xffffffffu, cb, o);
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
                if constexpr (LIST) {
                    const bool first = have && atomicOr(&row[w >> 5], 1u << (w & 31)) == 0u;
                    const u32 fm = __ballot_sync(0xffffffffu, first);
                    if (fm) {
                        u32 at = 0;
                        if (lane == (u32) (__ffs(fm) - 1)) at = atomicAdd(nlist, (u32) __popc(fm));
                        at = __shfl_sync(0xffffffffu, at, __ffs(fm) - 1);
                        if (first) lk[at + __popc(fm & lt)] = w >> 5;
                    }
                } else if (have) {
                    const u32 old = atomicOr(&row[w >> 5], 1u << (w & 31));
                    if (old == 0) atomicOr(&summ[w >> 10], 1u << ((w >> 5) & 31));
                }
                w = wn;
            }
        }
        grp = grp1;
        cur = nxt;
    }
}

// The next non-empty unit from the shared queue (len 0: none left). Called by
// one thread.
__device__ __forceinline__ Unit fetch_unit(const Unit *__restrict__ units, u64 nunits, StepCounters *ctr) {
    for (;;) {
        const u64 i = atomicAdd(&ctr->fetch, 1ull);
        if (i >= nunits) return Unit{0, 0, 0};
        const Unit u = units[i];
        if (u.len) return u;
    }
}

// One semi-naive TC step over the units of a delta (persistent CTAs).
//
// Per unit (source x, delta rows y): every join word (x, w), w an edge target
// of a row y, is ORed into a shared-memory copy of row x; a summary bit per
// 32 row words records which words were touched (set by the lane that first
// touches a word). The fold then visits only touched words: one atomicOr
// (with return) on the matrix per word, coalesced over 32 consecutive words;
// new bits = row & ~old, and those whose target has out-edges become rows of
// the next delta, which the emit writes from the words that hold them.
//
// Latency is hidden rather than waited for: the next unit is fetched while
// the current one runs; each warp loads the next row group's rows and edge
// offsets while it expands the current group; next-delta rows and unit slots
// come from per-CTA reservations (a global atomic only when one runs out);
// counters are summed per thread and added once at the end. Three CTA
// barriers separate a unit's phases (a fourth only when a row reservation
// runs out).
__global__ void __launch_bounds__(UT, 4)
bitmat_unit_step_kernel(const u32 *__restrict__ off, const u32 *__restrict__ val, const uint2 *__restrict__ rows,
                        const Unit *__restrict__ units, u64 nunits, u32 *__restrict__ m, u64 stride, u32 words,
                        uint2 *__restrict__ out, u64 out_cap, Unit *__restrict__ uout, u64 uout_cap, u64 unit_rows,
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
    if (tid == 0) {
        s.e.next_group = 0;
        s.ocur = s.oend = s.ucur = s.uend = s.pend_ocur = s.pend_oend = 0;
        s.next = fetch_unit(units, nunits, ctr);
    }
    if (lane == 0) s.acc[warp][0] = s.acc[warp][1] = s.acc[warp][2] = 0;
    for (;;) {
        if (tid == 0) s.cur = s.next;
        __syncthreads();  // (1) unit known; row, summary and group counter are clear
        const Unit U = s.cur;
        if (U.len == 0) break;
        if (tid == 0) {
            // every thread read the previous unit's reservation before this
            // barrier; the new one is read after barrier (3)
            s.ocur = s.pend_ocur;
            s.oend = s.pend_oend;
            s.next = fetch_unit(units, nunits, ctr);  // read only at the next barrier (1)
        }
        // ---- join words (x, w) of the unit into the shared row ----
        expand_unit(s.e, row, summ, rows, val, U, lane, warp, lt, le);
        __syncthreads();  // (2) the row is complete
        // ---- fold the touched words into M: new bits = row & ~M ----
        // Every new bit counts in |delta|; only targets with out-edges become
        // rows of the next delta. Warp w takes summary chunks w, w + UW, ...
        const u64 mrow = (u64) U.x * stride;
        u32 nrows_w = 0, fresh = 0;
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
                const u32 h0 = a0 ? __ldg(hasout + k0) : 0u, h1 = a1 ? __ldg(hasout + k1) : 0u;
                const u32 o0 = a0 ? atomicOr(&m[mrow + k0], v0) : ~0u;
                const u32 o1 = a1 ? atomicOr(&m[mrow + k1], v1) : ~0u;
                const u32 f0 = v0 & ~o0, f1 = v1 & ~o1;
                const u32 r0 = f0 & h0, r1 = f1 & h1;
                if (a0) row[k0] = r0;
                if (a1) row[k1] = r1;
                fresh += __popc(f0) + __popc(f1);
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
        if (lane == 0) s.wrows[warp] = nrows_w;
        __syncthreads();  // (3) per-warp counts
        const u32 cw = lane < UW ? s.wrows[lane] : 0u;
        const u32 cinc = warp_inclusive_sum(cw);
        const u32 total = __shfl_sync(0xffffffffu, cinc, 31);
        const u32 before = __shfl_sync(0xffffffffu, cinc - cw, warp);  // new rows of lower warps
        // The unit's rows go to the CTA's reservation [ocur, oend); what does
        // not fit goes to a fresh one [nb, ...) (every thread reads the same
        // words, so all take the same branch). Unit-relative position i lands
        // at ocur + i below `avail`, at nb + (i - avail) above.
        const u64 ocur = s.ocur;
        const u64 avail = min((u64) total, s.oend - ocur);
        u64 nb = 0;
        if (total > avail) {
            if (tid == 0) {
                const u64 need = total - avail;
                const u64 size = max(need, OCHUNK);
                s.nbase = atomicAdd(&ctr->words, (unsigned long long) size);
                s.pend_ocur = s.nbase + need;
                s.pend_oend = s.nbase + size;
            }
            __syncthreads();  // (4, when a reservation runs out) the fresh one
            nb = s.nbase;
        } else if (tid == 0) {
            s.pend_ocur = ocur + total;  // s.ocur takes it after the next barrier (1)
            s.pend_oend = s.oend;
        }
        // ---- emit the new rows (targets of x) and clear the row ----
        // New bits are sparse within a word, so each lane walks its own word.
        // A row is written as the target's edge range; its loads are in flight
        // while the lane moves on to the next bit (the row is stored one bit
        // later), and its degree adds to the next join size.
        u64 p = before;  // unit-relative position
        u32 dsum = 0;
        bool pend = false;
        uint2 prow = make_uint2(0, 0);
        u64 pq = 0;
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
                const u32 tb = (kb + lane) * 32;
                while (fr) {
                    const u32 t = tb + (__ffs(fr) - 1);
                    fr &= fr - 1;
                    const u32 b = __ldg(off + t), e = __ldg(off + t + 1);
                    if (pend) {
                        const u64 a = pq < avail ? ocur + pq : nb + (pq - avail);
                        if (a < out_cap) out[a] = make_uint2(prow.x, prow.y - prow.x);
                        else atomicOr(err, DL_DEVERR_CAPACITY);  // more rows than reserved: reported
                        dsum += prow.y - prow.x;
                    }
                    prow = make_uint2(b, e);
                    pq = q++;
                    pend = true;
                }
                p += __shfl_sync(0xffffffffu, incl, 31);
            }
        }
        if (pend) {
            const u64 a = pq < avail ? ocur + pq : nb + (pq - avail);
            if (a < out_cap) out[a] = make_uint2(prow.x, prow.y - prow.x);
            else atomicOr(err, DL_DEVERR_CAPACITY);
            dsum += prow.y - prow.x;
        }
        {
            const u32 fw = warp_sum(fresh);
            const u64 dw = warp_sum((u64) dsum);
            if (lane == 0) {
                s.acc[warp][0] += fw;
                s.acc[warp][1] += dw;
                s.acc[warp][2] += nrows_w;
            }
        }
        // The unit's entries of the next delta (at most unit_rows rows each,
        // one range per reservation): slots from the CTA's reservation of unit
        // slots (thread 0 only).
        if (tid == 0 && total) {
            for (int part = 0; part < 2; ++part) {
                const u64 len = part == 0 ? avail : total - avail;
                const u64 start = part == 0 ? ocur : nb;
                for (u64 i = 0; i < len; i += unit_rows) {
                    if (s.ucur == s.uend) {
                        s.ucur = atomicAdd(&ctr->units, (unsigned long long) UCHUNK);
                        s.uend = s.ucur + UCHUNK;
                    }
                    const u64 slot = s.ucur++;
                    if (slot < uout_cap)
                        uout[slot] = Unit{U.x, (u32) min(unit_rows, len - i), start + i};
                    else
                        atomicOr(err, DL_DEVERR_CAPACITY);
                }
            }
        }
        if (tid == 0) s.e.next_group = 0;  // read again only after barrier (1)
    }
    // Unused reserved unit slots become empty units (skipped by fetch_unit).
    if (tid == 0)
        for (u64 slot = s.ucur; slot < s.uend; ++slot)
            if (slot < uout_cap) uout[slot] = Unit{0, 0, 0};
    if (lane == 0) {
        if (s.acc[warp][0]) atomicAdd(&ctr->fresh, s.acc[warp][0]);
        if (s.acc[warp][1]) atomicAdd(&ctr->join, s.acc[warp][1]);
        if (s.acc[warp][2]) atomicAdd(&ctr->rows, s.acc[warp][2]);
    }
}

// ---- SG on the bit matrix ----------------------------------------------
//
// sg(x, y) :- e(a, x), sg(a, b), e(b, y): with full as a bit matrix M (row x,
// column y), the new tuples of a delta unit (a, rows b) are
// R & ~M[x] for every x in e(a, .), where R = the union of e(b, .) over the
// unit's rows -- the same shared-memory row the TC step builds, folded into
// every row x of a's out-edges instead of into row a. The base rule
// sg(x, y) :- e(p, x), e(p, y), x != y is the same step on the units
// (p, rows {p}) with bit x cleared from R when it is folded into row x.
template <int NW>
struct SgSmem {
    ExpandSmemT<NW> e;
    Unit cur, next;
    u32 next_x;                      // next fold target of the unit (a's out-edge index)
    u32 nlist;                       // touched words of R in the list
    u64 res[NW][4];                  // per warp: next-delta rows [cur, end), unit slots [cur, end)
    unsigned long long acc[NW][3];   // per warp: new tuples, next-step bound, rows written
    // followed by: u32 row[words], u32 lk[words] (the touched words of R,
    // listed by the expansion in the order they were first touched)
};

constexpr u64 WCHUNK = 4096;  // next-delta rows a warp reserves at a time

// Writes the units of one fold target x: rows [start, start + len) of the
// next delta (at most unit_rows per unit), slots from the warp's reservation.
// Lane 0 only.
__device__ __forceinline__ void sg_close_range(u64 *res, u32 x, u64 start, u64 len, u64 unit_rows,
                                               Unit *__restrict__ uout, u64 uout_cap, StepCounters *ctr, u32 *err) {
    for (u64 i = 0; i < len; i += unit_rows) {
        if (res[2] == res[3]) {
            res[2] = atomicAdd(&ctr->units, (unsigned long long) UCHUNK);
            res[3] = res[2] + UCHUNK;
        }
        const u64 slot = res[2]++;
        if (slot < uout_cap) uout[slot] = Unit{x, (u32) min(unit_rows, len - i), start + i};
        else atomicOr(err, DL_DEVERR_CAPACITY);
    }
}

// NT threads per CTA: 512 for long rows; 128 (up to 12 CTAs per SM) when rows
// are short enough, so that the many small units of SG run in more, smaller
// CTAs (a unit's barriers then hold 4 warps instead of 16). The bound leaves
// 40 registers a thread: at 32 the kernel spilled.
template <int NT>
__global__ void __launch_bounds__(NT, 1536 / NT)
sg_unit_step_kernel(const u32 *__restrict__ off, const u32 *__restrict__ val, const uint2 *__restrict__ rows,
                    const Unit *__restrict__ units, u64 nunits, u32 *__restrict__ m, u64 stride, u32 words,
                    uint2 *__restrict__ out, u64 out_cap, Unit *__restrict__ uout, u64 uout_cap, u64 unit_rows,
                    const u32 *__restrict__ hasout, StepCounters *__restrict__ ctr, u32 *err, int base_rule) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NW = NT / 32;
    SgSmem<NW> &s = *reinterpret_cast<SgSmem<NW> *>(smem_raw);
    u32 *row = reinterpret_cast<u32 *>(smem_raw + sizeof(SgSmem<NW>));
    u32 *lk = row + words;
    const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const u32 lt = lanemask_lt();
    const u32 le = lane == 31 ? ~0u : (2u << lane) - 1;
    for (u32 k = tid; k < words; k += NT) row[k] = 0;
    if (lane == 0) {
        s.res[warp][0] = s.res[warp][1] = s.res[warp][2] = s.res[warp][3] = 0;
        s.acc[warp][0] = s.acc[warp][1] = s.acc[warp][2] = 0;
    }
    if (tid == 0) {
        s.e.next_group = 0;
        s.nlist = 0;
        s.next = fetch_unit(units, nunits, ctr);
    }
    for (;;) {
        if (tid == 0) {
            s.cur = s.next;
            s.next_x = 0;
        }
        __syncthreads();  // (1) unit known; row, list, group and target counters are clear
        const Unit U = s.cur;
        if (U.len == 0) break;
        if (tid == 0) s.next = fetch_unit(units, nunits, ctr);  // read only at the next barrier (1)
        // R, and the list of its touched words (any order)
        expand_unit<true>(s.e, row, nullptr, rows, val, U, lane, warp, lt, le, lk, &s.nlist);
        __syncthreads();  // (2) R and its list are complete
        const u32 nlist = s.nlist;
        // ---- fold R into every row x of a's out-edges; emit each x's new rows ----
        // A warp takes one x at a time and walks the list 32 words per step,
        // the 32 matrix atomics of a step in flight together. A new row is
        // written as its target's edge range, one bit later than its loads.
        const u32 xb = __ldg(off + U.x), xn = __ldg(off + U.x + 1) - xb;
        u32 fresh = 0, rows_w = 0;
        u64 bound = 0;  // sum over new rows (x, y) of deg(x) deg(y): the next step's new tuples are below it
        for (;;) {
            u32 i = 0;
            if (lane == 0) i = atomicAdd(&s.next_x, 1u);
            i = __shfl_sync(0xffffffffu, i, 0);
            if (i >= xn) break;
            const u32 x = __ldg(val + xb + i);
            const u32 ox = __ldg(off + x);
            const u32 dx = __ldg(off + x + 1) - ox;  // fold fan-out of a unit of x next step
            const u64 mrow = (u64) x * stride;
            const u32 self_word = base_rule ? (x >> 5) : ~0u;
            u64 *res = s.res[warp];
            u64 xstart = res[0], cur = res[0];
            bool pend = false;
            u64 pa = 0;
            uint2 prow = make_uint2(0, 0);
            for (u32 c0 = 0; c0 < nlist; c0 += 32) {
                const bool have = c0 + lane < nlist;
                const u32 k = have ? lk[c0 + lane] : 0u;
                u32 v = have ? row[k] : 0u;
                if (k == self_word) v &= ~(1u << (x & 31));  // base rule: x != y
                const u32 o = v ? atomicOr(&m[mrow + k], v) : ~0u;
                const u32 f = v & ~o;
                fresh += __popc(f);
                const u32 fr = (f && dx) ? f & __ldg(hasout + k) : 0u;  // rows only if both can join
                const u32 cnt = __popc(fr);
                const u32 incl = warp_inclusive_sum(cnt);
                const u32 tot = __shfl_sync(0xffffffffu, incl, 31);
                if (!tot) continue;
                if (cur + tot > res[1]) {  // the warp's reservation runs out: close x's range so far
                    if (pend) {  // the pending row belongs to the range being closed
                        if (pa < out_cap) out[pa] = make_uint2(prow.x, prow.y - prow.x);
                        else atomicOr(err, DL_DEVERR_CAPACITY);
                        bound += (u64) (prow.y - prow.x) * dx;
                        pend = false;
                    }
                    if (lane == 0) {
                        sg_close_range(res, x, xstart, cur - xstart, unit_rows, uout, uout_cap, ctr, err);
                        const u64 size = max((u64) tot, WCHUNK);
                        res[0] = atomicAdd(&ctr->words, (unsigned long long) size);
                        res[1] = res[0] + size;
                    }
                    __syncwarp();
                    xstart = cur = res[0];
                }
                u64 q = cur + (incl - cnt);
                u32 bits = fr;
                while (bits) {
                    const u32 t = k * 32 + (__ffs(bits) - 1);
                    bits &= bits - 1;
                    const u32 b = __ldg(off + t), e = __ldg(off + t + 1);
                    if (pend) {
                        if (pa < out_cap) out[pa] = make_uint2(prow.x, prow.y - prow.x);
                        else atomicOr(err, DL_DEVERR_CAPACITY);  // reported: the host reruns on the sorted runs
                        bound += (u64) (prow.y - prow.x) * dx;
                    }
                    prow = make_uint2(b, e);
                    pa = q++;
                    pend = true;
                }
                cur += tot;
                rows_w += cnt;
            }
            if (pend) {
                if (pa < out_cap) out[pa] = make_uint2(prow.x, prow.y - prow.x);
                else atomicOr(err, DL_DEVERR_CAPACITY);
                bound += (u64) (prow.y - prow.x) * dx;
            }
            if (lane == 0) {
                sg_close_range(res, x, xstart, cur - xstart, unit_rows, uout, uout_cap, ctr, err);
                res[0] = cur;
            }
            __syncwarp();
        }
        {
            const u32 fw = warp_sum(fresh), rw = warp_sum(rows_w);
            const u64 bw = warp_sum(bound);
            if (lane == 0) {
                s.acc[warp][0] += fw;
                s.acc[warp][1] += bw;
                s.acc[warp][2] += rw;
            }
        }
        __syncthreads();  // (3) every fold target is done with R
        // ---- clear R (the list holds every touched word) ----
        for (u32 i2 = tid; i2 < nlist; i2 += NT) row[lk[i2]] = 0;
        if (tid == 0) s.nlist = 0;  // read again only after barrier (2)
        if (tid == 0) s.e.next_group = 0;  // read again only after barrier (1)
    }
    // Unused reserved unit slots become empty units (skipped by fetch_unit).
    if (lane == 0) {
        for (u64 slot = s.res[warp][2]; slot < s.res[warp][3]; ++slot)
            if (slot < uout_cap) uout[slot] = Unit{0, 0, 0};
        if (s.acc[warp][0]) atomicAdd(&ctr->fresh, s.acc[warp][0]);
        if (s.acc[warp][1]) atomicAdd(&ctr->join, s.acc[warp][1]);
        if (s.acc[warp][2]) atomicAdd(&ctr->rows, s.acc[warp][2]);
    }
}

// Base units of SG: node p -> row p = (off[p], deg p) and unit (p, rows {p})
// (empty when p has no out-edges); *bound += deg(p)^2, the base's new tuples
// are below it.
__global__ void sg_base_units_kernel(const u32 *__restrict__ off, u64 n, uint2 *__restrict__ rows,
                                     Unit *__restrict__ units, unsigned long long *__restrict__ bound) {
    u64 b2 = 0;
    for (u64 p = (u64) blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (u64) gridDim.x * blockDim.x) {
        const u32 b = off[p], d = off[p + 1] - b;
        rows[p] = make_uint2(b, d);
        units[p] = Unit{(u32) p, d ? 1u : 0u, p};
        b2 += (u64) d * d;
    }
    b2 = warp_sum(b2);
    if ((threadIdx.x & 31) == 0 && b2) atomicAdd(bound, (unsigned long long) b2);
}

// Row sums: counts[x] = set bits of row x among its first `words` words.
__global__ void bitmat_row_popc_kernel(const u32 *__restrict__ m, u64 n, u64 stride, u64 words,
                                       unsigned long long *__restrict__ counts) {
    const u32 lane = threadIdx.x & 31;
    const u64 warps = (u64) gridDim.x * (blockDim.x / 32);
    for (u64 x = ((u64) blockIdx.x * blockDim.x + threadIdx.x) / 32; x < n; x += warps) {
        const u32 *r = m + x * stride;
        u32 c = 0;
        for (u64 k = lane; k < words; k += 32) c += __popc(__ldcs(r + k));
        c = warp_sum(c);
        if (lane == 0) counts[x] = c;
    }
}

// a result row as one little-endian 8-byte word: (column id, row id) for a
// matrix row's bits read as column ids (TC's (x, z) of target z), (row id,
// column id) for SG's rows
template <bool RowFirst>
__device__ __forceinline__ u64 pack_row(u32 row_id, u32 col_id) {
    return RowFirst ? ((u64) col_id << 32) | row_id : ((u64) row_id << 32) | col_id;
}
__device__ __forceinline__ u32 xid(const int32_t *__restrict__ ids, bool affine, int32_t base, u64 x) {
    return (u32) (affine ? (int32_t) (base + (int64_t) x) : __ldg(ids + x));
}

// a[r] bit b -> a[b] bit r: a 32 x 32 bit transpose inside one thread's
// registers by recursive block swaps (round j exchanges bit j of the row
// index with bit j of the bit index; H. S. Warren, Hacker's Delight, 2nd
// ed., section 7-3).
__device__ __forceinline__ void transpose32_regs(u32 (&a)[32]) {
    // rounds 16 and 8 move whole half-words and bytes: one byte permute per word
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const u32 lo = a[k], hi = a[k + 16];
        a[k] = __byte_perm(lo, hi, 0x5410);
        a[k + 16] = __byte_perm(lo, hi, 0x7632);
    }
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        if (k & 8) continue;
        const u32 lo = a[k], hi = a[k + 8];
        a[k] = __byte_perm(lo, hi, 0x6240);
        a[k + 8] = __byte_perm(lo, hi, 0x7351);
    }
#pragma unroll
    for (int j = 4; j >= 1; j >>= 1) {
        const u32 m = j == 4 ? 0x0F0F0F0Fu : j == 2 ? 0x33333333u : 0x55555555u;
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            if (k & j) continue;
            const u32 t = ((a[k] >> j) ^ a[k + j]) & m;
            a[k + j] ^= t;
            a[k] ^= t << j;
        }
    }
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    const unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// TC's result rows (x, z) in the reference's order (by z, then x) come from
// the columns of the matrix M (row x, bit z). Each pass below walks M in
// tiles of CX_ROWS source rows x CX_WORDS column words (128 bytes of every
// row, read with 16-byte cp.async into shared memory, the next tile in
// flight while the current one is worked on):
//   transpose pass (the default form): each tile's target-major words are
//     stored as 64-byte segments of T (row = target) with per-target counts;
//   count pass (column form): per tile and target z, the set bits of column
//     z in the tile's rows -> off[xb][z] (xb = the tile's row block); a
//     column scan turns off[.][z] into offsets within column z, a scan of
//     the column totals gives each z its first row;
//   rows pass (column form): the same walk writes every set bit (x, z) of a
//     tile to out[first[z] + off[xb][z] + rank of x among the tile's bits].
// In a tile, thread (warp w, lane l) reads the 32 x 32 bit block (row block
// rb = l % 16, column word cw = (w + l) % 32) one row at a time -- the 32
// lanes read 32 different column words, so no bank conflicts -- transposes
// it in registers and stores the 32 target words to a target-major tile
// (1024 targets x 16 words); four lanes then take each target row, 4 words
// (one 16-byte load) each.
constexpr int CX_ROWS = 512;                  // source rows of a tile
constexpr int CX_WORDS = 32;                  // column words of a tile
constexpr int CX_TARGETS = CX_WORDS * 32;     // targets of a tile
constexpr int CX_XW = CX_ROWS / 32;           // words of a target row in a tile
constexpr int CX_THREADS = 512;
struct ColSmem {
    u32 in[2][CX_ROWS][CX_WORDS];  // source tiles (two buffers)
    u32 live[2][CX_ROWS / 32];     // the tiles' row-written bits
    u32 outw[CX_TARGETS][CX_XW];   // the current tile, target-major
    u64 base[CX_TARGETS];          // rows pass: first output row of each target in this tile
    u32 cnt[CX_TARGETS];           // count pass: set bits of each target in this tile
};
static_assert(CX_WORDS == 32 && CX_ROWS / 32 == CX_THREADS / 32, "one block per thread and tile");

enum ColMode { COL_COUNT = 0, COL_ROWS = 1, COL_TRANSPOSE = 2 };

template <int MODE>
__device__ __forceinline__ void bitmat_columns_body(const u32 *__restrict__ m, const u32 *__restrict__ live,
                                                    u64 n, u64 stride, u64 xblocks,
                                                    u64 t_first, u64 tiles, u32 *__restrict__ off,
                                                    const u64 *__restrict__ first,
                                                    const int32_t *__restrict__ ids, bool affine, int32_t base,
                                                    u64 *__restrict__ out, u32 *__restrict__ tout,
                                                    unsigned long long *__restrict__ counts) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ColSmem &s = *reinterpret_cast<ColSmem *>(smem_raw);
    const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // tiles are numbered column block major; CTA k takes a contiguous range
    // of tiles [t_first, t_first + tiles)
    const u64 t_begin = t_first + tiles * blockIdx.x / gridDim.x;
    const u64 t_end = t_first + tiles * (blockIdx.x + 1) / gridDim.x;
    auto issue = [&](u64 t, int buf) {  // 16-byte chunks tid, tid + 512, ...: 8 per source row
        const u64 x0 = (t % xblocks) * CX_ROWS;
        const u32 *src = m + (t / xblocks) * CX_WORDS;
#pragma unroll
        for (int i = 0; i < CX_ROWS * CX_WORDS / 4 / CX_THREADS; ++i) {
            const u32 chunk = tid + i * CX_THREADS;
            const u32 r = chunk / (CX_WORDS / 4), c4 = chunk % (CX_WORDS / 4);
            u32 *dst = &s.in[buf][r][c4 * 4];
            if (x0 + r < n) cp_async16(dst, src + (x0 + r) * stride + c4 * 4);
            else *reinterpret_cast<uint4 *>(dst) = make_uint4(0u, 0u, 0u, 0u);
        }
        // the tile's 16 words of `live` (padded to whole tiles by the caller)
        if (tid < CX_ROWS / 32 / 4) cp_async16(&s.live[buf][4 * tid], live + x0 / 32 + 4 * tid);
    };
    const u32 rb = lane & 15, cw = (warp + lane) & 31, hi = lane >> 4;
    const u32 q = tid & 3;  // this thread's quarter of a target row
    constexpr int TPT = CX_TARGETS * 4 / CX_THREADS;  // target quarters per thread and tile
    if constexpr (MODE == COL_COUNT) {
        for (u32 i = tid; i < CX_TARGETS; i += CX_THREADS) s.cnt[i] = 0;  // ordered by barrier (1)
    }
    // transpose: set bits of this thread's target quarters in the current column block
    u32 tcnt[TPT];
#pragma unroll
    for (int k = 0; k < TPT; ++k) tcnt[k] = 0;
    u64 tcb = t_begin < t_end ? t_begin / xblocks : 0;
    auto flush_counts = [&](u64 cb) {  // the four quarters of a target are lanes 4j..4j+3
#pragma unroll
        for (int k = 0; k < TPT; ++k) {
            u32 c = tcnt[k];
            c += __shfl_xor_sync(0xffffffffu, c, 1);
            c += __shfl_xor_sync(0xffffffffu, c, 2);
            const u64 z = cb * CX_TARGETS + (tid >> 2) + k * (CX_THREADS / 4);
            if (q == 0 && c && z < n) atomicAdd(counts + z, (unsigned long long) c);
            tcnt[k] = 0;
        }
    };
    int buf = 0;
    if (t_begin < t_end) issue(t_begin, 0);
    cp_async_commit();
    for (u64 t = t_begin; t < t_end; ++t, buf ^= 1) {
        // s.in[buf ^ 1] was last read before the previous tile's second barrier
        if (t + 1 < t_end) issue(t + 1, buf ^ 1);
        cp_async_commit();
        const u64 xb = t % xblocks, cb = t / xblocks, z0 = cb * CX_TARGETS;
        u64 pb[CX_TARGETS / CX_THREADS];  // rows pass: first rows of targets tid, tid + 512 in this tile
        if constexpr (MODE == COL_ROWS) {
#pragma unroll
            for (int k = 0; k < CX_TARGETS / CX_THREADS; ++k) {
                const u64 z = z0 + tid + k * CX_THREADS;
                pb[k] = z < n ? first[z] + off[xb * n + z] : 0;
            }
        }
        if constexpr (MODE == COL_TRANSPOSE) {
            if (cb != tcb) {  // uniform across the CTA
                flush_counts(tcb);
                tcb = cb;
            }
        }
        cp_async_wait_prev();
        __syncthreads();  // (1) tile t has landed; the previous tile's results are out
        u32 a[32];
        if constexpr (MODE == COL_COUNT) {
            // counts only: rotate row words right by `lane` before the
            // transpose, so that a[b] then belongs to target 32 cw + (b + lane)
            // % 32 and the 32 lanes' shared-memory atomics hit 32 banks
            // rows the fixpoint never wrote (sources without out-edges: not
            // zeroed, they may hold an earlier run's bits) read as zero
            const u32 lw = s.live[buf][rb];
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                const u32 w = ((lw >> r) & 1u) ? s.in[buf][32 * rb + r][cw] : 0u;
                a[r] = __funnelshift_r(w, w, lane);
            }
            transpose32_regs(a);
#pragma unroll
            for (int b = 0; b < 32; ++b) {
                const u32 c = __popc(a[b]);
                if (c) atomicAdd(&s.cnt[32 * cw + ((b + lane) & 31)], c);
            }
            __syncthreads();  // (2) the tile's counts are complete
            for (u32 i = tid; i < CX_TARGETS; i += CX_THREADS) {
                const u64 z = z0 + i;
                if (z < n) off[xb * n + z] = s.cnt[i];
                s.cnt[i] = 0;
            }
        } else {
            if constexpr (MODE == COL_ROWS) {
#pragma unroll
                for (int k = 0; k < CX_TARGETS / CX_THREADS; ++k) s.base[tid + k * CX_THREADS] = pb[k];
            }
            const u32 lw = s.live[buf][rb];  // unwritten rows read as zero
#pragma unroll
            for (int r = 0; r < 32; ++r) a[r] = ((lw >> r) & 1u) ? s.in[buf][32 * rb + r][cw] : 0u;
            transpose32_regs(a);
            // a[b] = word rb of target 32 cw + b; the upper half-warp stores
            // b ^ 1 while the lower stores b, so the 32 stores hit 32 banks
#pragma unroll
            for (int b = 0; b < 32; ++b) s.outw[32 * cw + (b ^ hi)][rb] = hi ? a[b ^ 1] : a[b];
            __syncthreads();  // (2) the target-major tile is complete
            if constexpr (MODE == COL_TRANSPOSE) {
                // four lanes per target row segment (64 bytes): 8 targets per warp store
#pragma unroll
                for (int k = 0; k < TPT; ++k) {
                    const u32 i = (tid >> 2) + k * (CX_THREADS / 4);
                    const uint4 w4 = *reinterpret_cast<const uint4 *>(&s.outw[i][4 * q]);
                    tcnt[k] += __popc(w4.x) + __popc(w4.y) + __popc(w4.z) + __popc(w4.w);
                    const u64 z = z0 + i;
                    if (z < n) *reinterpret_cast<uint4 *>(tout + z * stride + xb * CX_XW + 4 * q) = w4;
                }
            } else {
                // four lanes per target, four words (128 source rows) per lane
#pragma unroll 2
                for (u32 i = tid >> 2; i < CX_TARGETS; i += CX_THREADS / 4) {
                    const uint4 w4 = *reinterpret_cast<const uint4 *>(&s.outw[i][4 * q]);
                    const u32 c = __popc(w4.x) + __popc(w4.y) + __popc(w4.z) + __popc(w4.w);
                    u32 incl = c;
                    u32 y = __shfl_up_sync(0xffffffffu, incl, 1, 4);
                    if (q >= 1) incl += y;
                    y = __shfl_up_sync(0xffffffffu, incl, 2, 4);
                    if (q >= 2) incl += y;
                    const u64 z = z0 + i;
                    if (z >= n || c == 0) continue;
                    u64 p = s.base[i] + (incl - c);
                    const u32 zid = xid(ids, affine, base, z);
                    const u64 x0 = (xb * CX_XW + 4 * q) * 32;
                    // the lane's 128 bits as one sequence: one pass per set bit
                    u64 lo = ((u64) w4.y << 32) | w4.x, hi2 = ((u64) w4.w << 32) | w4.z;
                    while (lo | hi2) {
                        u32 bit;
                        if (lo) {
                            bit = (u32) __ffsll((long long) lo) - 1;
                            lo &= lo - 1;
                        } else {
                            bit = 64 + (u32) __ffsll((long long) hi2) - 1;
                            hi2 &= hi2 - 1;
                        }
                        out[p++] = pack_row<false>(zid, xid(ids, affine, base, x0 + bit));
                    }
                }
            }
        }
    }
    if constexpr (MODE == COL_TRANSPOSE) {
        if (t_begin < t_end) flush_counts(tcb);
    }
}

__global__ void __launch_bounds__(CX_THREADS, 1)
bitmat_column_count_kernel(const u32 *__restrict__ m, const u32 *__restrict__ live, u64 n, u64 stride, u64 xblocks,
                           u64 tiles, u32 *__restrict__ off) {
    bitmat_columns_body<COL_COUNT>(m, live, n, stride, xblocks, 0, tiles, off, nullptr, nullptr, false, 0, nullptr,
                                   nullptr, nullptr);
}

__global__ void __launch_bounds__(CX_THREADS, 1)
bitmat_column_rows_kernel(const u32 *__restrict__ m, const u32 *__restrict__ live, u64 n, u64 stride, u64 xblocks,
                          u64 t_first, u64 tiles, const u32 *__restrict__ off, const u64 *__restrict__ first,
                          const int32_t *__restrict__ ids, bool affine, int32_t base, u64 *__restrict__ out) {
    bitmat_columns_body<COL_ROWS>(m, live, n, stride, xblocks, t_first, tiles, const_cast<u32 *>(off), first, ids,
                                  affine, base, out, nullptr, nullptr);
}

// t = the transpose of m (n rows of `stride` words each; rows whose bit in
// `live` is clear read as zero), counts[z] += the set bits of row z of t
// (counts zeroed by the caller).
__global__ void __launch_bounds__(CX_THREADS, 1)
bitmat_transpose_count_kernel(const u32 *__restrict__ m, const u32 *__restrict__ live, u64 n, u64 stride,
                              u64 xblocks, u64 tiles, u32 *__restrict__ t, unsigned long long *__restrict__ counts) {
    bitmat_columns_body<COL_TRANSPOSE>(m, live, n, stride, xblocks, 0, tiles, nullptr, nullptr, nullptr, false, 0,
                                       nullptr, t, counts);
}

// Zero the rows of m whose bit in `live` is set (one warp per row, 16-byte
// stores): TC writes only the rows of sources with out-edges, and readers of
// the matrix treat the other rows as zero.
__global__ void bitmat_zero_rows_kernel(u32 *__restrict__ m, u64 n, u64 stride, const u32 *__restrict__ live) {
    const u64 warps = (u64) gridDim.x * (blockDim.x / 32);
    const u32 lane = threadIdx.x & 31;
    for (u64 x = (u64) blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); x < n; x += warps) {
        if (!((__ldg(live + (x >> 5)) >> (x & 31)) & 1u)) continue;
        uint4 *row = reinterpret_cast<uint4 *>(m + x * stride);
        for (u64 k = lane; k < stride / 4; k += 32) row[k] = make_uint4(0u, 0u, 0u, 0u);
    }
}

// off[.][z]: per row block counts of column z -> exclusive prefix over the
// row blocks; tot[z] = the column's total (at most n < 2^31 bits).
__global__ void column_offsets_kernel(u32 *__restrict__ off, u64 n, u64 xblocks, unsigned long long *__restrict__ tot) {
    const u64 z = (u64) blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= n) return;
    u32 run = 0;
    u64 xb = 0;
    for (; xb + 4 <= xblocks; xb += 4) {
        u32 *p = off + xb * n + z;
        const u32 c0 = p[0], c1 = p[n], c2 = p[2 * n], c3 = p[3 * n];
        p[0] = run;
        p[n] = run += c0;
        p[2 * n] = run += c1;
        p[3 * n] = run += c2;
        run += c3;
    }
    for (; xb < xblocks; ++xb) {
        const u32 c = off[xb * n + z];
        off[xb * n + z] = run;
        run += c;
    }
    tot[z] = run;
}

// Position of the k-th set bit (k from 0) of w, which has more than k set
// bits: a binary search on the popcounts of the low halves.
__device__ __forceinline__ u32 select_bit(u32 w, u32 k) {
    u32 pos = 0, c;
    c = __popc(w & 0xFFFFu);
    if (k >= c) { k -= c; w >>= 16; pos += 16; }
    c = __popc(w & 0xFFu);
    if (k >= c) { k -= c; w >>= 8; pos += 8; }
    c = __popc(w & 0xFu);
    if (k >= c) { k -= c; w >>= 4; pos += 4; }
    c = __popc(w & 0x3u);
    if (k >= c) { k -= c; w >>= 2; pos += 2; }
    if (k >= (w & 1u)) pos += 1;
    return pos;
}

// Row w of the matrix -> result rows for its set bits x, ascending, from
// out[first[w]] on: (ids[w], ids[x]) for SG's matrix (its order (x, y) by
// (x, y)), (ids[x], ids[w]) for TC's transpose (row = target z: (x, z) by
// (z, x)). One warp per row; a lane takes 4 consecutive words per step (one
// 16-byte load, two steps' loads in flight). A sparse step (at most EX_STAGE
// rows) is written by word: each lane walks its words' bits into a
// shared-memory stage, which leaves with consecutive stores. A dense step is
// written by output position: lane i writes rows i, i + 32, ... of the step,
// finding the lane that holds the row by a binary search over the warp's
// prefix counts and the bit inside its word by popcounts, so every lane
// writes a row per pass and the stores are consecutive. (Measured: by word
// is faster on TC's sparse transpose rows, by position 2.4x faster on SG's
// dense rows.)
constexpr int EX_THREADS = 256;
constexpr int EX_STAGE = 256;
template <bool RowFirst>
__global__ void __launch_bounds__(EX_THREADS) bitmat_extract_rows_kernel(const u32 *__restrict__ t, u64 w_begin,
                                                                         u64 w_end, u64 stride, u64 words,
                                                                         const u64 *__restrict__ first,
                                                                         const int32_t *__restrict__ ids,
                                                                         bool affine, int32_t base,
                                                                         u64 *__restrict__ out) {
    __shared__ u64 stage[EX_THREADS / 32][EX_STAGE];
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u64 *st = stage[warp];
    const u64 warps = (u64) gridDim.x * (EX_THREADS / 32);
    for (u64 w = w_begin + (u64) blockIdx.x * (EX_THREADS / 32) + warp; w < w_end; w += warps) {
        const u32 *row = t + w * stride;
        u64 pos = first[w];
        // a dense id range needs no table lookup (ids[r] == base + r)
        const u32 idw = (u32) (affine ? (int32_t) (base + (int64_t) w) : ids[w]);
        // stride is a multiple of 32 words: a lane's vector stays in the row.
        auto load = [&](u64 k) {
            return k < words ? __ldcs(reinterpret_cast<const uint4 *>(row + k)) : make_uint4(0, 0, 0, 0);
        };
        uint4 n1 = load((u64) lane * 4), n2 = load((u64) lane * 4 + 128);
        for (u64 k0 = 0; k0 < words; k0 += 128) {
            const u64 k = k0 + lane * 4;
            const uint4 q = n1;
            n1 = n2;
            n2 = load(k + 256);
            u32 v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (k + c >= words) v[c] = 0;  // past the used columns
            const u32 cnt = __popc(v[0]) + __popc(v[1]) + __popc(v[2]) + __popc(v[3]);
            const u32 incl = warp_inclusive_sum(cnt);
            const u32 sum = __shfl_sync(0xffffffffu, incl, 31);
            if (sum == 0) continue;
            const u32 excl = incl - cnt;
            if (sum <= EX_STAGE) {
                u32 p = excl;
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    for (u32 b = v[c]; b; b &= b - 1)
                        st[p++] = pack_row<RowFirst>(idw, xid(ids, affine, base, (k + c) * 32 + (__ffs(b) - 1)));
                __syncwarp();
                for (u32 i = lane; i < sum; i += 32) out[pos + i] = st[i];
                __syncwarp();
                pos += sum;
                continue;
            }
            for (u32 r0 = 0; r0 < sum; r0 += 32) {
                const u32 r = r0 + lane;
                // owner: the last lane whose exclusive prefix is <= r (it
                // holds row r whenever r < sum)
                u32 L = 0;
#pragma unroll
                for (u32 step = 16; step >= 1; step >>= 1)
                    if (__shfl_sync(0xffffffffu, excl, L + step) <= r) L += step;
                u32 kk = r - __shfl_sync(0xffffffffu, excl, L);
                const u32 w0 = __shfl_sync(0xffffffffu, v[0], L), w1 = __shfl_sync(0xffffffffu, v[1], L);
                const u32 w2 = __shfl_sync(0xffffffffu, v[2], L), w3 = __shfl_sync(0xffffffffu, v[3], L);
                u32 c = 0, word = w0, pc = __popc(w0);
                if (kk >= pc) { kk -= pc; c = 1; word = w1; pc = __popc(w1); }
                if (c == 1 && kk >= pc) { kk -= pc; c = 2; word = w2; pc = __popc(w2); }
                if (c == 2 && kk >= pc) { kk -= pc; c = 3; word = w3; }
                if (r < sum) {
                    const u64 x = (k0 + 4 * L + c) * 32 + select_bit(word, kk);
                    out[pos + r] = pack_row<RowFirst>(idw, xid(ids, affine, base, x));
                }
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
u64 bitmat_column_offset_bytes(u64 n) { return std::max<u64>((n + CX_ROWS - 1) / CX_ROWS * n * 4, 4); }

bool bitmat_choose(Context &ctx, const dl_options &opt, u64 n, bool sg) {
    if (opt.dedup != DL_DEDUP_AUTO && opt.dedup != DL_DEDUP_BITMAP) return false;
    // a row (TC), or a row and its touched-word list (SG), must fit in shared memory
    if ((n + 31) / 32 * 4 * (sg ? 2 : 1) + sizeof(SgSmem<UW>) + 4096 > 227 * 1024) return false;
    // TC also keeps the per (row block, target) offsets of its result rows
    const u64 need = bitmat_bytes(n) + (sg ? 0 : bitmat_column_offset_bytes(n));
    // a context that already holds the matrix buffer (a repeated run) needs
    // no driver query: the memory is its own
    if (opt.dedup == DL_DEDUP_AUTO && ctx.ws.bitmat[0].cap >= bitmat_bytes(n) &&
        need <= ((u64) ctx.tune.bitmap_max_gib << 30))
        return true;
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


// Whether a TC run's result rows leave through the matrix's transpose (a
// second n x n matrix; the faster form) rather than from its columns.
static bool tc_result_by_transpose(Context &ctx, u64 n) {
    if (ctx.tune.bitmap_result == 1) return true;
    if (ctx.tune.bitmap_result == 2) return false;
    const u64 need = bitmat_bytes(n);
    if (2 * need > ((u64) ctx.tune.bitmap_max_gib << 30)) return false;
    // a buffer the context keeps that the transpose would reuse: no query
    if (ctx.ws.bitmat[1].cap >= need) return true;
    for (const DevBuf &b : ctx.spares)
        if (b.cap >= need && b.cap <= 4 * need) return true;
    size_t free_b = 0, total_b = 0;
    DL_CUDA(cudaMemGetInfo(&free_b, &total_b));
    u64 cached = ctx.ws.bitmat[1].cap;
    for (const DevBuf &b : ctx.spares) cached += b.cap;
    return need + (1ull << 30) <= (u64) free_b + cached;
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
    u32 *m = M.as<u32>();
    // sources with out-edges: the only rows the fixpoint writes (every unit's
    // source has out-edges), so only they are zeroed; the other rows are
    // read as zero by the result's kernels
    // (padded to whole 512-row tiles: the result's kernels read a tile's 16 words at once)
    ctx.reserve(ws.bit_hasout, ((words_used + 15) / 16 * 16 + 16) * 4);
    DL_LAUNCH(ctx, K_PREP, 4.0 * n + 4.0 * words_used,
              hasout_kernel<<<grid_for(words_used, T256, ctx), T256, 0, ctx.stream>>>(g.csr.off, n, words_used,
                                                                                      ws.bit_hasout.as<u32>()));
    DL_LAUNCH(ctx, K_PREP, 0,
              bitmat_zero_rows_kernel<<<grid_for(n * 32, T256, ctx, 8), T256, 0, ctx.stream>>>(
                  m, n, stride, ws.bit_hasout.as<u32>()));
    StepCounters *ctr = reinterpret_cast<StepCounters *>(&ctx.ctrl->scalar[52]);
    // delta_0 = the edges: one row per CSR value (its edge range), units from
    // the CSR's offsets; the rows live in jbuf[1], the first step writes jbuf[0]
    const uint2 *rows = nullptr;
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
        ctx.reserve(ws.jbuf[1], ne * 8);
        DL_LAUNCH(ctx, K_PREP, 20.0 * ne,
                  edge_rows_kernel<<<grid_for(ne, T256, ctx), T256, 0, ctx.stream>>>(g.csr.off, g.csr.val, ne,
                                                                                     ws.jbuf[1].as<uint2>()));
        rows = ws.jbuf[1].as<uint2>();
        DL_CUDA(cudaMemsetAsync(&ctr->join, 0, sizeof(u64), ctx.stream));
        DL_LAUNCH(ctx, K_PREP, 8.0 * ne,
                  edge_degree_sum_kernel<<<grid_for(ne, T256, ctx), T256, 0, ctx.stream>>>(g.csr.off, g.csr.val, ne,
                                                                                           &ctr->join));
        DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, &ctr->join, sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
        join = ctx.host_scalars[0];
    }
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
            const unsigned grid = (unsigned) std::min<u64>(nunits, resident);
            // New rows <= join words. CTAs reserve rows in blocks of OCHUNK (a
            // unit that overflows one continues in the next), so at most the
            // last reservation of every CTA is left partly unused; unit slots
            // are reserved UCHUNK at a time.
            DevBuf &obuf = ws.jbuf[slot];
            const u64 ocap = join + (u64) grid * OCHUNK;
            ctx.reserve(obuf, ocap * 8);
            const u64 ucap = nunits + join / unit_rows + 1 + (u64) grid * UCHUNK;
            ctx.reserve(*ubuf_next, ucap * sizeof(Unit));
            DL_CUDA(cudaMemsetAsync(ctr, 0, sizeof(StepCounters), ctx.stream));
            // algorithmic bytes: delta rows (8 B) and units in, one edge target per join word, new rows and units out
            DL_LAUNCH(ctx, K_BITMAP_EXPAND, 8.0 * nrows + 16.0 * nunits + 4.0 * join,
                      kern<<<grid, UT, smem, ctx.stream>>>(g.csr.off, g.csr.val, rows, ubuf->as<Unit>(), nunits, m,
                                                           stride, (u32) words_used, obuf.as<uint2>(), ocap,
                                                           ubuf_next->as<Unit>(), ucap, unit_rows,
                                                           ws.bit_hasout.as<u32>(), ctr, &ctx.ctrl->err));
            DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, ctr, sizeof(StepCounters), cudaMemcpyDeviceToHost, ctx.stream));
            ctx.sync();
            const u64 next_rows = ctx.host_scalars[5];  // rows written (host_scalars[1]: rows reserved)
            next_join = ctx.host_scalars[2];
            next_units = ctx.host_scalars[3];
            nnew = ctx.host_scalars[4];
            ctx.prof_add_bytes(K_BITMAP_EXPAND, 8.0 * next_rows + 16.0 * next_units);
            rows = obuf.as<uint2>();
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
    // The result rows are written when they are copied out
    // (bitmat_extract_rows), in the reference's order (by target, then
    // source), from either
    //  - the transpose T of M (row = target) and each target's first row,
    //    when a second matrix fits (bitmap_result 0 or 1), or
    //  - M's columns, with per (512-row block, target) offsets (1/16 of a
    //    matrix) and each target's first row (bitmap_result 2, or 0 when the
    //    transpose does not fit).
    if (nfull) {
        const u64 xblocks = (n + CX_ROWS - 1) / CX_ROWS, tiles = (stride / CX_WORDS) * xblocks;
        const unsigned cg = (unsigned) std::min<u64>(tiles, (u64) ctx.sm_count);
        ctx.reserve(ws.offsets, (n + 1) * 8);
        u64 *counts = ws.offsets.as<u64>();
        const bool by_transpose = tc_result_by_transpose(ctx, n);
        DevBuf &O = ws.bitmat[1];  // T, or the column offsets
        if (by_transpose) {
            ctx.reserve(O, bitmat_bytes(n));
            DL_CUDA(cudaMemsetAsync(counts, 0, n * 8, ctx.stream));
            DL_CUDA(cudaFuncSetAttribute(bitmat_transpose_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int) sizeof(ColSmem)));
            DL_LAUNCH(ctx, K_BITMAP_COLUMNS, 2.0 * bitmat_bytes(n),
                      bitmat_transpose_count_kernel<<<cg, CX_THREADS, sizeof(ColSmem), ctx.stream>>>(
                          m, ws.bit_hasout.as<u32>(), n, stride, xblocks, tiles, O.as<u32>(),
                          reinterpret_cast<unsigned long long *>(counts)));
        } else {
            ctx.reserve(O, bitmat_column_offset_bytes(n));
            DL_CUDA(cudaFuncSetAttribute(bitmat_column_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int) sizeof(ColSmem)));
            DL_LAUNCH(ctx, K_BITMAP_COLUMNS, 1.0 * bitmat_bytes(n) + 4.0 * xblocks * n,
                      bitmat_column_count_kernel<<<cg, CX_THREADS, sizeof(ColSmem), ctx.stream>>>(
                          m, ws.bit_hasout.as<u32>(), n, stride, xblocks, tiles, O.as<u32>()));
            DL_LAUNCH(ctx, K_BITMAP_COLUMNS, 8.0 * xblocks * n + 8.0 * n,
                      column_offsets_kernel<<<grid_for(n, T256, ctx, 64), T256, 0, ctx.stream>>>(
                          O.as<u32>(), n, xblocks, reinterpret_cast<unsigned long long *>(counts)));
        }
        ctx.reserve(ws.w0, (n + 1) * 8);
        const u64 total = exclusive_scan(ctx, counts, n, ws.w0.as<u64>());
        if (total != nfull)
            throw Error(DL_ERR_INTERNAL, "bit matrix holds " + std::to_string(total) + " tuples, expected " +
                                             std::to_string(nfull));
        if (by_transpose) {
            r.bm_t = O;  // M stays in the workspace for the next run
        } else {
            r.bm_t = M;
            M = DevBuf();
            r.bm_off = O;
            r.bm_live = ws.bit_hasout;  // the rows pass reads M again when the rows are copied out
            ws.bit_hasout = DevBuf();
            r.bm_cols = true;
        }
        O = DevBuf();
        r.bm_first = ws.w0;
        ws.w0 = DevBuf();
        r.bm_n = n;
        r.bm_stride = stride;
        r.bm_words = words_used;
    }
    r.from_bitmat = true;
    return nfull;
}

u64 sg_bitmap_fixpoint(Context &ctx, Run &r, const Graph &g, const dl_options &opt, PhaseTimer &pt) {
    Workspace &ws = ctx.ws;
    const u64 n = g.n_ids;
    const u64 stride = bitmat_stride(n);
    const u64 unit_rows = std::max<u64>(1, ctx.tune.bitmap_unit_rows);
    const u64 words_used = (n + 31) / 32;
    const size_t row_smem = 2 * words_used * 4 + 16;  // R and its touched-word list
    const size_t smem = sizeof(SgSmem<UW>) + row_smem;
    if (smem > 227 * 1024) throw Error(DL_ERR_OUT_OF_MEMORY, "bit-matrix rows of " + std::to_string(n) +
                                                              " nodes do not fit in shared memory");
    DevBuf &M = ws.bitmat[0];
    ctx.reserve(M, std::max<u64>(bitmat_bytes(n), 4));
    DL_CUDA(cudaMemsetAsync(M.p, 0, bitmat_bytes(n), ctx.stream));
    u32 *m = M.as<u32>();
    StepCounters *ctr = reinterpret_cast<StepCounters *>(&ctx.ctrl->scalar[52]);
    ctx.reserve(ws.bit_hasout, std::max<u64>(words_used, 1) * 4);
    DL_LAUNCH(ctx, K_PREP, 4.0 * n + 4.0 * words_used,
              hasout_kernel<<<grid_for(words_used, T256, ctx), T256, 0, ctx.stream>>>(g.csr.off, n, words_used,
                                                                                      ws.bit_hasout.as<u32>()));
    // base units (p, rows {p}) in offsets / jbuf[1]; the first step writes jbuf[0]
    DevBuf *ubuf = &ws.offsets, *ubuf_next = &ws.offsets_next;
    ctx.reserve(*ubuf, std::max<u64>(n, 1) * sizeof(Unit));
    ctx.reserve(ws.jbuf[1], std::max<u64>(n, 1) * 8);
    DL_CUDA(cudaMemsetAsync(&ctr->join, 0, sizeof(u64), ctx.stream));
    DL_LAUNCH(ctx, K_PREP, 8.0 * n + 24.0 * n,
              sg_base_units_kernel<<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(
                  g.csr.off, n, ws.jbuf[1].as<uint2>(), ubuf->as<Unit>(), &ctr->join));
    DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, &ctr->join, sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    u64 bound = ctx.host_scalars[0];
    const uint2 *rows = ws.jbuf[1].as<uint2>();
    u64 nunits = n, nrows = n;
    // 128-thread CTAs when 8 or more of them fit on an SM (short rows), else 512
    const size_t smem_s = sizeof(SgSmem<4>) + row_smem;
    int per_sm_s = 0, per_sm = 0;
    DL_CUDA(cudaFuncSetAttribute(sg_unit_step_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem_s));
    DL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_s, sg_unit_step_kernel<128>, 128, smem_s));
    DL_CUDA(cudaFuncSetAttribute(sg_unit_step_kernel<UT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    DL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sg_unit_step_kernel<UT>, UT, smem));
    const bool small = per_sm_s >= 8;
    const int nt = small ? 128 : UT;
    const u64 resident = (u64) ctx.sm_count * std::max(small ? per_sm_s : per_sm, 1);
    u64 nfull = 0;
    int slot = 0;
    // the free device memory, read once: a driver query per iteration costs
    // more than many of SG's small steps
    size_t free_b = 0, total_b = 0;
    DL_CUDA(cudaMemGetInfo(&free_b, &total_b));
    for (int it = 0;; ++it) {  // it 0: the base rule (sg.cu:170-217); then sg.cu:244-390
        pt.mark(it == 0 ? PH_INIT : PH_JOIN);
        u64 nnew = 0, next_units = 0, next_rows = 0, next_bound = 0;
        if (nunits && bound) {
            const unsigned grid = (unsigned) std::min<u64>(nunits, resident);
            const u64 warps = (u64) grid * (nt / 32);
            // New rows < bound; a warp's reservations are at least 3/4 used
            // (a switch leaves less than one summary word's rows, <= 1024,
            // behind). The buffer is also capped by the device memory left; a
            // step that overflows it reports DL_DEVERR_CAPACITY and the caller
            // reruns the program on the sorted runs.
            const u64 need = bound + bound / 3 + warps * WCHUNK;
            // rows (8 B) at most 1/16 of the memory free at the start, unit
            // slots (16 B, at most one per row) at most 1/8
            const u64 cap_rows = std::max<u64>(warps * WCHUNK, (u64) free_b / 16 / 8);
            const u64 ocap = std::min(need, cap_rows);
            DevBuf &obuf = ws.jbuf[slot];
            ctx.reserve(obuf, ocap * 8);
            const u64 ucap = ocap + warps * UCHUNK;  // every unit written holds at least one row
            ctx.reserve(*ubuf_next, ucap * sizeof(Unit));
            DL_CUDA(cudaMemsetAsync(ctr, 0, sizeof(StepCounters), ctx.stream));
            pt.mark(PH_DEDUP);
            if (small)
                DL_LAUNCH(ctx, K_BITMAP_EXPAND, 8.0 * nrows + 16.0 * nunits,
                          sg_unit_step_kernel<128><<<grid, 128, smem_s, ctx.stream>>>(
                              g.csr.off, g.csr.val, rows, ubuf->as<Unit>(), nunits, m, stride, (u32) words_used,
                              obuf.as<uint2>(), ocap, ubuf_next->as<Unit>(), ucap, unit_rows,
                              ws.bit_hasout.as<u32>(), ctr, &ctx.ctrl->err, it == 0 ? 1 : 0));
            else
                DL_LAUNCH(ctx, K_BITMAP_EXPAND, 8.0 * nrows + 16.0 * nunits,
                          sg_unit_step_kernel<UT><<<grid, UT, smem, ctx.stream>>>(
                              g.csr.off, g.csr.val, rows, ubuf->as<Unit>(), nunits, m, stride, (u32) words_used,
                              obuf.as<uint2>(), ocap, ubuf_next->as<Unit>(), ucap, unit_rows,
                              ws.bit_hasout.as<u32>(), ctr, &ctx.ctrl->err, it == 0 ? 1 : 0));
            DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, ctr, sizeof(StepCounters), cudaMemcpyDeviceToHost, ctx.stream));
            ctx.sync();  // a capacity overflow throws DL_ERR_OVERFLOW here
            next_rows = ctx.host_scalars[5];
            next_bound = ctx.host_scalars[2];
            next_units = ctx.host_scalars[3];
            nnew = ctx.host_scalars[4];
            ctx.prof_add_bytes(K_BITMAP_EXPAND, 8.0 * next_rows + 16.0 * next_units);
            rows = obuf.as<uint2>();
            slot ^= 1;
            std::swap(ubuf, ubuf_next);
        }
        pt.mark(PH_MERGE);
        nfull += nnew;
        if (it > 0) {
            r.deltas.push_back((i64) nnew);
            r.joins.push_back((i64) nrows);
            r.fulls.push_back((i64) nfull);
        }
        nunits = next_units;
        nrows = next_rows;
        bound = next_bound;
        if (it > 0 && nnew == 0) break;  // |full| unchanged
        if (it > 0 && opt.max_iterations > 0 && it >= opt.max_iterations) break;
    }
    pt.mark(PH_FINAL);
    // result rows in the reference's SG order (x, y) by (x, y): straight from
    // M's rows when they are copied out
    if (nfull) {
        ctx.reserve(ws.offsets, (n + 1) * 8);
        u64 *counts = ws.offsets.as<u64>();
        DL_LAUNCH(ctx, K_BITMAP_EXTRACT, 4.0 * n * words_used,
                  bitmat_row_popc_kernel<<<grid_for(n * 32, T256, ctx, 8), T256, 0, ctx.stream>>>(
                      m, n, stride, words_used, reinterpret_cast<unsigned long long *>(counts)));
        ctx.reserve(ws.w0, (n + 1) * 8);
        const u64 total = exclusive_scan(ctx, counts, n, ws.w0.as<u64>());
        if (total != nfull)
            throw Error(DL_ERR_INTERNAL, "bit matrix holds " + std::to_string(total) + " tuples, expected " +
                                             std::to_string(nfull));
        r.bm_t = M;
        M = DevBuf();
        r.bm_first = ws.w0;
        ws.w0 = DevBuf();
        r.bm_n = n;
        r.bm_stride = stride;
        r.bm_words = words_used;
        r.bm_row_first = true;
    }
    r.from_bitmat = true;
    return nfull;
}

}  // namespace detail

// One wave of the extraction kernel (every CTA resident at once; rows are
// strided over them), so no partial second wave runs at low occupancy.
static unsigned extract_grid(Context &ctx, u64 n) {
    using namespace detail;
    int per_sm = 0;
    DL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bitmat_extract_rows_kernel<true>, EX_THREADS, 0));
    const u64 wave = (u64) ctx.sm_count * std::max(per_sm, 1);
    return (unsigned) std::max<u64>(1, std::min<u64>(wave, (n + EX_THREADS / 32 - 1) / (EX_THREADS / 32)));
}

// The result rows of a bit-matrix run leave in units: TC's column blocks
// (1024 targets: rows (x, z) ordered by (z, x), from the matrix's columns)
// or SG's matrix rows (rows (x, y) ordered by (x, y)).
u64 bitmat_units(const Run &r) {
    using namespace detail;
    return r.bm_cols ? r.bm_stride / CX_WORDS : r.bm_n;
}

// Index into bm_first of the first target (TC) or row (SG) of `unit`; n for
// the end.
u64 bitmat_unit_index(const Run &r, u64 unit) {
    using namespace detail;
    return std::min<u64>(r.bm_n, r.bm_cols ? unit * CX_TARGETS : unit);
}

// The rows of units [u0, u1) into their places in `out` (device memory, all
// result rows). Units are the rows of the stored matrix (SG's M, TC's
// transpose) or, for TC from M's columns, its column blocks.
void bitmat_extract_rows(Context &ctx, const Run &r, int32_t *out, u64 u0, u64 u1) {
    using namespace detail;
    if (r.info.output_rows == 0 || u0 >= u1) return;
    const u64 n = r.bm_n;
    if (!r.bm_cols) {
        if (r.bm_row_first)
            DL_LAUNCH(ctx, K_BITMAP_EXTRACT, 4.0 * (u1 - u0) * r.bm_words,
                      bitmat_extract_rows_kernel<true><<<extract_grid(ctx, u1 - u0), EX_THREADS, 0, ctx.stream>>>(
                          r.bm_t.as<u32>(), u0, u1, r.bm_stride, r.bm_words, r.bm_first.as<u64>(),
                          r.ids.as<int32_t>(), r.ids_affine, r.id_base, reinterpret_cast<u64 *>(out)));
        else
            DL_LAUNCH(ctx, K_BITMAP_EXTRACT, 4.0 * (u1 - u0) * r.bm_words,
                      bitmat_extract_rows_kernel<false><<<extract_grid(ctx, u1 - u0), EX_THREADS, 0, ctx.stream>>>(
                          r.bm_t.as<u32>(), u0, u1, r.bm_stride, r.bm_words, r.bm_first.as<u64>(),
                          r.ids.as<int32_t>(), r.ids_affine, r.id_base, reinterpret_cast<u64 *>(out)));
        return;
    }
    const u64 xblocks = (n + CX_ROWS - 1) / CX_ROWS, tiles = (u1 - u0) * xblocks;
    DL_CUDA(cudaFuncSetAttribute(bitmat_column_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int) sizeof(ColSmem)));
    const unsigned cg = (unsigned) std::min<u64>(tiles, (u64) ctx.sm_count);
    // algorithmic bytes: the units' columns of the matrix and their offsets
    // (the rows' 8 bytes each are added by the caller)
    DL_LAUNCH(ctx, K_BITMAP_EXTRACT, 128.0 * xblocks * CX_ROWS * (u1 - u0) + 4.0 * xblocks * CX_TARGETS * (u1 - u0),
              bitmat_column_rows_kernel<<<cg, CX_THREADS, sizeof(ColSmem), ctx.stream>>>(
                  r.bm_t.as<u32>(), r.bm_live.as<u32>(), n, r.bm_stride, xblocks, u0 * xblocks, tiles,
                  r.bm_off.as<u32>(),
                  r.bm_first.as<u64>(), r.ids.as<int32_t>(), r.ids_affine, r.id_base, reinterpret_cast<u64 *>(out)));
}

}  // namespace dl
