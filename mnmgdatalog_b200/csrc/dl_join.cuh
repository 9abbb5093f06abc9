// Index sources for the join's count and emit passes (see dl_join.cu).
#pragma once

#include "dl_internal.h"
#include "dl_scan.cuh"

namespace dl {

constexpr int JN_THREADS = 256;
constexpr int JN_TILE = 2048;  // merged (probe row + output) slots per CTA

struct JoinSmem {
    u64 obeg[JN_TILE + 1];    // first output of each loaded probe row
    u64 begin[JN_TILE + 1];   // first match of each loaded probe row in the index
    u32 payload[JN_TILE + 1]; // probe value carried into the output
    u32 hist[8 * 256];        // radix histogram of emitted words (optional)
};

// Engine relation over dense node indices: off[k]..off[k+1] are the values
// of key k. Probe words are (k << bits) | v.
template <EmitKind K>
struct CsrSrc {
    const u32 *off;
    const u32 *val;
    const u64 *probe;
    int bits;
    static constexpr bool kSelfFilter = (K == EmitKind::ZV_NOSELF);
    static constexpr bool kWrite = true;
    static constexpr int kProfKind = K_JOIN_EMIT;
    static double prof_bytes(u64 n, u64 total) { return 8.0 * n + 16.0 * total; }
    __device__ __forceinline__ u64 degree(u64 i) const {
        const u32 k = (u32) (probe[i] >> bits);
        return (u64) (off[k + 1] - off[k]);
    }
    __device__ __forceinline__ void item(u64 i, u64 &begin, u64 &payload) const {
        const u64 p = probe[i];
        begin = off[(u32) (p >> bits)];
        payload = p & ((1ull << bits) - 1);
    }
    __device__ __forceinline__ u64 word(u64 idx, u64 v) const {
        const u64 z = val[idx];
        if (K == EmitKind::VZ) return (v << bits) | z;
        if (K == EmitKind::ZV_NOSELF && z == v) return ~0ull;
        return (z << bits) | v;
    }
};

// 16-byte slot of the C-ABI hash table; count == 0 marks an empty slot, so
// every int32 key (the reference's -1 sentinel included) can be stored.
struct __align__(16) HashSlot {
    int key;
    u32 begin;
    u32 count;
    u32 unused;
};

struct HashTable {
    DevBuf table;  // slots
    DevBuf vals;   // values of the key-sorted relation
    u64 slots = 0, distinct = 0, rows = 0;
};

// Probe words are raw Entity words (value << 32 | key); output words are
// Entity {key = indexed value, value = probe value} (common/join.cu:26-48).
struct HashSrc {
    const HashSlot *slots;
    const u32 *vals;
    u64 mask;
    const u64 *probe;
    static constexpr bool kSelfFilter = false;
    static constexpr bool kWrite = true;
    static constexpr int kProfKind = K_JOIN_EMIT;
    static double prof_bytes(u64 n, u64 total) { return 8.0 * n + 16.0 * total; }
    __device__ __forceinline__ void lookup(u32 key, u64 &begin, u64 &count) const {
        u64 h = fmix32(key) & mask;
        for (u64 step = 0; step <= mask; ++step) {
            const int4 s = __ldg(reinterpret_cast<const int4 *>(slots) + h);  // one 128-bit load
            if ((u32) s.z == 0u) break;
            if ((u32) s.x == key) {
                begin = (u32) s.y;
                count = (u32) s.z;
                return;
            }
            h = (h + 1) & mask;
        }
        begin = 0;
        count = 0;
    }
    __device__ __forceinline__ u64 degree(u64 i) const {
        u64 b, c;
        lookup((u32) probe[i], b, c);
        return c;
    }
    __device__ __forceinline__ void item(u64 i, u64 &begin, u64 &payload) const {
        const u64 p = probe[i];
        u64 c;
        lookup((u32) p, begin, c);
        payload = p >> 32;
    }
    __device__ __forceinline__ u64 word(u64 idx, u64 v) const { return (v << 32) | (u64) vals[idx]; }
};

// Key-sorted raw Entity relation searched by binary search (get_join_nl).
struct SortedSrc {
    const u64 *rel;
    u64 n_rel;
    const u64 *probe;
    static constexpr bool kSelfFilter = false;
    static constexpr bool kWrite = true;
    static constexpr int kProfKind = K_JOIN_EMIT;
    static double prof_bytes(u64 n, u64 total) { return 8.0 * n + 16.0 * total; }
    __device__ __forceinline__ u64 bound(int key, bool upper) const {
        u64 lo = 0, hi = n_rel;
        while (lo < hi) {
            const u64 mid = (lo + hi) >> 1;
            const int k = (int) (u32) rel[mid];
            if (k < key || (upper && k == key)) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    }
    __device__ __forceinline__ u64 degree(u64 i) const {
        const int key = (int) (u32) probe[i];
        return bound(key, true) - bound(key, false);
    }
    __device__ __forceinline__ void item(u64 i, u64 &begin, u64 &payload) const {
        const u64 p = probe[i];
        begin = bound((int) (u32) p, false);
        payload = p >> 32;
    }
    __device__ __forceinline__ u64 word(u64 idx, u64 v) const { return (v << 32) | (rel[idx] >> 32); }
};

// WCC min-label propagation (wcc.cu:255-387 as one kernel per iteration).
// Probe words are delta entries (node << 32) | label, the label being the
// node's label at the end of the previous iteration (Jacobi semantics, as
// in the reference's join of t_delta with the edges). Each match lowers the
// neighbour's label with atomicMin; the first thread that lowers a node in
// this iteration appends it to the next delta list.
struct WccSrc {
    const u32 *off;
    const u32 *val;
    const u64 *delta;
    u32 *label;
    u32 *flag;
    u32 *next_nodes;
    u32 *next_count;
    static constexpr bool kSelfFilter = false;
    static constexpr bool kWrite = false;
    static constexpr int kProfKind = K_WCC_PROPAGATE;
    static double prof_bytes(u64 n, u64 total) { return 8.0 * n + 36.0 * total; }
    __device__ __forceinline__ u64 degree(u64 i) const {
        const u32 k = (u32) (delta[i] >> 32);
        return (u64) (off[k + 1] - off[k]);
    }
    __device__ __forceinline__ void item(u64 i, u64 &begin, u64 &payload) const {
        const u64 p = delta[i];
        begin = off[(u32) (p >> 32)];
        payload = (u32) p;
    }
    __device__ __forceinline__ u64 word(u64 idx, u64 l) const {
        const u32 nbr = val[idx];
        const u32 lab = (u32) l;
        if (lab < label[nbr]) {  // cheap pre-check; atomicMin decides
            const u32 old = atomicMin(&label[nbr], lab);
            if (lab < old && atomicExch(&flag[nbr], 1u) == 0u) next_nodes[atomicAdd(next_count, 1u)] = nbr;
        }
        return 0;
    }
};

template <class Src>
__global__ void __launch_bounds__(JN_THREADS)
join_emit_kernel(Src src, u64 n_probe, const u64 *__restrict__ offsets, u64 total, const u64 *__restrict__ splits,
                 u64 *__restrict__ out, u64 *__restrict__ hist, int ndig, u64 *self_pairs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    JoinSmem &s = *reinterpret_cast<JoinSmem *>(smem_raw);
    const int tid = threadIdx.x;
    const u64 tile = blockIdx.x;
    const u64 d0 = tile * JN_TILE;
    const u64 d1 = min(d0 + JN_TILE, n_probe + total);
    const u64 i0 = splits[tile], i1 = splits[tile + 1];
    const u64 o0 = d0 - i0, o1 = d1 - i1;
    const u64 istart = i0 > 0 ? i0 - 1 : 0;
    const u32 ni = (u32) (i1 - istart);
    if (ndig > 0)
        for (int i = tid; i < ndig * 256; i += JN_THREADS) s.hist[i] = 0;
    for (u32 j = tid; j < ni; j += JN_THREADS) {
        const u64 gi = istart + j;
        u64 begin, payload;
        src.item(gi, begin, payload);
        s.obeg[j] = offsets[gi];
        s.begin[j] = begin;
        s.payload[j] = payload;
    }
    __syncthreads();
    u32 selfs = 0;
    u32 j = 0;
    for (u64 o = o0 + tid; o < o1; o += JN_THREADS) {
        // owner = last loaded row whose first output is <= o; rows only move
        // forward with o, so continue from the previous owner.
        u32 lo = j, hi = ni;
        while (lo < hi) {
            const u32 mid = (lo + hi) >> 1;
            if (s.obeg[mid] <= o) lo = mid + 1;
            else hi = mid;
        }
        j = lo - 1;
        const u64 w = src.word(s.begin[j] + (o - s.obeg[j]), s.payload[j]);
        if (!Src::kWrite) continue;
        out[o] = w;
        if (Src::kSelfFilter && w == ~0ull) ++selfs;
        if (ndig > 0) {
#pragma unroll
            for (int d = 0; d < 8; ++d)
                if (d < ndig) atomicAdd(&s.hist[d * 256 + ((w >> (8 * d)) & 255u)], 1u);
        }
    }
    if (Src::kSelfFilter) {
        selfs = warp_sum(selfs);
        if ((tid & 31) == 0 && selfs) atomicAdd((unsigned long long *) self_pairs, (unsigned long long) selfs);
    }
    if (ndig > 0) {
        __syncthreads();
        for (int i = tid; i < ndig * 256; i += JN_THREADS) {
            const u32 c = s.hist[i];
            if (c) atomicAdd((unsigned long long *) &hist[i], (unsigned long long) c);
        }
    }
}

// Join emit fused with the first LSD radix pass (bits 0-7 of the output
// words), for sources whose output words take their low byte from the probe
// row (CsrSrc<ZV> with bits >= 8: (z << bits) | v). The first pass of an LSD
// sort needs no stability -- there is no earlier order to keep -- so a tile
// ranks its words per digit with shared-memory atomics, reserves each
// digit's range with one atomic on a global cursor (cursor[d] starts at the
// digit's bucket start, from digit0_hist_kernel), stages the words grouped by
// digit and writes every run with consecutive stores.
struct JoinBucketSmem {
    u64 obeg[JN_TILE + 1];
    u64 begin[JN_TILE + 1];  // first match of each row; then the staged words
    u32 payload[JN_TILE + 1];
    u32 cnt[256];
    u32 pre[256];
    u64 base[256];
    u32 scratch[JN_THREADS / 32 + 1];
};

template <class Src>
__global__ void __launch_bounds__(JN_THREADS)
join_emit_bucket_kernel(Src src, u64 n_probe, const u64 *__restrict__ offsets, u64 total,
                        const u64 *__restrict__ splits, u64 *__restrict__ out,
                        unsigned long long *__restrict__ cursor, u32 *err) {
    static_assert(JN_THREADS == 256, "one thread per digit");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    JoinBucketSmem &s = *reinterpret_cast<JoinBucketSmem *>(smem_raw);
    constexpr u32 VT = JN_TILE / JN_THREADS;
    const int tid = threadIdx.x;
    const u64 tile = blockIdx.x;
    const u64 d0 = tile * JN_TILE;
    const u64 d1 = min(d0 + JN_TILE, n_probe + total);
    const u64 i0 = splits[tile], i1 = splits[tile + 1];
    const u64 o0 = d0 - i0, o1 = d1 - i1;
    const u64 istart = i0 > 0 ? i0 - 1 : 0;
    const u32 ni = (u32) (i1 - istart);
    const u32 no = (u32) (o1 - o0);
    s.cnt[tid] = 0;
    for (u32 j = tid; j < ni; j += JN_THREADS) {
        const u64 gi = istart + j;
        u64 begin, payload;
        src.item(gi, begin, payload);
        s.obeg[j] = offsets[gi];
        s.begin[j] = begin;
        s.payload[j] = payload;
    }
    __syncthreads();
    u64 wv[VT];
    u32 rk[VT];
    u32 j = 0;
#pragma unroll
    for (u32 k = 0; k < VT; ++k) {
        wv[k] = 0;
        rk[k] = 0;
        const u64 o = o0 + tid + (u64) k * JN_THREADS;
        if (o < o1) {
            u32 lo = j, hi = ni;  // owner: last loaded row whose first output is <= o
            while (lo < hi) {
                const u32 mid = (lo + hi) >> 1;
                if (s.obeg[mid] <= o) lo = mid + 1;
                else hi = mid;
            }
            j = lo - 1;
            const u64 w = src.word(s.begin[j] + (o - s.obeg[j]), s.payload[j]);
            wv[k] = w;
            rk[k] = atomicAdd(&s.cnt[w & 255u], 1u);
        }
    }
    __syncthreads();  // counts complete; s.begin no longer read
    u32 tot;
    const u32 c = s.cnt[tid];
    const u32 pre = block_exclusive_sum<JN_THREADS / 32>(c, s.scratch, &tot);
    s.pre[tid] = pre;
    if (c) s.base[tid] = (u64) atomicAdd(&cursor[tid], (unsigned long long) c) - pre;
    __syncthreads();
#pragma unroll
    for (u32 k = 0; k < VT; ++k) {
        const u64 o = o0 + tid + (u64) k * JN_THREADS;
        if (o < o1) s.begin[s.pre[wv[k] & 255u] + rk[k]] = wv[k];
    }
    __syncthreads();
    for (u32 i = tid; i < no; i += JN_THREADS) {
        const u64 w = s.begin[i];
        const u64 pos = s.base[w & 255u] + i;
        if (pos < total) out[pos] = w;
        else atomicOr(err, DL_DEVERR_CAPACITY);  // histogram and emit disagree: reported, never written
    }
}

// Degree-weighted histogram of the probe rows' low byte: the number of join
// output words per value of their bits 0-7 (for sources like the above).
template <class Src>
__global__ void __launch_bounds__(256) digit0_hist_kernel(Src src, const u64 *__restrict__ probe, u64 n,
                                                          unsigned long long *__restrict__ hist) {
    __shared__ unsigned long long h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64) gridDim.x * blockDim.x) {
        const u64 deg = src.degree(i);
        if (deg) atomicAdd(&h[probe[i] & 255u], (unsigned long long) deg);
    }
    __syncthreads();
    if (h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// hist[0..255] -> exclusive prefix (the digits' bucket starts), in place.
static __global__ void __launch_bounds__(256) bucket_starts_kernel(unsigned long long *hist) {
    __shared__ unsigned long long part[256 / 32];
    const u32 lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned long long v = hist[threadIdx.x];
    unsigned long long x = v;  // inclusive warp scan
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= (u32) d) x += y;
    }
    if (lane == 31) part[w] = x;
    __syncthreads();
    unsigned long long before = 0;
    for (u32 i = 0; i < w; ++i) before += part[i];
    hist[threadIdx.x] = before + x - v;
}

static __global__ void lbs_partition_kernel(const u64 *__restrict__ offsets, u64 n, u64 total, u64 n_splits,
                                     u64 *__restrict__ splits) {
    const u64 t = (u64) blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_splits) return;
    const u64 diag = min(t * (u64) JN_TILE, n + total);
    // rows are the "a" sequence (key = first output), outputs the "b" sequence
    // (key = position); a row precedes the outputs at or after its offset.
    u64 lo = diag > total ? diag - total : 0;
    u64 hi = diag < n ? diag : n;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (offsets[mid] <= diag - 1 - mid) lo = mid + 1;
        else hi = mid;
    }
    splits[t] = lo;
}

template <class Src>
struct DegreeOp {
    Src src;
    __device__ u64 operator()(u64 i) const { return src.degree(i); }
};

template <class Src>
u64 count_matches(Context &ctx, const Src &src, u64 n, u64 *offsets) {
    if (n == 0) return 0;
    const u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    u64 *lb = ctx.lookback_words(tiles);
    u32 *ctr = ctx.tile_counter(48);
    u64 *tot = &ctx.ctrl->scalar[2];
    DL_CUDA(cudaMemsetAsync(ctr, 0, sizeof(u32), ctx.stream));
    DL_LAUNCH(ctx, K_JOIN_COUNT, 16.0 * n, scan_kernel<DegreeOp<Src>><<<(unsigned) tiles, SCAN_THREADS, 0, ctx.stream>>>(
        DegreeOp<Src>{src}, n, offsets, lb, ctr, ctx.next_epoch(), &ctx.ctrl->err, tot));
    DL_CUDA(cudaMemcpyAsync(ctx.host_scalars, tot, sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    return ctx.host_scalars[0];
}

template <class Src>
void emit_matches(Context &ctx, const Src &src, u64 n, const u64 *offsets, u64 total, u64 *out, u64 *hist, int ndig,
                  u64 *self_pairs) {
    if (total == 0) return;
    const u64 tiles = (n + total + JN_TILE - 1) / JN_TILE;
    ctx.lbs_splits.reserve((tiles + 1) * sizeof(u64));
    u64 *splits = ctx.lbs_splits.as<u64>();
    DL_LAUNCH(ctx, K_JOIN_PARTITION, 0, lbs_partition_kernel<<<(unsigned) ((tiles + 1 + 255) / 256), 256, 0, ctx.stream>>>(offsets, n, total, tiles + 1,
                                                                                     splits));
    auto kern = join_emit_kernel<Src>;
    DL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sizeof(JoinSmem)));
    DL_LAUNCH(ctx, Src::kProfKind, Src::prof_bytes(n, total), kern<<<(unsigned) tiles, JN_THREADS, sizeof(JoinSmem), ctx.stream>>>(src, n, offsets, total, splits, out, hist,
                                                                         ndig, self_pairs));
}

// Join of probe rows against the CSR (EmitKind::ZV, bits >= 8) with the
// output already grouped by bits 0-7 of its words (the first LSD pass).
void join_emit_bucketed(Context &ctx, const Csr &csr, const u64 *probe, u64 n_probe, int bits, const u64 *offsets,
                        u64 total, u64 *out);

HashTable *hash_table_build(Context &ctx, const u64 *rel, u64 n, double load_factor);
u64 hash_join_count(Context &ctx, const HashTable &ht, const u64 *probe, u64 n, u64 *offsets);
void hash_join_emit(Context &ctx, const HashTable &ht, const u64 *probe, u64 n, const u64 *offsets, u64 total, u64 *out);
u64 sorted_join_count(Context &ctx, const u64 *rel, u64 n_rel, const u64 *probe, u64 n, u64 *offsets);
void sorted_join_emit(Context &ctx, const u64 *rel, u64 n_rel, const u64 *probe, u64 n, const u64 *offsets, u64 total,
                      u64 *out);

}  // namespace dl
