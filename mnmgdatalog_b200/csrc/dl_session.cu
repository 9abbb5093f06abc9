// Multi-instance fixpoint session: the batched and served forms.
//
// Many independent queries of one program run as ONE union fixpoint. Every
// admitted instance gets its own contiguous range of node ranks, so its
// tuples never meet another instance's: joins, sorts, the set difference and
// the merge of one iteration process every active instance at once, and the
// per-iteration launch and synchronisation cost is paid once for all of them.
// Instances are admitted at any iteration boundary (continuous batching):
// their edges are appended to the union's offset table (their ranks are above
// every rank in use, so the table stays sorted) and their initial delta joins
// the next iteration. Each instance keeps its own iteration count and delta
// sequence (a per-instance histogram of every iteration's delta) and leaves
// the union when it reaches its own fixpoint -- for WCC with the reference's
// stop rule an instance is frozen (its delta entries dropped) at the iteration
// where that rule fires, exactly where the reference program would stop.
// Results are bit-exact with running each query alone.
#include <algorithm>
#include <cstring>
#include <memory>

#include "dl_engine_detail.h"
#include "dl_join.cuh"
#include "dl_scan.cuh"
#include "dl_session.h"

namespace dl {
namespace {

using namespace detail;

#define GRID_STRIDE(i, n) \
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (u64) gridDim.x * blockDim.x)

// Instance of row r of a concatenation: last k with off[k] <= r.
__device__ __forceinline__ u32 segment_of(const u64 *__restrict__ off, u32 count, u64 r) {
    u32 a = 0, b = count;
    while (a < b) {
        const u32 m = (a + b) >> 1;
        if (off[m] <= r) a = m + 1;
        else b = m;
    }
    return a - 1;
}

// (instance << 32 | biased node id) for both columns of every row.
__global__ void session_tag_kernel(const int32_t *__restrict__ rows, u64 n, const u64 *__restrict__ off, u32 count,
                                   u64 *__restrict__ out) {
    GRID_STRIDE(r, n) {
        const u64 k = (u64) segment_of(off, count, r) << 32;
        out[2 * r] = k | ((u32) rows[2 * r] ^ 0x80000000u);
        out[2 * r + 1] = k | ((u32) rows[2 * r + 1] ^ 0x80000000u);
    }
}

// first[k] = index of the first tagged word of instance k (k in [0, count]).
__global__ void session_first_kernel(const u64 *__restrict__ u, u64 nu, u32 count, u64 *__restrict__ first) {
    GRID_STRIDE(k, (u64) count + 1) {
        const u64 target = k << 32;
        u64 l = 0, h = nu;
        while (l < h) {
            const u64 m = (l + h) >> 1;
            if (u[m] < target) l = m + 1;
            else h = m;
        }
        first[k] = l;
    }
}

__global__ void session_ids_kernel(const u64 *__restrict__ u, u64 nu, int32_t *__restrict__ ids) {
    GRID_STRIDE(i, nu) ids[i] = (int32_t) ((u32) u[i] ^ 0x80000000u);
}

__device__ __forceinline__ u64 lower_bound_u64(const u64 *__restrict__ a, u64 n, u64 x) {
    u64 l = 0, h = n;
    while (l < h) {
        const u64 m = (l + h) >> 1;
        if (a[m] < x) l = m + 1;
        else h = m;
    }
    return l;
}

// Rows of many instances -> words over union ranks (rank = base + position
// of (instance, id) among the sorted distinct tagged ids).
__global__ void session_pack_many_kernel(const int32_t *__restrict__ rows, u64 n, const u64 *__restrict__ off,
                                         u32 count, const u64 *__restrict__ u, u64 nu, u64 base, int bits,
                                         u64 *__restrict__ fwd, u64 *__restrict__ rev) {
    GRID_STRIDE(r, n) {
        const u64 k = (u64) segment_of(off, count, r) << 32;
        const u64 ra = base + lower_bound_u64(u, nu, k | ((u32) rows[2 * r] ^ 0x80000000u));
        const u64 rb = base + lower_bound_u64(u, nu, k | ((u32) rows[2 * r + 1] ^ 0x80000000u));
        if (fwd) fwd[r] = (ra << bits) | rb;
        if (rev) rev[r] = (rb << bits) | ra;
    }
}

// Appends the sorted words of ranks [lo, hi) to the union offset table:
// off[r] = base + (first word with key >= r) for r in [lo, hi].
__global__ void session_csr_kernel(const u64 *__restrict__ w, u64 n, int bits, u64 lo, u64 hi, u64 base,
                                   u32 *__restrict__ off, u32 *__restrict__ val) {
    GRID_STRIDE(k, hi - lo + 1) {
        const u64 target = (lo + k) << bits;
        u64 l = 0, h = n;
        while (l < h) {
            const u64 m = (l + h) >> 1;
            if (w[m] < target) l = m + 1;
            else h = m;
        }
        off[lo + k] = (u32) (base + l);
    }
    const u64 mask = (1ull << bits) - 1;
    GRID_STRIDE(i, n) val[base + i] = (u32) (w[i] & mask);
}

// Instance index of a rank: last active instance whose first rank <= r.
__device__ __forceinline__ u32 instance_of(const u64 *__restrict__ lo, u32 n, u64 r) {
    u32 a = 0, b = n;
    while (a < b) {
        const u32 m = (a + b) >> 1;
        if (lo[m] <= r) a = m + 1;
        else b = m;
    }
    return a - 1;
}

// Per-instance count of delta words; the rank is word >> shift.
__global__ void session_hist_kernel(const u64 *__restrict__ d, u64 n, int shift, const u64 *__restrict__ lo, u32 ninst,
                                    unsigned long long *__restrict__ cnt) {
    extern __shared__ u32 sh[];
    const bool smem = ninst <= 8192;
    if (smem)
        for (u32 i = threadIdx.x; i < ninst; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    GRID_STRIDE(i, n) {
        const u32 k = instance_of(lo, ninst, d[i] >> shift);
        if (k >= ninst) continue;  // below every active range: not counted
        if (smem) atomicAdd(&sh[k], 1u);
        else atomicAdd(&cnt[k], 1ull);
    }
    __syncthreads();
    if (smem)
        for (u32 i = threadIdx.x; i < ninst; i += blockDim.x)
            if (sh[i]) atomicAdd(&cnt[i], (unsigned long long) sh[i]);
}

// Word ranges of instances in the three sorted runs: for instance k (ranks
// lohi[k] .. lohi[n + k]) out[6k..6k+5] = [first, end) in run 0, 1 and 2.
struct Runs3 {
    const u64 *w[3];
    u64 n[3];
};
__global__ void session_bounds_kernel(Runs3 runs, const u64 *__restrict__ lohi, u32 n, int bits,
                                      u64 *__restrict__ out) {
    GRID_STRIDE(t, 6 * (u64) n) {
        const u64 k = t / 6, which = t % 6, r = which >> 1;
        const u64 target = (which & 1 ? lohi[n + k] : lohi[k]) << bits;
        out[t] = lower_bound_u64(runs.w[r], runs.n[r], target);
    }
}

__global__ void session_label_init_kernel(u32 *__restrict__ label, u32 *__restrict__ flag, u64 lo, u64 hi,
                                          u64 *__restrict__ delta) {
    GRID_STRIDE(i, hi - lo) {
        const u64 r = lo + i;
        label[r] = (u32) r;
        flag[r] = 0;
        delta[i] = (r << 32) | r;
    }
}

__global__ void session_next_delta_kernel(const u32 *__restrict__ nodes, u64 count, const u32 *__restrict__ label,
                                          u32 *__restrict__ flag, u64 *__restrict__ delta) {
    GRID_STRIDE(i, count) {
        const u32 v = nodes[i];
        delta[i] = ((u64) v << 32) | label[v];
        flag[v] = 0;
    }
}

// Slot t of a concatenation of instance rank ranges (instance k from slot
// off[k], ranks lo[k]...): counts the component label of the node into
// cnt[off[k] + label - lo[k]] and copies the node's label.
__global__ void session_wcc_count_kernel(const u32 *__restrict__ label, const u64 *__restrict__ lo,
                                         const u64 *__restrict__ off, u32 n, u64 total, u32 *__restrict__ cnt,
                                         u32 *__restrict__ labels_out) {
    GRID_STRIDE(t, total) {
        const u32 k = segment_of(off, n, t);
        const u32 l = label[lo[k] + (t - off[k])];
        labels_out[t] = l;
        atomicAdd(&cnt[off[k] + (l - lo[k])], 1u);
    }
}

struct NonZero {
    const u32 *c;
    __device__ __forceinline__ u64 degree(u64 i) const { return c[i] != 0u; }
};

// Components of every instance (local ranks, ascending), the largest size
// per instance, and where each instance's components start.
__global__ void session_wcc_comp_kernel(const u32 *__restrict__ cnt, const u64 *__restrict__ pos,
                                        const u64 *__restrict__ off, u32 n, u64 total, u32 *__restrict__ comp,
                                        unsigned long long *__restrict__ largest, u64 *__restrict__ start) {
    GRID_STRIDE(t, total) {
        const u32 k = segment_of(off, n, t);
        if (t == off[k]) start[k] = pos[t];
        const u32 c = cnt[t];
        if (c) {
            comp[pos[t]] = (u32) (t - off[k]);
            atomicMax(&largest[k], (unsigned long long) c);
        }
    }
}

// Keep delta words whose instance is still active (freezing finished ones).
struct KeepActive {
    const u64 *lo;
    const uint8_t *live;
    u32 n;
    int shift;
    __device__ bool operator()(u64 cur, u64, bool) const {
        const u32 k = instance_of(lo, n, cur >> shift);
        return k < n && live[k] != 0;
    }
};

template <bool KeyFirst>
__global__ void session_unpack_kernel(const u64 *__restrict__ w, u64 n, int bits, u64 base,
                                      const int32_t *__restrict__ ids, int32_t *__restrict__ out) {
    const u64 mask = (1ull << bits) - 1;
    GRID_STRIDE(i, n) {
        const u64 x = w[i];
        const int32_t hi = ids[(x >> bits) - base], lo = ids[(x & mask) - base];
        int2 r;
        r.x = KeyFirst ? hi : lo;
        r.y = KeyFirst ? lo : hi;
        reinterpret_cast<int2 *>(out)[i] = r;
    }
}

__global__ void session_unpack_comp_kernel(const u32 *__restrict__ comp, u64 n, const int32_t *__restrict__ ids,
                                           int32_t *__restrict__ out) {
    GRID_STRIDE(i, n) {
        int2 r;
        r.x = ids[comp[i]];
        r.y = 0;
        reinterpret_cast<int2 *>(out)[i] = r;
    }
}

// labels: union label rank of each local node; ids indexed by local rank.
__global__ void session_unpack_labels_kernel(const u32 *__restrict__ label, u64 lo, u64 n,
                                             const int32_t *__restrict__ ids, int32_t *__restrict__ out) {
    GRID_STRIDE(i, n) out[i] = ids[label[i] - lo];
}

// Keeps the words whose instance (rank = word >> shift) is live.
template <class Keep>
u64 session_select(Context &ctx, u64 *buf, u64 n, Keep keep, int slot) {
    if (n == 0) return 0;
    const u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    u64 *lb = ctx.lookback_words(tiles);
    u32 *ctr = ctx.tile_counter(slot);
    u64 *cnt = &ctx.ctrl->scalar[28];
    DL_CUDA(cudaMemsetAsync(ctr, 0, sizeof(u32), ctx.stream));
    DL_LAUNCH(ctx, K_SELECT, 16.0 * n,
              select_kernel<Keep><<<(unsigned) tiles, SCAN_THREADS, 0, ctx.stream>>>(
                  buf, n, buf, keep, lb, ctr, ctx.next_epoch(), &ctx.ctrl->err, cnt));
    DL_CUDA(cudaMemcpyAsync(ctx.host_scalars + 4, cnt, sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    return ctx.host_scalars[4];
}

// Grows a buffer keeping its first `keep` bytes.
void grow_keep(Context &ctx, DevBuf &b, size_t bytes, size_t keep) {
    if (b.p && b.cap >= bytes) return;
    DevBuf nb;
    ctx.allocate(nb, std::max(bytes, b.cap * 3 / 2));
    if (keep && b.p) DL_CUDA(cudaMemcpyAsync(nb.p, b.p, keep, cudaMemcpyDeviceToDevice, ctx.stream));
    ctx.sync();
    b.release();
    b = nb;
}

}  // namespace

struct SessionImpl {
    Context ctx;  // private workspace; shares the caller's stream
    Context *parent = nullptr;
    int program = DL_PROGRAM_TC;
    dl_options opt{};
    int bits = 30;
    u64 rank_cap = 0;
    u64 next_rank = 0;
    DevBuf off, val;  // union offset table over ranks, values
    u64 n_vals = 0;
    FullSet F = [] {
        FullSet f;
        f.three = true;
        return f;
    }();
    u64 dead = 0;  // words of finished instances still in the full runs
    DevBuf delta;  // union delta (probe of the next iteration)
    u64 n_delta = 0;
    DevBuf label, flag, nextl;  // WCC
    DevBuf inst_lo, inst_hi;    // device copies of the active instances' rank ranges
    DevBuf counts;              // per instance delta counts
    DevBuf range_lo;            // first ranks of the instances of a range count
    DevBuf admit_off, admit_first;  // row offsets / first tagged ids of an admission
    DevBuf live;                // per active instance flag (WCC freezing)
    std::vector<SessionInstance> inst;
    std::vector<i64> active;    // instance ids in rank order
    std::vector<i64> finished;  // finished since the last poll
    bool inst_dirty = true;
};

namespace {

Graph union_graph(SessionImpl &s) {
    Graph g;
    g.n_ids = (u32) s.next_rank;
    g.bits = s.bits;
    g.csr.off = s.off.as<u32>();
    g.csr.val = s.val.as<u32>();
    g.csr.n_keys = (u32) s.next_rank;
    g.csr.n_vals = s.n_vals;
    // both rank fields are below next_rank: sort only the bits that can vary
    g.nwin = plan_windows(s.bits, bits_for(std::max<u64>(s.next_rank, 2)), g.win);
    return g;
}

// Sorts the n words of buf (alt: ping-pong) whose rank fields are below
// 2^used_bits and drops duplicates.
u64 *sort_unique_fields(Context &ctx, DevBuf &buf, DevBuf &alt, u64 n, int field_bits, int used_bits, u64 &n_out) {
    ctx.reserve(alt, std::max<u64>(n, 1) * 8);
    int w[8];
    const int nw = plan_windows(field_bits, used_bits, w);
    u64 *r = radix_sort_windows(ctx, buf.as<u64>(), alt.as<u64>(), n, w, nw);
    n_out = unique_words(ctx, r, n, r);
    return r;
}

// Inserts the words of a brand-new key range into the full relation.
void full_insert_new(SessionImpl &s, const u64 *w, u64 n) {
    Context &ctx = s.ctx;
    Workspace &ws = ctx.ws;
    FullSet &F = s.F;
    if (n == 0) return;
    // new ranks are above every word in the runs: the merge appends
    ctx.reserve(ws.tiny[1 - F.tcur], (F.ntiny + n) * 8);
    merge_words(ctx, ws.tiny[F.tcur].as<u64>(), F.ntiny, w, n, ws.tiny[1 - F.tcur].as<u64>(), Codec::Raw);
    F.tcur = 1 - F.tcur;
    F.ntiny += n;
    if (F.ntiny * ctx.tune.small_ratio >= F.nsmall) fold_tiny(ctx, F);  // also when the small run is empty
    if (F.nsmall && F.nsmall * ctx.tune.small_ratio >= F.nbig) {
        fold_tiny(ctx, F);
        ctx.reserve(ws.full[1 - F.cur], (F.nbig + F.nsmall) * 8);
        merge_words(ctx, ws.full[F.cur].as<u64>(), F.nbig, ws.small[F.scur].as<u64>(), F.nsmall,
                    ws.full[1 - F.cur].as<u64>(), Codec::Raw);
        F.cur = 1 - F.cur;
        F.nbig += F.nsmall;
        F.nsmall = 0;
        F.sample_ok = false;
        F.ssample_ok = false;
    }
}

void delta_append(SessionImpl &s, const u64 *w, u64 n) {
    if (n == 0) return;
    grow_keep(s.ctx, s.delta, (s.n_delta + n) * 8, s.n_delta * 8);
    DL_CUDA(cudaMemcpyAsync(s.delta.as<u64>() + s.n_delta, w, n * 8, cudaMemcpyDeviceToDevice, s.ctx.stream));
    s.n_delta += n;
}

void upload_active(SessionImpl &s) {
    if (!s.inst_dirty) return;
    const u64 na = s.active.size();
    std::vector<u64> lo(std::max<u64>(na, 1)), hi(std::max<u64>(na, 1));
    for (u64 i = 0; i < na; ++i) {
        lo[i] = s.inst[s.active[i]].rank_lo;
        hi[i] = s.inst[s.active[i]].rank_hi;
    }
    s.ctx.reserve(s.inst_lo, lo.size() * 8);
    s.ctx.reserve(s.inst_hi, hi.size() * 8);
    DL_CUDA(cudaMemcpyAsync(s.inst_lo.p, lo.data(), na * 8, cudaMemcpyHostToDevice, s.ctx.stream));
    DL_CUDA(cudaMemcpyAsync(s.inst_hi.p, hi.data(), na * 8, cudaMemcpyHostToDevice, s.ctx.stream));
    s.ctx.sync();  // lo/hi are host temporaries
    s.inst_dirty = false;
}

// Counts of the words of d (rank = word >> shift) per instance, given the
// instances' first ranks in increasing order on the device.
std::vector<u64> counts_by_lo(SessionImpl &s, const u64 *d, u64 n, int shift, const u64 *d_lo, u64 na) {
    Context &ctx = s.ctx;
    std::vector<u64> c(na, 0);
    if (na == 0 || n == 0) return c;
    ctx.reserve(s.counts, na * 8);
    DL_CUDA(cudaMemsetAsync(s.counts.p, 0, na * 8, ctx.stream));
    const unsigned smem = na <= 8192 ? (unsigned) (na * 4) : 0u;
    DL_LAUNCH(ctx, K_PREP, 8.0 * n,
              session_hist_kernel<<<grid_for(n, 256, ctx, 8), 256, smem, ctx.stream>>>(
                  d, n, shift, d_lo, (u32) na, (unsigned long long *) s.counts.p));
    DL_CUDA(cudaMemcpyAsync(c.data(), s.counts.p, na * 8, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    return c;
}

// Per-active-instance counts.
std::vector<u64> delta_counts(SessionImpl &s, const u64 *d, u64 n, int shift) {
    if (s.active.empty() || n == 0) return std::vector<u64>(s.active.size(), 0);
    upload_active(s);
    return counts_by_lo(s, d, n, shift, s.inst_lo.as<u64>(), s.active.size());
}

// Counts for the instances whose first ranks are `lo` (increasing).
std::vector<u64> range_counts(SessionImpl &s, const u64 *d, u64 n, int shift, const std::vector<u64> &lo) {
    if (lo.empty() || n == 0) return std::vector<u64>(lo.size(), 0);
    s.ctx.reserve(s.range_lo, lo.size() * 8);
    DL_CUDA(cudaMemcpyAsync(s.range_lo.p, lo.data(), lo.size() * 8, cudaMemcpyHostToDevice, s.ctx.stream));
    return counts_by_lo(s, d, n, shift, s.range_lo.as<u64>(), lo.size());  // syncs before `lo` goes
}

// A device block shared by the instances extracted or admitted together; its
// memory returns to the session's buffer cache with the last instance.
std::shared_ptr<DevBuf> make_block(Context &ctx, size_t bytes) {
    DevBuf *b = new DevBuf;
    try {
        ctx.reserve(*b, std::max<size_t>(bytes, 8));
    } catch (...) {
        delete b;
        throw;
    }
    Context *c = &ctx;
    return std::shared_ptr<DevBuf>(b, [c](DevBuf *x) {
        c->give_back(*x);
        delete x;
    });
}

// Uploads the rank ranges of `ids` ([lo..., hi...]) to s.range_lo.
void upload_ranges(SessionImpl &s, const std::vector<i64> &ids) {
    const u64 n = ids.size();
    std::vector<u64> h(2 * n);
    for (u64 k = 0; k < n; ++k) {
        h[k] = s.inst[ids[k]].rank_lo;
        h[n + k] = s.inst[ids[k]].rank_hi;
    }
    s.ctx.reserve(s.range_lo, 2 * n * 8);
    DL_CUDA(cudaMemcpyAsync(s.range_lo.p, h.data(), 2 * n * 8, cudaMemcpyHostToDevice, s.ctx.stream));
    s.ctx.sync();  // h is a host temporary
}

// Sorted words of finished TC/SG instances out of the full runs, into one
// block (each instance's words are a key range of each run).
void extract_words(SessionImpl &s, const std::vector<i64> &ids) {
    Context &ctx = s.ctx;
    Workspace &ws = ctx.ws;
    const u64 n = ids.size();
    upload_ranges(s, ids);
    ctx.reserve(s.counts, 6 * n * 8);
    Runs3 runs;
    runs.w[0] = ws.full[s.F.cur].as<u64>();
    runs.n[0] = s.F.nbig;
    runs.w[1] = ws.small[s.F.scur].as<u64>();
    runs.n[1] = s.F.nsmall;
    runs.w[2] = ws.tiny[s.F.tcur].as<u64>();
    runs.n[2] = s.F.ntiny;
    DL_LAUNCH(ctx, K_PREP, 0,
              session_bounds_kernel<<<grid_for(6 * n, 256, ctx, 4), 256, 0, ctx.stream>>>(
                  runs, s.range_lo.as<u64>(), (u32) n, s.bits, s.counts.as<u64>()));
    std::vector<u64> hb(6 * n);
    DL_CUDA(cudaMemcpyAsync(hb.data(), s.counts.p, 6 * n * 8, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    u64 total = 0, pair_max = 0;
    for (u64 k = 0; k < n; ++k) {
        const u64 na = hb[6 * k + 1] - hb[6 * k], nb = hb[6 * k + 3] - hb[6 * k + 2], nc = hb[6 * k + 5] - hb[6 * k + 4];
        total += na + nb + nc;
        if (na && nb && nc) pair_max = std::max(pair_max, na + nb);
    }
    auto block = make_block(ctx, total * 8);
    DevBuf tmp;  // run 0 + run 1 slices of an instance that has words in all three runs
    if (pair_max) ctx.reserve(tmp, pair_max * 8);
    u64 at = 0;
    for (u64 k = 0; k < n; ++k) {
        SessionInstance &in = s.inst[ids[k]];
        const u64 *src[3];
        u64 len[3];
        int m = 0;
        for (int r = 0; r < 3; ++r) {
            const u64 b = hb[6 * k + 2 * r], e = hb[6 * k + 2 * r + 1];
            if (e > b) {
                src[m] = runs.w[r] + b;
                len[m] = e - b;
                ++m;
            }
        }
        u64 *dst = block->as<u64>() + at;
        u64 cnt = 0;
        if (m == 1) {
            DL_CUDA(cudaMemcpyAsync(dst, src[0], len[0] * 8, cudaMemcpyDeviceToDevice, ctx.stream));
            cnt = len[0];
        } else if (m == 2) {
            merge_words(ctx, src[0], len[0], src[1], len[1], dst, Codec::Raw);
            cnt = len[0] + len[1];
        } else if (m == 3) {
            merge_words(ctx, src[0], len[0], src[1], len[1], tmp.as<u64>(), Codec::Raw);
            merge_words(ctx, tmp.as<u64>(), len[0] + len[1], src[2], len[2], dst, Codec::Raw);
            cnt = len[0] + len[1] + len[2];
        }
        in.result_block = block;
        in.result_off = at;
        in.n_result = cnt;
        at += cnt;
        s.dead += cnt;
    }
    if (pair_max) {
        ctx.sync();  // the merges that read tmp are done
        ctx.give_back(tmp);
    }
}

// Components (ascending local ranks), largest component and per-node labels
// of finished WCC instances, all in one pass over their rank ranges.
void extract_components(SessionImpl &s, const std::vector<i64> &ids) {
    Context &ctx = s.ctx;
    const u64 n = ids.size();
    std::vector<u64> off(n + 1, 0);
    for (u64 k = 0; k < n; ++k) off[k + 1] = off[k] + s.inst[ids[k]].n_ids;
    const u64 total = off[n];
    upload_ranges(s, ids);
    // s.counts: slot offsets [n + 1] then largest [n] then component starts [n]
    ctx.reserve(s.counts, (3 * n + 1) * 8);
    u64 *d_off = s.counts.as<u64>(), *d_big = d_off + n + 1, *d_start = d_big + n;
    DL_CUDA(cudaMemcpyAsync(d_off, off.data(), (n + 1) * 8, cudaMemcpyHostToDevice, ctx.stream));
    DL_CUDA(cudaMemsetAsync(d_big, 0, n * 8, ctx.stream));
    DevBuf cnt, pos;
    ctx.reserve(cnt, std::max<u64>(total, 1) * 4);
    ctx.reserve(pos, std::max<u64>(total, 1) * 8);
    DL_CUDA(cudaMemsetAsync(cnt.p, 0, total * 4, ctx.stream));
    auto labels = make_block(ctx, total * 4);
    const u64 *lo = s.range_lo.as<u64>();
    DL_LAUNCH(ctx, K_PREP, 0,
              session_wcc_count_kernel<<<grid_for(total, 256, ctx, 8), 256, 0, ctx.stream>>>(
                  s.label.as<u32>(), lo, d_off, (u32) n, total, cnt.as<u32>(), labels->as<u32>()));
    const u64 nc = count_matches(ctx, NonZero{cnt.as<u32>()}, total, pos.as<u64>());
    auto comps = make_block(ctx, nc * 4);
    DL_LAUNCH(ctx, K_PREP, 0,
              session_wcc_comp_kernel<<<grid_for(total, 256, ctx, 8), 256, 0, ctx.stream>>>(
                  cnt.as<u32>(), pos.as<u64>(), d_off, (u32) n, total, comps->as<u32>(),
                  (unsigned long long *) d_big, d_start));
    std::vector<u64> h(2 * n);
    DL_CUDA(cudaMemcpyAsync(h.data(), d_big, 2 * n * 8, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    for (u64 k = 0; k < n; ++k) {
        SessionInstance &in = s.inst[ids[k]];
        const u64 start = h[n + k], end = k + 1 < n ? h[n + k + 1] : nc;
        in.result_block = comps;
        in.result_off = start;
        in.n_result = end - start;
        in.largest = (i64) h[k];
        in.labels_block = labels;
        in.labels_off = off[k];
    }
    ctx.give_back(cnt);
    ctx.give_back(pos);
}

void mark_done(SessionImpl &s, SessionInstance &in) {
    in.active = false;
    in.done = true;
    s.finished.push_back(in.id);
}

void finish(SessionImpl &s, const std::vector<i64> &ids) {
    if (ids.empty()) return;
    if (s.program == DL_PROGRAM_WCC) extract_components(s, ids);
    else extract_words(s, ids);
    for (i64 id : ids) mark_done(s, s.inst[id]);
}

// Drops the union state once no instance is active: ranks, offsets and the
// full relation start again from zero (results live with their instances).
void reset_if_idle(SessionImpl &s) {
    if (!s.active.empty()) return;
    s.next_rank = 0;
    s.n_vals = 0;
    s.F = FullSet();
    s.F.three = true;
    s.dead = 0;
    s.n_delta = 0;
    s.inst_dirty = true;
}

// Words whose key rank lies in an active instance's range.
struct KeepLive {
    const u64 *lo, *hi;
    u32 n;
    int shift;
    __device__ bool operator()(u64 cur, u64, bool) const {
        const u64 r = cur >> shift;
        const u32 k = instance_of(lo, n, r);
        return k < n && r < hi[k];
    }
};

// Removes the words of finished instances from the full runs once they are
// at least half of the full relation.
void maybe_compact(SessionImpl &s) {
    if (s.program == DL_PROGRAM_WCC || s.active.empty()) return;
    const u64 total = s.F.size();
    if (s.dead == 0 || s.dead * 2 < total) return;
    Context &ctx = s.ctx;
    Workspace &ws = ctx.ws;
    upload_active(s);
    KeepLive keep{s.inst_lo.as<u64>(), s.inst_hi.as<u64>(), (u32) s.active.size(), s.bits};
    s.F.nbig = session_select(ctx, ws.full[s.F.cur].as<u64>(), s.F.nbig, keep, 60);
    s.F.nsmall = session_select(ctx, ws.small[s.F.scur].as<u64>(), s.F.nsmall, keep, 60);
    s.F.ntiny = session_select(ctx, ws.tiny[s.F.tcur].as<u64>(), s.F.ntiny, keep, 60);
    s.F.sample_ok = false;
    s.F.ssample_ok = false;
    if (s.F.nsmall == 0) fold_tiny(ctx, s.F);  // a tiny run needs a small run
    s.dead = 0;
}

void retire(SessionImpl &s, const std::vector<i64> &done, const std::vector<i64> &still) {
    finish(s, done);
    if (still.size() != s.active.size()) {
        s.active = still;
        s.inst_dirty = true;
    }
    reset_if_idle(s);
}

u64 wcc_step(SessionImpl &s) {
    Context &ctx = s.ctx;
    Workspace &ws = ctx.ws;
    ctx.reserve(ws.offsets, std::max<u64>(s.n_delta, 1) * 8);
    u32 *next_count = reinterpret_cast<u32 *>(&ctx.ctrl->scalar[32]);
    DL_CUDA(cudaMemsetAsync(next_count, 0, 4, ctx.stream));
    Graph g = union_graph(s);
    WccSrc src{g.csr.off, g.csr.val, s.delta.as<u64>(), s.label.as<u32>(), s.flag.as<u32>(), s.nextl.as<u32>(),
               next_count};
    const u64 total = count_matches(ctx, src, s.n_delta, ws.offsets.as<u64>());  // wcc.cu:255-300
    if (total) emit_matches(ctx, src, s.n_delta, ws.offsets.as<u64>(), total, nullptr, nullptr, 0, nullptr);
    DL_CUDA(cudaMemcpyAsync(ctx.host_scalars + 6, next_count, 4, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    const u64 nn = *reinterpret_cast<u32 *>(ctx.host_scalars + 6);
    grow_keep(ctx, s.delta, std::max<u64>(nn, 1) * 8, 0);  // the emit has read the old delta
    if (nn)  // rebuild the delta from the appended nodes
        DL_LAUNCH(ctx, K_PREP, 0,
                  session_next_delta_kernel<<<grid_for(nn, 256, ctx, 16), 256, 0, ctx.stream>>>(
                      s.nextl.as<u32>(), nn, s.label.as<u32>(), s.flag.as<u32>(), s.delta.as<u64>()));
    s.n_delta = nn;
    const std::vector<u64> c = delta_counts(s, s.delta.as<u64>(), nn, 32);
    std::vector<i64> still, done;
    std::vector<uint8_t> live(s.active.size(), 1);
    bool frozen_rows = false;
    for (u64 k = 0; k < s.active.size(); ++k) {
        SessionInstance &in = s.inst[s.active[k]];
        const i64 cnt = (i64) c[k];
        in.deltas.push_back(cnt);
        bool stop = s.opt.wcc_stop == DL_WCC_STOP_FIXPOINT ? cnt == 0 : cnt == in.prev_delta;  // wcc.cu:366-383
        in.prev_delta = cnt;
        if (!stop && s.opt.max_iterations > 0 && (int) in.deltas.size() >= s.opt.max_iterations) stop = true;
        if (stop) {
            live[k] = 0;
            frozen_rows |= cnt != 0;
            done.push_back(s.active[k]);
        } else {
            still.push_back(s.active[k]);
        }
    }
    if (frozen_rows) {  // an instance stopped with a non-empty delta: drop its rows
        ctx.reserve(s.live, live.size());
        DL_CUDA(cudaMemcpyAsync(s.live.p, live.data(), live.size(), cudaMemcpyHostToDevice, ctx.stream));
        KeepActive keep{s.inst_lo.as<u64>(), s.live.as<uint8_t>(), (u32) s.active.size(), 32};
        s.n_delta = session_select(ctx, s.delta.as<u64>(), s.n_delta, keep, 61);  // syncs: `live` may go
    }
    retire(s, done, still);
    return s.active.size();
}

u64 fixpoint_step(SessionImpl &s) {
    Context &ctx = s.ctx;
    Workspace &ws = ctx.ws;
    Graph g = union_graph(s);
    PhaseTimer pt(ctx, false);
    u64 nnew = 0;
    u64 *dnew = nullptr;
    if (s.program == DL_PROGRAM_TC) {  // tc.cu:216-314
        u64 nj = 0;
        u64 *j = join_and_sort(ctx, g, s.delta.as<u64>(), s.n_delta, EmitKind::ZV, nj, nullptr, pt);
        dnew = absorb(ctx, s.F, j, nj, nnew);
    } else {  // sg.cu:244-390
        u64 n1 = 0, n2 = 0;
        u64 *j1 = join_and_sort(ctx, g, s.delta.as<u64>(), s.n_delta, EmitKind::VZ, n1, nullptr, pt);
        if (n1) n1 = unique_words(ctx, j1, n1, j1);
        if (n1) {
            u64 *j2 = join_and_sort(ctx, g, j1, n1, EmitKind::VZ, n2, nullptr, pt);
            dnew = absorb(ctx, s.F, j2, n2, nnew);
        }
    }
    // the new delta sits in one of the join buffers: trade it for the old delta's buffer
    if (nnew) std::swap(s.delta, holder(ws, dnew));
    s.n_delta = nnew;
    const std::vector<u64> c = delta_counts(s, s.delta.as<u64>(), nnew, s.bits);
    std::vector<i64> still, done;
    for (u64 k = 0; k < s.active.size(); ++k) {
        SessionInstance &in = s.inst[s.active[k]];
        in.deltas.push_back((i64) c[k]);
        bool stop = c[k] == 0;  // |full| unchanged
        if (!stop && s.opt.max_iterations > 0 && (int) in.deltas.size() >= s.opt.max_iterations) stop = true;
        (stop ? done : still).push_back(s.active[k]);
    }
    if (!done.empty() && nnew && still.size() < s.active.size()) {
        // an instance stopped by max_iterations keeps rows in the delta: drop them
        bool rows_left = false;
        for (u64 k = 0; k < s.active.size(); ++k)
            if (c[k] && std::find(done.begin(), done.end(), s.active[k]) != done.end()) rows_left = true;
        if (rows_left) {
            std::vector<uint8_t> live(s.active.size(), 1);
            for (u64 k = 0; k < s.active.size(); ++k)
                if (std::find(done.begin(), done.end(), s.active[k]) != done.end()) live[k] = 0;
            ctx.reserve(s.live, live.size());
            DL_CUDA(cudaMemcpyAsync(s.live.p, live.data(), live.size(), cudaMemcpyHostToDevice, ctx.stream));
            KeepActive keep{s.inst_lo.as<u64>(), s.live.as<uint8_t>(), (u32) s.active.size(), s.bits};
            s.n_delta = session_select(ctx, s.delta.as<u64>(), s.n_delta, keep, 61);
        }
    }
    retire(s, done, still);
    maybe_compact(s);
    return s.active.size();
}

}  // namespace

SessionImpl *session_create(Context &parent, int program, const dl_options &opt, u64 max_nodes) {
    if (program != DL_PROGRAM_TC && program != DL_PROGRAM_SG && program != DL_PROGRAM_WCC)
        throw Error(DL_ERR_INVALID_ARGUMENT, "sessions run TC, SG or WCC");
    auto s = std::make_unique<SessionImpl>();
    s->program = program;
    s->opt = opt;
    if (program == DL_PROGRAM_WCC) {
        // WCC words are (rank << 32 | label rank)
        s->bits = 32;
        s->rank_cap = 0xFFFFFFFFull;
    } else {
        // TC/SG words hold two rank fields of `bits` bits; the sorts only
        // visit the bits the ranks in use can set
        s->bits = max_nodes ? std::max(1, bits_for(max_nodes)) : 32;
        if (max_nodes >= 0xFFFFFFFFull) throw Error(DL_ERR_INVALID_ARGUMENT, "max_nodes above 2^32 - 2");
        s->rank_cap = s->bits == 32 ? 0xFFFFFFFFull : (1ull << s->bits);
    }
    Context &c = s->ctx;
    s->parent = &parent;
    c.device = parent.device;
    c.stream = parent.stream;
    c.sm_count = parent.sm_count;
    c.prof_on = parent.prof_on;
    c.tune = parent.tune;
    void *p = nullptr;
    DL_CUDA(cudaMalloc(&p, sizeof(Ctrl)));
    c.ctrl = (Ctrl *) p;
    DL_CUDA(cudaMemset(p, 0, sizeof(Ctrl)));
    DL_CUDA(cudaMallocHost((void **) &c.host_scalars, 64 * sizeof(u64)));
    std::memset(c.host_scalars, 0, 64 * sizeof(u64));
    c.spares = std::move(parent.spares);  // the parent's cached buffers serve the session
    parent.spares.clear();
    return s.release();
}

void session_destroy(SessionImpl *s) {
    if (!s) return;
    Context &c = s->ctx;
    cudaStreamSynchronize(c.stream);
    c.prof_resolve();
    // Every buffer goes back to the parent context's cache: the next run or
    // session on it reuses the memory instead of allocating it again.
    Context &p = *s->parent;
    for (auto &in : s->inst) {  // blocks return to the session's cache
        in.ids_block.reset();
        in.result_block.reset();
        in.labels_block.reset();
    }
    DevBuf *bufs[] = {&s->off,     &s->val,    &s->delta,    &s->label,     &s->flag,
                      &s->nextl,   &s->inst_lo, &s->inst_hi, &s->counts,    &s->live,
                      &s->range_lo, &s->admit_off, &s->admit_first};
    for (DevBuf *b : bufs) p.give_back(*b);
    Workspace &w = c.ws;
    DevBuf *wbufs[] = {&w.input,    &w.ids,      &w.w0,       &w.w1,      &w.csr_off,  &w.csr_val,
                       &w.full[0],  &w.full[1],  &w.small[0], &w.small[1], &w.tiny[0], &w.tiny[1],
                       &w.sample,   &w.sample_small, &w.jbuf[0],
                       &w.jbuf[1],  &w.offsets,  &w.wcc_label, &w.wcc_flag, &w.wcc_next};
    for (DevBuf *b : wbufs) p.give_back(*b);
    for (auto &b : c.spares) p.give_back(b);
    c.spares.clear();
    c.release_all();  // look-back words, histograms, split points, events
    if (c.ctrl) cudaFree(c.ctrl);
    if (c.host_scalars) cudaFreeHost(c.host_scalars);
    delete s;
}

std::vector<i64> session_admit_many(SessionImpl &s, const int32_t *const *rows, const u64 *nrows, u64 count,
                                    bool on_device) {
    Context &ctx = s.ctx;
    Workspace &ws = ctx.ws;
    if (count >= (1ull << 31)) throw Error(DL_ERR_INVALID_ARGUMENT, "too many instances in one admission");
    std::vector<u64> off(count + 1, 0);
    for (u64 k = 0; k < count; ++k) off[k + 1] = off[k] + nrows[k];
    const u64 N = off[count];
    const u64 first_id = s.inst.size();
    std::vector<i64> ids(count);
    for (u64 k = 0; k < count; ++k) {
        s.inst.emplace_back();
        SessionInstance &in = s.inst.back();
        in.id = (i64) (first_id + k);
        in.input_rows = (i64) nrows[k];
        in.rank_lo = in.rank_hi = s.next_rank;
        ids[k] = in.id;
    }
    auto inst = [&](u64 k) -> SessionInstance & { return s.inst[first_id + k]; };
    if (N == 0) {  // no instance enters its loop: zero iterations, empty results
        for (u64 k = 0; k < count; ++k) mark_done(s, inst(k));
        return ids;
    }
    try {
        // every instance's rows, back to back, and their row offsets
        ctx.reserve(ws.input, N * 8);
        for (u64 k = 0; k < count; ++k)
            if (nrows[k])
                DL_CUDA(cudaMemcpyAsync(ws.input.as<int32_t>() + 2 * off[k], rows[k], nrows[k] * 8,
                                        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx.stream));
        ctx.reserve(s.admit_off, (count + 1) * 8);
        DL_CUDA(cudaMemcpyAsync(s.admit_off.p, off.data(), (count + 1) * 8, cudaMemcpyHostToDevice, ctx.stream));
        const int32_t *in_rows = ws.input.as<int32_t>();
        const u64 *d_off = s.admit_off.as<u64>();
        // distinct (instance, node id) pairs, sorted: position = union rank
        // offset (tc.cu:171-176 ranks nothing; node ids are only renamed)
        const u64 m = 2 * N;
        ctx.reserve(ws.w0, m * 8);
        ctx.reserve(ws.w1, m * 8);
        DL_LAUNCH(ctx, K_PREP, 0,
                  session_tag_kernel<<<grid_for(N, 256, ctx, 16), 256, 0, ctx.stream>>>(in_rows, N, d_off, (u32) count,
                                                                                         ws.w0.as<u64>()));
        u64 nu = 0;
        u64 *u = sort_unique_into(ctx, ws.w0, ws.w1, m, 32 + bits_for(count), nu);
        const u64 B = s.next_rank;
        if (B + nu > s.rank_cap)
            throw Error(DL_ERR_OVERFLOW, "session node capacity exhausted (" + std::to_string(s.rank_cap) + " ranks)");
        DevBuf &wu = ws.w0.p == u ? ws.w0 : ws.w1;
        DevBuf &wo = ws.w0.p == u ? ws.w1 : ws.w0;
        ctx.reserve(s.admit_first, (count + 1) * 8);
        DL_LAUNCH(ctx, K_PREP, 0,
                  session_first_kernel<<<grid_for(count + 1, 256, ctx, 16), 256, 0, ctx.stream>>>(
                      u, nu, (u32) count, s.admit_first.as<u64>()));
        std::vector<u64> first(count + 1);
        DL_CUDA(cudaMemcpyAsync(first.data(), s.admit_first.p, (count + 1) * 8, cudaMemcpyDeviceToHost, ctx.stream));
        // node ids of the admitted ranks, shared by the instances of this admission
        auto block = make_block(ctx, nu * 4);
        DL_LAUNCH(ctx, K_PREP, 0,
                  session_ids_kernel<<<grid_for(nu, 256, ctx, 16), 256, 0, ctx.stream>>>(u, nu, block->as<int32_t>()));
        // rows -> rank words; the edge relation keyed by source (tc.cu:171-176,
        // sg.cu:150-153, wcc.cu:140-167: WCC stores both directions)
        const int bits = s.bits;
        const bool wcc = s.program == DL_PROGRAM_WCC, tc = s.program == DL_PROGRAM_TC;
        if (tc) ctx.reserve(ws.jbuf[0], N * 8);
        u64 *fw = wo.as<u64>();
        u64 *rv = wcc ? fw + N : (tc ? ws.jbuf[0].as<u64>() : nullptr);
        DL_LAUNCH(ctx, K_PREP, 0,
                  session_pack_many_kernel<<<grid_for(N, 256, ctx, 16), 256, 0, ctx.stream>>>(
                      in_rows, N, d_off, (u32) count, u, nu, B, bits, fw, rv));
        u64 ne = 0;
        const int used = bits_for(std::max<u64>(B + nu, 2));
        u64 *e = sort_unique_fields(ctx, wo, wu, wcc ? m : N, bits, used, ne);
        if (s.n_vals + ne >= (1ull << 32)) throw Error(DL_ERR_OVERFLOW, "session edge capacity exhausted");
        grow_keep(ctx, s.off, (B + nu + 1) * 4, (B + 1) * 4);
        grow_keep(ctx, s.val, (s.n_vals + ne + 1) * 4, s.n_vals * 4);
        DL_LAUNCH(ctx, K_PREP, 0,
                  session_csr_kernel<<<grid_for(std::max<u64>(ne, nu + 1), 256, ctx, 16), 256, 0, ctx.stream>>>(
                      e, ne, bits, B, B + nu, s.n_vals, s.off.as<u32>(), s.val.as<u32>()));
        s.n_vals += ne;
        s.next_rank = B + nu;
        ctx.sync();  // `first` is ready
        for (u64 k = 0; k < count; ++k) {
            SessionInstance &in = inst(k);
            in.rank_lo = B + first[k];
            in.rank_hi = B + first[k + 1];
            in.n_ids = (u32) (first[k + 1] - first[k]);
            in.ids_block = block;
            in.ids_off = first[k];
        }
        std::vector<bool> empty_base(count, false);
        if (tc) {
            u64 nd;
            u64 *d = sort_unique_fields(ctx, ws.jbuf[0], ws.jbuf[1], N, bits, used, nd);  // tc.cu:178-189
            full_insert_new(s, d, nd);
            delta_append(s, d, nd);
        } else if (s.program == DL_PROGRAM_SG) {
            // sg.cu:170-217: the base rule of the admitted instances, probing the union table
            Graph g = union_graph(s);
            u64 *selfs = &ctx.ctrl->scalar[30];
            DL_CUDA(cudaMemsetAsync(selfs, 0, 8, ctx.stream));
            u64 nb = 0;
            PhaseTimer pt(ctx, false);
            u64 *b = join_and_sort(ctx, g, e, ne, EmitKind::ZV_NOSELF, nb, selfs, pt);
            DL_CUDA(cudaMemcpyAsync(ctx.host_scalars + 5, selfs, 8, cudaMemcpyDeviceToHost, ctx.stream));
            ctx.sync();
            const u64 nv = nb - ctx.host_scalars[5];  // self pairs sorted to the end
            const u64 nd = nv ? unique_words(ctx, b, nv, b) : 0;
            std::vector<u64> lo(count);
            for (u64 k = 0; k < count; ++k) lo[k] = inst(k).rank_lo;
            const std::vector<u64> c = range_counts(s, b, nd, bits, lo);
            for (u64 k = 0; k < count; ++k) empty_base[k] = c[k] == 0;
            full_insert_new(s, b, nd);
            delta_append(s, b, nd);
        } else {  // wcc.cu:211-231: cc(n, n) for every node, all nodes in the first delta
            grow_keep(ctx, s.label, (B + nu) * 4, B * 4);
            grow_keep(ctx, s.flag, (B + nu) * 4, B * 4);
            grow_keep(ctx, s.nextl, (B + nu + 1) * 4, 0);
            grow_keep(ctx, s.delta, (s.n_delta + nu) * 8, s.n_delta * 8);
            DL_LAUNCH(ctx, K_PREP, 0,
                      session_label_init_kernel<<<grid_for(nu, 256, ctx, 16), 256, 0, ctx.stream>>>(
                          s.label.as<u32>(), s.flag.as<u32>(), B, B + nu, s.delta.as<u64>() + s.n_delta));
            s.n_delta += nu;
            for (u64 k = 0; k < count; ++k) inst(k).prev_delta = (i64) inst(k).n_ids;
        }
        ctx.sync();
        for (u64 k = 0; k < count; ++k) {
            SessionInstance &in = inst(k);
            if (nrows[k] == 0) {
                mark_done(s, in);
            } else if (empty_base[k]) {  // the loop runs once on an empty delta (sg.cu:244-390)
                in.deltas.push_back(0);
                mark_done(s, in);
            } else {
                in.active = true;
                s.active.push_back(in.id);
            }
        }
        s.inst_dirty = true;
    } catch (...) {
        // the union tables may hold part of these instances; their ranks are never reused
        for (u64 k = 0; k < count; ++k) {
            inst(k).done = true;
            inst(k).released = true;
        }
        throw;
    }
    return ids;
}

i64 session_admit(SessionImpl &s, const int32_t *rows, u64 n, bool on_device) {
    return session_admit_many(s, &rows, &n, 1, on_device)[0];
}

u64 session_step(SessionImpl &s) {
    if (s.active.empty()) return 0;
    return s.program == DL_PROGRAM_WCC ? wcc_step(s) : fixpoint_step(s);
}

u64 session_poll(SessionImpl &s, int64_t *ids, u64 capacity) {
    const u64 n = std::min<u64>(capacity, s.finished.size());
    for (u64 i = 0; i < n; ++i) ids[i] = s.finished[i];
    s.finished.erase(s.finished.begin(), s.finished.begin() + (std::ptrdiff_t) n);
    return n;
}

void session_fold_profile(SessionImpl &s, Context &parent) {
    s.ctx.sync();  // resolves the timed launches
    for (int k = 0; k < K_COUNT; ++k) {
        KernelStat &a = parent.kstat[k];
        KernelStat &b = s.ctx.kstat[k];
        a.launches += b.launches;
        a.timed += b.timed;
        a.seconds += b.seconds;
        a.bytes += b.bytes;
        b = KernelStat();
    }
    s.ctx.prof_on = parent.prof_on;
}

const SessionInstance &session_instance(const SessionImpl &s, i64 id) {
    if (id < 0 || id >= (i64) s.inst.size()) throw Error(DL_ERR_INVALID_ARGUMENT, "unknown instance " + std::to_string(id));
    return s.inst[id];
}

void session_info(const SessionImpl &s, i64 id, dl_run_info &info) {
    const SessionInstance &in = session_instance(s, id);
    std::memset(&info, 0, sizeof(info));
    info.program = s.program;
    info.iterations = (int32_t) in.deltas.size();
    info.input_rows = in.input_rows;
    info.output_rows = info.output_tuples = in.done ? (i64) in.n_result : 0;
    info.largest_component = in.largest;
    info.nodes = in.n_ids;
}

static SessionInstance &finished_instance(SessionImpl &s, i64 id) {
    session_instance(s, id);
    SessionInstance &in = s.inst[id];
    if (!in.done) throw Error(DL_ERR_INVALID_ARGUMENT, "instance " + std::to_string(id) + " has not finished");
    if (in.released) throw Error(DL_ERR_INVALID_ARGUMENT, "instance " + std::to_string(id) + " was released");
    return in;
}

void session_copy_output(SessionImpl &s, i64 id, int32_t *dst, u64 capacity, bool on_device) {
    SessionInstance &in = finished_instance(s, id);
    Context &ctx = s.ctx;
    const u64 n = in.n_result;
    if (capacity < n) throw Error(DL_ERR_INVALID_ARGUMENT, "output capacity too small");
    if (n == 0) return;
    DevBuf stage;
    int32_t *tmp = dst;
    if (!on_device) {
        ctx.reserve(stage, n * 8);
        tmp = stage.as<int32_t>();
    }
    const int32_t *ids = in.ids();
    const unsigned g = grid_for(n, 256, ctx, 16);
    if (s.program == DL_PROGRAM_WCC)
        DL_LAUNCH(ctx, K_PREP, 0, session_unpack_comp_kernel<<<g, 256, 0, ctx.stream>>>(in.result_u32(), n, ids, tmp));
    else if (s.program == DL_PROGRAM_SG)
        DL_LAUNCH(ctx, K_PREP, 0,
                  session_unpack_kernel<true><<<g, 256, 0, ctx.stream>>>(in.result_words(), n, s.bits, in.rank_lo,
                                                                          ids, tmp));
    else
        DL_LAUNCH(ctx, K_PREP, 0,
                  session_unpack_kernel<false><<<g, 256, 0, ctx.stream>>>(in.result_words(), n, s.bits, in.rank_lo,
                                                                           ids, tmp));
    if (!on_device) DL_CUDA(cudaMemcpyAsync(dst, tmp, n * 8, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    ctx.give_back(stage);
}

void session_copy_labels(SessionImpl &s, i64 id, int32_t *node_ids, int32_t *labels, u64 capacity) {
    SessionInstance &in = finished_instance(s, id);
    if (s.program != DL_PROGRAM_WCC) throw Error(DL_ERR_INVALID_ARGUMENT, "labels exist only for WCC sessions");
    Context &ctx = s.ctx;
    const u64 n = in.n_ids;
    if (capacity < n) throw Error(DL_ERR_INVALID_ARGUMENT, "label capacity too small");
    if (n == 0) return;
    DevBuf stage;
    ctx.reserve(stage, n * 4);
    DL_LAUNCH(ctx, K_PREP, 0,
              session_unpack_labels_kernel<<<grid_for(n, 256, ctx, 16), 256, 0, ctx.stream>>>(
                  in.labels(), in.rank_lo, n, in.ids(), stage.as<int32_t>()));
    DL_CUDA(cudaMemcpyAsync(labels, stage.p, n * 4, cudaMemcpyDeviceToHost, ctx.stream));
    DL_CUDA(cudaMemcpyAsync(node_ids, in.ids(), n * 4, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    ctx.give_back(stage);
}

void session_release(SessionImpl &s, i64 id) {
    SessionInstance &in = finished_instance(s, id);
    in.result_block.reset();  // each block goes with its last instance
    in.labels_block.reset();
    in.ids_block.reset();
    in.released = true;
}

u64 session_device_bytes(const SessionImpl &s) {
    const Context &c = s.ctx;
    const Workspace &w = c.ws;
    u64 b = 0;
    const DevBuf *bufs[] = {&s.off,     &s.val,       &s.delta,    &s.label,      &s.flag,       &s.nextl,
                            &w.input,   &w.ids,       &w.w0,       &w.w1,         &w.csr_off,    &w.csr_val,
                            &w.full[0], &w.full[1],   &w.small[0], &w.small[1],   &w.tiny[0],    &w.tiny[1],
                            &w.sample,  &w.sample_small, &w.jbuf[0],
                            &w.jbuf[1], &w.offsets,   &c.lookback, &c.radix_part, &c.lbs_splits, &c.sort_hist,
                            &c.merge_splits};
    for (const DevBuf *x : bufs) b += x->cap;  // cached spare buffers are not counted: they are free memory
    std::vector<const DevBuf *> blocks;
    for (const auto &in : s.inst)
        for (const DevBuf *x : {in.ids_block.get(), in.result_block.get(), in.labels_block.get()})
            if (x && std::find(blocks.begin(), blocks.end(), x) == blocks.end()) blocks.push_back(x);
    for (const DevBuf *x : blocks) b += x->cap;
    return b;
}

u64 session_active(const SessionImpl &s) { return s.active.size(); }
u64 session_instance_count(const SessionImpl &s) { return s.inst.size(); }

}  // namespace dl
