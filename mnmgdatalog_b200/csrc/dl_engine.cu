// Fixpoint drivers for the four programs (tc.cu, sg.cu, wcc.cu,
// single_join.cu) on one GPU, over dense node indices.
//
// Init maps every node id of the input to its rank among the distinct ids
// (sorted, so rank order == id order) and packs a tuple (a, b) into the
// 2*B-bit word (rank(a) << B) | rank(b), B = bits needed for a rank. Word order
// equals the reference's set_cmp order, so sorted word arrays are the
// reference's sorted Entity arrays, and the radix sort only touches 2*B bits.
// The indexed relation of every join (the edges, keyed by source) becomes an
// offset table over ranks (CSR): the hash probe of the reference
// (common/hash_table.cu, common/join.cu) turns into one offset lookup.
//
// Per iteration (TC):  count+scan -> emit J (+radix histogram) -> radix sort
// J -> fused unique/set-difference/merge (delta, full') -> |delta| to host.
// Nothing is allocated inside the loop once buffers reach their high-water
// mark; every device wait is bounded (see dl_device.cuh).
#include "dl_internal.h"
#include "dl_join.cuh"
#include "dl_scan.cuh"
#include "dl_engine.h"
#include "dl_engine_detail.h"

namespace dl {
namespace detail {


#define GRID_STRIDE(i, n) for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (u64) gridDim.x * blockDim.x)

__global__ void ids_to_words_kernel(const int32_t *__restrict__ v, u64 n, u64 *__restrict__ out) {
    GRID_STRIDE(i, n) out[i] = (u64) ((u32) v[i] ^ 0x80000000u);
}

__global__ void words_to_ids_kernel(const u64 *__restrict__ w, u64 n, int32_t *__restrict__ ids) {
    GRID_STRIDE(i, n) ids[i] = (int32_t) ((u32) w[i] ^ 0x80000000u);
}

__device__ __forceinline__ u32 rank_of(const int32_t *__restrict__ ids, u32 n, int32_t x) {
    u32 lo = 0, hi = n;
    while (lo < hi) {
        const u32 mid = (lo + hi) >> 1;
        if (ids[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Rows (a, b) -> fwd word (rank a, rank b) and/or rev word (rank b, rank a).
__global__ void pack_rows_kernel(const int32_t *__restrict__ rows, u64 n, const int32_t *__restrict__ ids, u32 n_ids,
                                 int bits, u64 *__restrict__ fwd, u64 *__restrict__ rev) {
    GRID_STRIDE(i, n) {
        const u64 a = rank_of(ids, n_ids, rows[2 * i]);
        const u64 b = rank_of(ids, n_ids, rows[2 * i + 1]);
        if (fwd) fwd[i] = (a << bits) | b;
        if (rev) rev[i] = (b << bits) | a;
    }
}

// Offsets of a sorted word array grouped by key rank: off[k] = first word
// whose key is >= k, for k in [0, n_keys].
__global__ void csr_offsets_kernel(const u64 *__restrict__ w, u64 n, int bits, u32 n_keys, u32 *__restrict__ off) {
    GRID_STRIDE(k, (u64) n_keys + 1) {
        const u64 target = k << bits;
        u64 lo = 0, hi = n;
        while (lo < hi) {
            const u64 mid = (lo + hi) >> 1;
            if (w[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        off[k] = (u32) lo;
    }
}

__global__ void csr_values_kernel(const u64 *__restrict__ w, u64 n, u64 mask, u32 *__restrict__ val) {
    GRID_STRIDE(i, n) val[i] = (u32) (w[i] & mask);
}

// Sorted words -> output rows of the reference's file.
//   KeyFirst = false: word (z << B | x) -> row (x, z)   (TC, single_join)
//   KeyFirst = true : word (x << B | y) -> row (x, y)   (SG)
template <bool KeyFirst>
__global__ void unpack_rows_kernel(const u64 *__restrict__ w, u64 n, int bits, const int32_t *__restrict__ ids,
                                   int32_t *__restrict__ out) {
    const u64 mask = (1ull << bits) - 1;
    GRID_STRIDE(i, n) {
        const u64 x = w[i];
        const int32_t hi = ids[x >> bits], lo = ids[x & mask];
        int2 r;
        r.x = KeyFirst ? hi : lo;
        r.y = KeyFirst ? lo : hi;
        reinterpret_cast<int2 *>(out)[i] = r;
    }
}

__global__ void wcc_init_kernel(u32 n, u32 *__restrict__ label, u32 *__restrict__ flag, u64 *__restrict__ delta) {
    GRID_STRIDE(u, (u64) n) {
        label[u] = (u32) u;
        flag[u] = 0;
        delta[u] = (u << 32) | u;
    }
}

__global__ void wcc_next_delta_kernel(const u32 *__restrict__ nodes, u64 count, const u32 *__restrict__ label,
                                      u32 *__restrict__ flag, u64 *__restrict__ delta) {
    GRID_STRIDE(i, count) {
        const u32 v = nodes[i];
        delta[i] = ((u64) v << 32) | label[v];
        flag[v] = 0;
    }
}

__global__ void wcc_count_kernel(const u32 *__restrict__ label, u32 n, u32 *__restrict__ cnt) {
    GRID_STRIDE(u, (u64) n) atomicAdd(&cnt[label[u]], 1u);
}

// Scan source: 1 for every label rank that names a component.
struct NonZeroCounter {
    const u32 *cnt;
    __device__ __forceinline__ u64 degree(u64 i) const { return cnt[i] != 0u; }
};

__global__ void wcc_components_kernel(const u32 *__restrict__ cnt, u32 n, const u64 *__restrict__ pos,
                                      u32 *__restrict__ comp, unsigned long long *__restrict__ largest) {
    GRID_STRIDE(c, (u64) n) {
        const u32 k = cnt[c];
        if (k) {
            comp[pos[c]] = (u32) c;
            atomicMax(largest, (unsigned long long) k);
        }
    }
}

__global__ void unpack_components_kernel(const u32 *__restrict__ comp, u64 n, const int32_t *__restrict__ ids,
                                         int32_t *__restrict__ out) {
    GRID_STRIDE(i, n) {
        int2 r;
        r.x = ids[comp[i]];
        r.y = 0;
        reinterpret_cast<int2 *>(out)[i] = r;
    }
}

__global__ void unpack_labels_kernel(const u32 *__restrict__ label, u32 n, const int32_t *__restrict__ ids,
                                     int32_t *__restrict__ out) {
    GRID_STRIDE(u, (u64) n) out[u] = ids[label[u]];
}



int bits_for(u64 n) {
    int b = 1;
    while ((1ull << b) < n) ++b;
    return b;
}

// Copies the input rows to the device (if needed), ranks node ids, packs
// rows into words. `fwd`/`rev` receive unsorted words (either may be null).
const int32_t *stage_input(Context &ctx, const int32_t *rows, u64 n, bool on_device) {
    if (on_device || n == 0) return rows;
    ctx.reserve(ctx.ws.input, n * 8);
    DL_CUDA(cudaMemcpyAsync(ctx.ws.input.p, rows, n * 8, cudaMemcpyHostToDevice, ctx.stream));
    return ctx.ws.input.as<int32_t>();
}

void rank_nodes(Context &ctx, const int32_t *rows, u64 n, Graph &g) {
    Workspace &ws = ctx.ws;
    const u64 m = 2 * n;
    ctx.reserve(ws.w0, m * 8);
    ctx.reserve(ws.w1, m * 8);
    DL_LAUNCH(ctx, K_PREP, 0, ids_to_words_kernel<<<grid_for(m, T256, ctx), T256, 0, ctx.stream>>>(rows, m, ws.w0.as<u64>()));
    u64 *s = radix_sort(ctx, ws.w0.as<u64>(), ws.w1.as<u64>(), m, Codec::Raw, 32);
    const u64 nu = unique_words(ctx, s, m, s);
    ctx.reserve(ws.ids, nu * 4);
    DL_LAUNCH(ctx, K_PREP, 0, words_to_ids_kernel<<<grid_for(nu, T256, ctx), T256, 0, ctx.stream>>>(s, nu, ws.ids.as<int32_t>()));
    g.n_ids = (u32) nu;
    g.bits = bits_for(nu);
    g.ids = ws.ids.as<int32_t>();
}

__global__ void id_range_kernel(int32_t *__restrict__ ids, u64 n, int32_t base) {
    GRID_STRIDE(i, n) ids[i] = (int32_t) ((int64_t) base + (int64_t) i);
}

template <class Fits>
bool densify_ids(Context &ctx, Graph &g, Fits fits) {
    if (g.n_ids == 0) return false;
    int32_t ends[2];
    DL_CUDA(cudaMemcpyAsync(&ends[0], g.ids, 4, cudaMemcpyDeviceToHost, ctx.stream));
    DL_CUDA(cudaMemcpyAsync(&ends[1], g.ids + g.n_ids - 1, 4, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    const u64 range = (u64) ((int64_t) ends[1] - (int64_t) ends[0]) + 1;
    if (range > (u64) g.n_ids + g.n_ids / 8 || range > 0x7FFFFFFFull || !fits(range)) return false;
    Workspace &ws = ctx.ws;
    ctx.reserve(ws.ids, range * 4);
    DL_LAUNCH(ctx, K_PREP, 4.0 * range,
              id_range_kernel<<<grid_for(range, T256, ctx), T256, 0, ctx.stream>>>(ws.ids.as<int32_t>(), range,
                                                                                  ends[0]));
    g.n_ids = (u32) range;
    g.bits = bits_for(range);
    g.ids = ws.ids.as<int32_t>();
    g.ids_affine = true;
    g.id_base = ends[0];
    return true;
}

// Sorted, duplicate-free words (key rank << bits | value rank) -> CSR.
void build_csr(Context &ctx, const u64 *words, u64 n, Graph &g) {
    Workspace &ws = ctx.ws;
    ctx.reserve(ws.csr_off, ((u64) g.n_ids + 1) * 4);
    ctx.reserve(ws.csr_val, std::max<u64>(n, 1) * 4);
    DL_LAUNCH(ctx, K_PREP, 0, csr_offsets_kernel<<<grid_for((u64) g.n_ids + 1, T256, ctx), T256, 0, ctx.stream>>>(words, n, g.bits, g.n_ids,
                                                                                         ws.csr_off.as<u32>()));
    if (n) {
        DL_LAUNCH(ctx, K_PREP, 0, csr_values_kernel<<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(words, n, (1ull << g.bits) - 1,
                                                                          ws.csr_val.as<u32>()));
    }
    g.csr.off = ws.csr_off.as<u32>();
    g.csr.val = ws.csr_val.as<u32>();
    g.csr.n_keys = g.n_ids;
    g.csr.n_vals = n;
}

// Sorts `n` words held in buf (ping-pong with alt) and drops duplicates.
// Returns the buffer holding the result (one of buf/alt) and its length.
u64 *sort_unique_into(Context &ctx, DevBuf &buf, DevBuf &alt, u64 n, int key_bits, u64 &n_out) {
    ctx.reserve(alt, std::max<u64>(n, 1) * 8);
    u64 *s = radix_sort(ctx, buf.as<u64>(), alt.as<u64>(), n, Codec::Raw, key_bits);
    n_out = unique_words(ctx, s, n, s);
    return s;
}

DevBuf &holder(Workspace &ws, const u64 *p) { return ws.jbuf[0].p == p ? ws.jbuf[0] : ws.jbuf[1]; }
DevBuf &other(Workspace &ws, const u64 *p) { return ws.jbuf[0].p == p ? ws.jbuf[1] : ws.jbuf[0]; }

// One semi-naive join step: count, emit (with the radix histogram), sort.
// The probe words live in jbuf[probe_slot]; J is written to the other jbuf
// and sorted using the probe's buffer as ping-pong (the probe is dead after
// the emit). Returns the buffer that holds sorted J.
u64 *join_and_sort(Context &ctx, const Graph &g, const u64 *probe, u64 n_probe, EmitKind kind, u64 &n_j,
                   u64 *self_pairs, PhaseTimer &pt) {
    Workspace &ws = ctx.ws;
    pt.mark(PH_JOIN);
    ctx.reserve(ws.offsets, std::max<u64>(n_probe, 1) * 8);
    const u64 total = join_count(ctx, g.csr, probe, n_probe, g.bits, ws.offsets.as<u64>());
    n_j = total;
    ctx.run_join_total += total;
    ctx.run_join_max = std::max(ctx.run_join_max, total);
    DevBuf &jout = other(ws, probe);
    ctx.reserve(jout, std::max<u64>(total, 1) * 8);
    if (total == 0) return jout.as<u64>();
    const int key_bits = 2 * g.bits;
    // TC words (z << bits | v) take bits 0-7 from the probe row: the emit
    // itself groups them by that digit, and the sort starts at bit 8
    const bool first_pass = ctx.tune.join_first_pass && kind == EmitKind::ZV && g.bits >= 8 &&
                            !radix_wants_histogram(ctx) && (g.nwin == 0 || g.win[0] == 0);
    if (first_pass) {
        join_emit_bucketed(ctx, g.csr, probe, n_probe, g.bits, ws.offsets.as<u64>(), total, jout.as<u64>());
        pt.mark(PH_DEDUP);
        DevBuf &pbuf = holder(ws, probe);
        u64 *jptr = jout.as<u64>();
        ctx.reserve(pbuf, total * 8);  // probe is dead now
        int w[8];
        int nw = 0;
        if (g.nwin) {
            for (int i = 1; i < g.nwin; ++i) w[nw++] = g.win[i];
        } else {
            for (int sh = 8; sh < key_bits; sh += 8) w[nw++] = sh;
        }
        return radix_sort_windows(ctx, jptr, pbuf.as<u64>(), total, w, nw);
    }
    const bool fuse_hist = radix_wants_histogram(ctx) && !g.nwin;
    const int ndig = fuse_hist ? (key_bits + 7) / 8 : 0;
    u64 *hist = fuse_hist ? radix_hist_buffer(ctx) : nullptr;
    if (fuse_hist) radix_hist_clear(ctx);
    join_emit(ctx, g.csr, probe, n_probe, g.bits, ws.offsets.as<u64>(), total, kind, jout.as<u64>(), hist, ndig,
              self_pairs);
    pt.mark(PH_DEDUP);
    DevBuf &pbuf = holder(ws, probe);
    u64 *jptr = jout.as<u64>();
    ctx.reserve(pbuf, total * 8);  // probe is dead now
    if (g.nwin) return radix_sort_windows(ctx, jptr, pbuf.as<u64>(), total, g.win, g.nwin);
    return radix_sort(ctx, jptr, pbuf.as<u64>(), total, Codec::Raw, key_bits, hist);
}

// One join step without the sort: J in the join buffer that does not hold
// the probe (its order follows the probe rows).
u64 *join_unsorted(Context &ctx, const Graph &g, const u64 *probe, u64 n_probe, EmitKind kind, u64 &n_j,
                   PhaseTimer &pt) {
    Workspace &ws = ctx.ws;
    pt.mark(PH_JOIN);
    ctx.reserve(ws.offsets, std::max<u64>(n_probe, 1) * 8);
    const u64 total = join_count(ctx, g.csr, probe, n_probe, g.bits, ws.offsets.as<u64>());
    n_j = total;
    ctx.run_join_total += total;
    ctx.run_join_max = std::max(ctx.run_join_max, total);
    DevBuf &jout = other(ws, probe);
    ctx.reserve(jout, std::max<u64>(total, 1) * 8);
    if (total)
        join_emit(ctx, g.csr, probe, n_probe, g.bits, ws.offsets.as<u64>(), total, kind, jout.as<u64>(), nullptr, 0,
                  nullptr);
    return jout.as<u64>();
}

void finish_info(Run &r, Context &ctx, cudaEvent_t e0, cudaEvent_t e1, PhaseTimer &pt) {
    r.info.join_rows_total = (i64) ctx.run_join_total;
    r.info.join_rows_max = (i64) ctx.run_join_max;
    DL_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    DL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    r.info.seconds_total = ms * 1e-3;
    double ph[5];
    pt.finish(ph);
    r.info.seconds_init = ph[PH_INIT];
    r.info.seconds_join = ph[PH_JOIN];
    r.info.seconds_dedup = ph[PH_DEDUP];
    r.info.seconds_merge = ph[PH_MERGE];
    r.info.seconds_finalize = ph[PH_FINAL];
    r.info.iterations = (int32_t) r.deltas.size();
    if (r.program == DL_PROGRAM_SINGLE_JOIN) r.info.iterations = 1;
}

struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    EventPair() {
        DL_CUDA(cudaEventCreate(&a));
        DL_CUDA(cudaEventCreate(&b));
    }
    ~EventPair() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

// Moves the node id table into the run (the run outlives the workspace use).
void adopt_ids(Context &ctx, Run &r, const Graph &g) {
    r.ids = ctx.ws.ids;
    ctx.ws.ids = DevBuf();
    r.n_ids = g.n_ids;
    r.bits = g.bits;
    r.info.nodes = g.n_ids;
    r.ids_affine = g.ids_affine;
    r.id_base = g.id_base;
}

// The full relation of TC/SG as disjoint sorted duplicate-free runs: a large
// one (ws.full[cur]), a small one (ws.small[scur]) and, for plain runs, a
// tiny one (ws.tiny[tcur]). The reference keeps one sorted array and
// re-merges it with every delta (tc.cu:260-286), which costs O(|full|) per
// iteration even when the delta is tiny; here a sparse join output is checked
// against the large run by binary probes and only the small run is
// rewritten, and the small run is merged into the large one when it reaches
// 1/4 of it. Late iterations whose deltas are small against the small run
// probe it as well and rewrite only the tiny run, which is folded into the
// small run at 1/4 of it. The iteration's delta is the same set.

// Measured on B200: a binary probe costs ~50 ps per J word, the fused
// streaming step ~13 ps per word of (large run + J), so probing wins while
// |J| is below ~1/3 of the large run; the small run is folded into the large
// one only once it reaches 1/4 of it (otherwise at the end).
// The thresholds are per-context tuning (Tuning::dense_ratio, small_ratio;
// defaults 4 and 4).

// Sorted J (in one of ws.jbuf) -> delta (returned, in one of ws.jbuf);
// updates the full relation. Returns |delta| in n_delta.
u64 *absorb(Context &ctx, FullSet &F, u64 *j, u64 nj, u64 &n_delta) {
    Workspace &ws = ctx.ws;
    n_delta = 0;
    if (nj == 0) return j;
    const bool dense = nj * ctx.tune.dense_ratio >= F.nbig;
    DevBuf &d1buf = other(ws, j);
    if (F.nsmall == 0 && dense) {
        // fused: delta and the new large run in one pass
        ctx.reserve(ws.full[1 - F.cur], (F.nbig + nj) * 8);
        const u64 n = diff_merge_words(ctx, ws.full[F.cur].as<u64>(), F.nbig, j, nj, ws.full[1 - F.cur].as<u64>(),
                                       d1buf.as<u64>(), Codec::Raw);
        if (n) {
            F.cur = 1 - F.cur;
            F.nbig += n;
            F.sample_ok = false;
        }
        n_delta = n;
        return d1buf.as<u64>();
    }
    // delta' = dedup(J) \ large run
    u64 nd1;
    if (dense) {
        nd1 = diff_merge_words(ctx, ws.full[F.cur].as<u64>(), F.nbig, j, nj, nullptr, d1buf.as<u64>(), Codec::Raw);
    } else {
        if (!F.sample_ok) {
            run_sample(ctx, ws.full[F.cur].as<u64>(), F.nbig, ws.sample, F.ns);
            F.sample_ok = true;
        }
        nd1 = sparse_diff_words(ctx, ws.full[F.cur].as<u64>(), F.nbig, ws.sample.as<u64>(), F.ns, j, nj,
                                d1buf.as<u64>());
    }
    if (nd1 == 0) return j;
    DevBuf &jb = holder(ws, j);  // J is consumed
    if (F.three && F.nsmall && nd1 * ctx.tune.dense_ratio < F.nsmall) {
        // delta'' = delta' \ small run by probes; delta = delta'' \ tiny run,
        // tiny run' = tiny run u delta
        if (!F.ssample_ok) {
            run_sample(ctx, ws.small[F.scur].as<u64>(), F.nsmall, ws.sample_small, F.nss);
            F.ssample_ok = true;
        }
        ctx.reserve(jb, std::max<u64>(nd1, 1) * 8);
        const u64 nd2 = sparse_diff_words(ctx, ws.small[F.scur].as<u64>(), F.nsmall, ws.sample_small.as<u64>(),
                                          F.nss, d1buf.as<u64>(), nd1, jb.as<u64>());
        if (nd2 == 0) return jb.as<u64>();
        ctx.reserve(ws.tiny[1 - F.tcur], (F.ntiny + nd2) * 8);
        const u64 n = diff_merge_words(ctx, ws.tiny[F.tcur].as<u64>(), F.ntiny, jb.as<u64>(), nd2,
                                       ws.tiny[1 - F.tcur].as<u64>(), d1buf.as<u64>(), Codec::Raw);
        if (n) {
            F.tcur = 1 - F.tcur;
            F.ntiny += n;
        }
        n_delta = n;
        if (F.ntiny * ctx.tune.small_ratio >= F.nsmall) fold_tiny(ctx, F);
        return d1buf.as<u64>();
    }
    fold_tiny(ctx, F);  // the small run below is the whole rest of full
    // delta = delta' \ small run; small run' = small run u delta
    ctx.reserve(ws.small[1 - F.scur], (F.nsmall + nd1) * 8);
    const u64 n = diff_merge_words(ctx, ws.small[F.scur].as<u64>(), F.nsmall, d1buf.as<u64>(), nd1,
                                   ws.small[1 - F.scur].as<u64>(), jb.as<u64>(), Codec::Raw);
    if (n) {
        F.scur = 1 - F.scur;
        F.nsmall += n;
        F.ssample_ok = false;
    }
    n_delta = n;
    if (F.nsmall && F.nsmall * ctx.tune.small_ratio >= F.nbig) {
        ctx.reserve(ws.full[1 - F.cur], (F.nbig + F.nsmall) * 8);
        merge_words(ctx, ws.full[F.cur].as<u64>(), F.nbig, ws.small[F.scur].as<u64>(), F.nsmall,
                    ws.full[1 - F.cur].as<u64>(), Codec::Raw);
        F.cur = 1 - F.cur;
        F.nbig += F.nsmall;
        F.nsmall = 0;
        F.sample_ok = false;
        F.ssample_ok = false;
    }
    return jb.as<u64>();
}

// Merges the tiny run into the small run.
void fold_tiny(Context &ctx, FullSet &F) {
    Workspace &ws = ctx.ws;
    if (F.ntiny == 0) return;
    ctx.reserve(ws.small[1 - F.scur], (F.nsmall + F.ntiny) * 8);
    merge_words(ctx, ws.small[F.scur].as<u64>(), F.nsmall, ws.tiny[F.tcur].as<u64>(), F.ntiny,
                ws.small[1 - F.scur].as<u64>(), Codec::Raw);
    F.scur = 1 - F.scur;
    F.nsmall += F.ntiny;
    F.ntiny = 0;
    F.ssample_ok = false;
}

// Final full relation as one sorted run in ws.full[F.cur].
void settle(Context &ctx, FullSet &F) {
    Workspace &ws = ctx.ws;
    fold_tiny(ctx, F);
    if (F.nsmall == 0) return;
    ctx.reserve(ws.full[1 - F.cur], (F.nbig + F.nsmall) * 8);
    merge_words(ctx, ws.full[F.cur].as<u64>(), F.nbig, ws.small[F.scur].as<u64>(), F.nsmall,
                ws.full[1 - F.cur].as<u64>(), Codec::Raw);
    F.cur = 1 - F.cur;
    F.nbig += F.nsmall;
    F.nsmall = 0;
}

}  // namespace detail

using namespace detail;

// ---------------------------------------------------------------------------
// TC (tc.cu:42-423): path stored reversed as (z, x) keyed by z; edges keyed by
// source; Delta_0 = dedup(reversed edges); loop until |full| is unchanged.
static void run_tc_impl(Context &ctx, Run &r, const int32_t *rows_in, u64 n, bool on_device, const dl_options &opt) {
    Workspace &ws = ctx.ws;
    PhaseTimer pt(ctx, opt.phase_timing != 0);
    EventPair ev;
    DL_CUDA(cudaEventRecord(ev.a, ctx.stream));
    pt.mark(PH_INIT);
    const int32_t *rows = stage_input(ctx, rows_in, n, on_device);
    Graph g;
    u64 nfull = 0;
    int cur = 0;
    FullSet F;
    F.three = true;  // plain runs: large, small and tiny runs
    if (n > 0) {
        rank_nodes(ctx, rows, n, g);
        // On the bit-matrix path, a dense id range is ranked as is: the
        // result rows then need no rank -> id table lookups.
        const bool dense = densify_ids(ctx, g, [&](u64 range) {
            try {
                return bitmat_choose(ctx, opt, range, false);
            } catch (const Error &) {  // a forced bit matrix that fits only without the absent ids
                return false;
            }
        });
        ctx.reserve(ws.jbuf[0], n * 8);
        ctx.reserve(ws.jbuf[1], n * 8);
        DL_LAUNCH(ctx, K_PREP, 0, pack_rows_kernel<<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(rows, n, g.ids, g.n_ids, g.bits,
                                                                         ws.w0.as<u64>(), ws.jbuf[0].as<u64>()));
        u64 ne;
        u64 *e = sort_unique_into(ctx, ws.w0, ws.w1, n, 2 * g.bits, ne);
        build_csr(ctx, e, ne, g);
        if (dense || bitmat_choose(ctx, opt, g.n_ids, false)) {
            nfull = tc_bitmap_fixpoint(ctx, r, g, e, ne, opt, pt);  // result: the transpose, or the matrix and column offsets, in r
            cur = 0;
        } else {
            u64 nd;
            u64 *d = sort_unique_into(ctx, ws.jbuf[0], ws.jbuf[1], n, 2 * g.bits, nd);  // tc.cu:178-181
            ctx.reserve(ws.full[0], nd * 8);
            DL_CUDA(cudaMemcpyAsync(ws.full[0].p, d, nd * 8, cudaMemcpyDeviceToDevice, ctx.stream));  // tc.cu:188-189
            F.cur = 0;
            F.nbig = nd;
            u64 *delta = d;
            u64 ndelta = nd;
            for (int it = 0;; ++it) {  // tc.cu:216-314
                u64 nj = 0;
                u64 *j = join_and_sort(ctx, g, delta, ndelta, EmitKind::ZV, nj, nullptr, pt);
                pt.mark(PH_MERGE);
                u64 nnew = 0;
                delta = absorb(ctx, F, j, nj, nnew);
                ndelta = nnew;
                r.deltas.push_back((i64) nnew);
                r.joins.push_back((i64) nj);
                r.fulls.push_back((i64) F.size());
                if (nnew == 0) break;  // |full| unchanged
                if (opt.max_iterations > 0 && it + 1 >= opt.max_iterations) break;
            }
            settle(ctx, F);
            nfull = F.nbig;
            cur = F.cur;
        }
    }
    pt.mark(PH_FINAL);
    DL_CUDA(cudaEventRecord(ev.b, ctx.stream));
    pt.mark(PH_FINAL);
    adopt_ids(ctx, r, g);
    if (!r.from_bitmat) {
        r.words = ws.full[cur];
        ws.full[cur] = DevBuf();
        r.n_words = nfull;
    }
    r.info.output_rows = r.info.output_tuples = (i64) nfull;
    finish_info(r, ctx, ev.a, ev.b, pt);
}

// TC with the join output deduplicated by a hash set of full (dl_hashset.cu):
// the same iterations and deltas as run_tc_impl (delta' = dedup(J) \ full is a
// set), no per-iteration sort or merge; the result is sorted once at the end.
static void run_tc_hash_impl(Context &ctx, Run &r, const int32_t *rows_in, u64 n, bool on_device,
                             const dl_options &opt) {
    Workspace &ws = ctx.ws;
    PhaseTimer pt(ctx, opt.phase_timing != 0);
    EventPair ev;
    DL_CUDA(cudaEventRecord(ev.a, ctx.stream));
    pt.mark(PH_INIT);
    const int32_t *rows = stage_input(ctx, rows_in, n, on_device);
    Graph g;
    u64 nfull = 0;
    DevBuf result;
    if (n > 0) {
        rank_nodes(ctx, rows, n, g);
        ctx.reserve(ws.jbuf[0], n * 8);
        ctx.reserve(ws.jbuf[1], n * 8);
        DL_LAUNCH(ctx, K_PREP, 0, pack_rows_kernel<<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(rows, n, g.ids, g.n_ids, g.bits,
                                                                         ws.w0.as<u64>(), ws.jbuf[0].as<u64>()));
        u64 ne;
        u64 *e = sort_unique_into(ctx, ws.w0, ws.w1, n, 2 * g.bits, ne);
        build_csr(ctx, e, ne, g);
        u64 nd;
        u64 *d = sort_unique_into(ctx, ws.jbuf[0], ws.jbuf[1], n, 2 * g.bits, nd);  // tc.cu:178-181
        WordSet S;  // full (tc.cu:188-189), in ws.full[0/1]
        wordset_reserve(ctx, S, ws.full, nd);
        wordset_insert(ctx, S, ws.full, d, nd, nullptr);
        u64 *delta = d;
        u64 ndelta = nd;
        for (int it = 0;; ++it) {  // tc.cu:216-314
            u64 nj = 0;
            u64 *j = join_unsorted(ctx, g, delta, ndelta, EmitKind::ZV, nj, pt);
            pt.mark(PH_DEDUP);
            u64 nnew = 0;
            if (nj) {
                wordset_reserve(ctx, S, ws.full, nj);
                DevBuf &fb = holder(ws, delta);  // the probe is consumed: it receives the new words
                ctx.reserve(fb, nj * 8);
                nnew = wordset_insert(ctx, S, ws.full, j, nj, fb.as<u64>());
                delta = fb.as<u64>();
            }
            ndelta = nnew;
            r.deltas.push_back((i64) nnew);
            r.joins.push_back((i64) nj);
            r.fulls.push_back((i64) S.size);
            if (nnew == 0) break;  // |full| unchanged
            if (opt.max_iterations > 0 && it + 1 >= opt.max_iterations) break;
        }
        // the program's output order: the set's words, sorted once
        pt.mark(PH_FINAL);
        nfull = S.size;
        ctx.reserve(ws.jbuf[0], std::max<u64>(nfull, 1) * 8);
        ctx.reserve(ws.jbuf[1], std::max<u64>(nfull, 1) * 8);
        wordset_extract(ctx, S, ws.full, ws.jbuf[0].as<u64>());
        u64 *sorted = radix_sort(ctx, ws.jbuf[0].as<u64>(), ws.jbuf[1].as<u64>(), nfull, Codec::Raw, 2 * g.bits);
        DevBuf &hold = holder(ws, sorted);
        result = hold;
        hold = DevBuf();
    }
    DL_CUDA(cudaEventRecord(ev.b, ctx.stream));
    pt.mark(PH_FINAL);
    adopt_ids(ctx, r, g);
    r.words = result;
    r.n_words = nfull;
    r.info.output_rows = r.info.output_tuples = (i64) nfull;
    finish_info(r, ctx, ev.a, ev.b, pt);
}

// SG (sg.cu:40-477): base sg(x,y) :- e(p,x), e(p,y), x != y; recursive rule
// as two joins with the column swaps fused into the emit.
// SG's edge relation: the input rows as sorted duplicate-free words (in
// jbuf[0] or jbuf[1]).
static u64 *sg_edge_words(Context &ctx, const int32_t *rows, u64 n, const Graph &g, u64 &ne) {
    Workspace &ws = ctx.ws;
    ctx.reserve(ws.jbuf[0], n * 8);
    ctx.reserve(ws.jbuf[1], n * 8);
    DL_LAUNCH(ctx, K_PREP, 0, pack_rows_kernel<<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(rows, n, g.ids, g.n_ids, g.bits,
                                                                     ws.jbuf[0].as<u64>(), nullptr));
    return sort_unique_into(ctx, ws.jbuf[0], ws.jbuf[1], n, 2 * g.bits, ne);
}

static void run_sg_impl(Context &ctx, Run &r, const int32_t *rows_in, u64 n, bool on_device, const dl_options &opt) {
    Workspace &ws = ctx.ws;
    PhaseTimer pt(ctx, opt.phase_timing != 0);
    EventPair ev;
    DL_CUDA(cudaEventRecord(ev.a, ctx.stream));
    pt.mark(PH_INIT);
    const int32_t *rows = stage_input(ctx, rows_in, n, on_device);
    Graph g;
    u64 nfull = 0;
    int cur = 0;
    FullSet F;
    F.three = true;  // plain runs: large, small and tiny runs
    bool on_bitmat = false;
    if (n > 0) {
        rank_nodes(ctx, rows, n, g);
        // As for TC: a dense id range is ranked as is when the bit matrix is used.
        const bool dense = densify_ids(ctx, g, [&](u64 range) {
            try {
                return bitmat_choose(ctx, opt, range, true);
            } catch (const Error &) {
                return false;
            }
        });
        u64 ne;
        u64 *e = sg_edge_words(ctx, rows, n, g, ne);  // sg.cu:150-153
        build_csr(ctx, e, ne, g);                     // sg.cu:162
        if (dense || bitmat_choose(ctx, opt, g.n_ids, true)) {
            try {
                nfull = sg_bitmap_fixpoint(ctx, r, g, opt, pt);
                on_bitmat = true;
            } catch (const Error &err) {
                if (err.status != DL_ERR_OVERFLOW) throw;
                // a step outgrew the memory left for its new rows: the sorted runs
                // need no such bound; start over on them (same graph)
                r.deltas.clear();
                r.joins.clear();
                r.fulls.clear();
                r.from_bitmat = false;
                ctx.give_back(r.bm_t);
                ctx.give_back(r.bm_first);
                ctx.give_back(r.bm_off);
                nfull = 0;
            }
        }
    }
    if (n > 0 && !on_bitmat) {
        u64 ne;
        u64 *e = sg_edge_words(ctx, rows, n, g, ne);  // again: the bit-matrix attempt reused the buffers
        // Base rule (sg.cu:170-217): probe = deduplicated edges.
        u64 *selfs = &ctx.ctrl->scalar[8];
        DL_CUDA(cudaMemsetAsync(selfs, 0, sizeof(u64), ctx.stream));
        u64 nb = 0;
        u64 *b = join_and_sort(ctx, g, e, ne, EmitKind::ZV_NOSELF, nb, selfs, pt);
        DL_CUDA(cudaMemcpyAsync(ctx.host_scalars + 1, selfs, sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
        const u64 nvalid = nb - ctx.host_scalars[1];  // self pairs sorted to the end
        u64 nd = nvalid ? unique_words(ctx, b, nvalid, b) : 0;
        ctx.reserve(ws.full[0], std::max<u64>(nd, 1) * 8);
        if (nd) DL_CUDA(cudaMemcpyAsync(ws.full[0].p, b, nd * 8, cudaMemcpyDeviceToDevice, ctx.stream));
        F.cur = 0;
        F.nbig = nd;
        u64 *delta = b;
        u64 ndelta = nd;
        for (int it = 0;; ++it) {  // sg.cu:244-390
            u64 n1 = 0, n2 = 0, nnew = 0;
            u64 *j1 = join_and_sort(ctx, g, delta, ndelta, EmitKind::VZ, n1, nullptr, pt);  // (b, x)
            pt.mark(PH_DEDUP);
            if (n1) n1 = unique_words(ctx, j1, n1, j1);  // sg.cu:282-287
            if (n1) {
                u64 *j2 = join_and_sort(ctx, g, j1, n1, EmitKind::VZ, n2, nullptr, pt);  // (x, y)
                pt.mark(PH_MERGE);
                delta = absorb(ctx, F, j2, n2, nnew);  // sg.cu:349-368
            }
            ndelta = nnew;
            r.deltas.push_back((i64) nnew);
            r.joins.push_back((i64) (n1 + n2));
            r.fulls.push_back((i64) F.size());
            if (nnew == 0) break;
            if (opt.max_iterations > 0 && it + 1 >= opt.max_iterations) break;
        }
        settle(ctx, F);
        nfull = F.nbig;
        cur = F.cur;
    }
    pt.mark(PH_FINAL);
    DL_CUDA(cudaEventRecord(ev.b, ctx.stream));
    pt.mark(PH_FINAL);
    adopt_ids(ctx, r, g);
    if (!on_bitmat) {
        r.words = ws.full[cur];
        ws.full[cur] = DevBuf();
        r.n_words = nfull;
    }
    r.info.output_rows = r.info.output_tuples = (i64) nfull;
    finish_info(r, ctx, ev.a, ev.b, pt);
}

// WCC (wcc.cu:58-585): symmetric edges, cc(n, n), min-label propagation from
// the changed nodes only; stop rule per dl_wcc_stop.
static void run_wcc_impl(Context &ctx, Run &r, const int32_t *rows_in, u64 n, bool on_device, const dl_options &opt) {
    Workspace &ws = ctx.ws;
    PhaseTimer pt(ctx, opt.phase_timing != 0);
    EventPair ev;
    DL_CUDA(cudaEventRecord(ev.a, ctx.stream));
    pt.mark(PH_INIT);
    const int32_t *rows = stage_input(ctx, rows_in, n, on_device);
    Graph g;
    if (n > 0) {
        rank_nodes(ctx, rows, n, g);
        ctx.reserve(ws.jbuf[0], 2 * n * 8);
        ctx.reserve(ws.jbuf[1], 2 * n * 8);
        u64 *w = ws.jbuf[0].as<u64>();
        DL_LAUNCH(ctx, K_PREP, 0, pack_rows_kernel<<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(rows, n, g.ids, g.n_ids, g.bits, w, w + n));
        u64 ne;
        u64 *e = sort_unique_into(ctx, ws.jbuf[0], ws.jbuf[1], 2 * n, 2 * g.bits, ne);  // wcc.cu:140-167
        build_csr(ctx, e, ne, g);
        const u32 nn = g.n_ids;
        ctx.reserve(ws.wcc_label, (u64) nn * 4);
        ctx.reserve(ws.wcc_flag, (u64) nn * 4);
        ctx.reserve(ws.wcc_next, ((u64) nn + 1) * 4);
        ctx.reserve(ws.w0, (u64) nn * 8);
        ctx.reserve(ws.w1, (u64) nn * 8);
        u32 *label = ws.wcc_label.as<u32>(), *flag = ws.wcc_flag.as<u32>(), *next = ws.wcc_next.as<u32>();
        u64 *dcur = ws.w0.as<u64>(), *dnext = ws.w1.as<u64>();
        DL_LAUNCH(ctx, K_PREP, 0, wcc_init_kernel<<<grid_for(nn, T256, ctx), T256, 0, ctx.stream>>>(nn, label, flag, dcur));  // wcc.cu:211-231
        DL_CHECK_LAUNCH();
        u32 *next_count = reinterpret_cast<u32 *>(&ctx.ctrl->scalar[9]);
        u64 ndelta = nn;
        i64 prev = (i64) nn;
        for (int it = 0;; ++it) {  // wcc.cu:255-387
            pt.mark(PH_JOIN);
            ctx.reserve(ws.offsets, std::max<u64>(ndelta, 1) * 8);
            DL_CUDA(cudaMemsetAsync(next_count, 0, sizeof(u32), ctx.stream));
            WccSrc src{g.csr.off, g.csr.val, dcur, label, flag, next, next_count};
            const u64 total = count_matches(ctx, src, ndelta, ws.offsets.as<u64>());
            ctx.run_join_total += total;
            ctx.run_join_max = std::max(ctx.run_join_max, total);
            if (total) emit_matches(ctx, src, ndelta, ws.offsets.as<u64>(), total, nullptr, nullptr, 0, nullptr);
            pt.mark(PH_MERGE);
            DL_CUDA(cudaMemcpyAsync(ctx.host_scalars + 2, next_count, sizeof(u32), cudaMemcpyDeviceToHost, ctx.stream));
            ctx.sync();
            const u64 nnew = *reinterpret_cast<u32 *>(ctx.host_scalars + 2);
            if (nnew) {
                DL_LAUNCH(ctx, K_PREP, 0, wcc_next_delta_kernel<<<grid_for(nnew, T256, ctx), T256, 0, ctx.stream>>>(next, nnew, label, flag, dnext));
            }
            std::swap(dcur, dnext);
            ndelta = nnew;
            r.deltas.push_back((i64) nnew);
            r.joins.push_back((i64) total);
            r.fulls.push_back((i64) nn);
            if (opt.wcc_stop == DL_WCC_STOP_FIXPOINT) {
                if (nnew == 0) break;
            } else if ((i64) nnew == prev) {
                break;  // wcc.cu:366-383
            }
            prev = (i64) nnew;
            if (opt.max_iterations > 0 && it + 1 >= opt.max_iterations) break;
        }
        // Finalize (wcc.cu:389-472): component ids and the largest size.
        pt.mark(PH_FINAL);
        u32 *cnt = reinterpret_cast<u32 *>(ws.w1.p);  // reuse: nn u32 counters
        DL_CUDA(cudaMemsetAsync(cnt, 0, (u64) nn * 4, ctx.stream));
        DL_LAUNCH(ctx, K_PREP, 0, wcc_count_kernel<<<grid_for(nn, T256, ctx), T256, 0, ctx.stream>>>(label, nn, cnt));
        u64 *pos = ws.w0.as<u64>();
        u64 *largest = &ctx.ctrl->scalar[10];
        DL_CUDA(cudaMemsetAsync(largest, 0, sizeof(u64), ctx.stream));
        const u64 ncomp = count_matches(ctx, NonZeroCounter{cnt}, nn, pos);
        ctx.reserve(r.aux, std::max<u64>(ncomp, 1) * 4);
        DL_LAUNCH(ctx, K_PREP, 0, wcc_components_kernel<<<grid_for(nn, T256, ctx), T256, 0, ctx.stream>>>(
            cnt, nn, pos, r.aux.as<u32>(), reinterpret_cast<unsigned long long *>(largest)));
        DL_CUDA(cudaMemcpyAsync(ctx.host_scalars + 3, largest, sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
        r.n_aux = ncomp;
        r.info.output_rows = r.info.output_tuples = (i64) ncomp;
        r.info.largest_component = (i64) ctx.host_scalars[3];
        // Keep the per-node labels with the run.
        r.labels = ws.wcc_label;
        ws.wcc_label = DevBuf();
    }
    DL_CUDA(cudaEventRecord(ev.b, ctx.stream));
    pt.mark(PH_FINAL);
    adopt_ids(ctx, r, g);
    finish_info(r, ctx, ev.a, ev.b, pt);
}

// single_join (single_join.cu:135-309): R deduplicated and keyed by a; probe
// = dedup(R reversed); J = (c, a) for R(b, c), R(a, b); dedup.
static void run_single_join_impl(Context &ctx, Run &r, const int32_t *rows_in, u64 n, bool on_device,
                                 const dl_options &opt) {
    Workspace &ws = ctx.ws;
    PhaseTimer pt(ctx, opt.phase_timing != 0);
    EventPair ev;
    DL_CUDA(cudaEventRecord(ev.a, ctx.stream));
    pt.mark(PH_INIT);
    const int32_t *rows = stage_input(ctx, rows_in, n, on_device);
    Graph g;
    u64 nout = 0;
    if (n > 0) {
        rank_nodes(ctx, rows, n, g);
        ctx.reserve(ws.jbuf[0], n * 8);
        ctx.reserve(ws.jbuf[1], n * 8);
        DL_LAUNCH(ctx, K_PREP, 0, pack_rows_kernel<<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(rows, n, g.ids, g.n_ids, g.bits,
                                                                         ws.w0.as<u64>(), ws.jbuf[0].as<u64>()));
        u64 ne, np;
        u64 *e = sort_unique_into(ctx, ws.w0, ws.w1, n, 2 * g.bits, ne);  // single_join.cu:165-168
        build_csr(ctx, e, ne, g);
        u64 *p = sort_unique_into(ctx, ws.jbuf[0], ws.jbuf[1], n, 2 * g.bits, np);  // single_join.cu:200-203
        u64 nj = 0;
        u64 *j = join_and_sort(ctx, g, p, np, EmitKind::ZV, nj, nullptr, pt);  // single_join.cu:223
        nout = nj ? unique_words(ctx, j, nj, j) : 0;                           // single_join.cu:259-264
        DevBuf &hold = holder(ws, j);
        r.words = hold;
        hold = DevBuf();
        r.n_words = nout;
        r.deltas.push_back((i64) nout);
    }
    DL_CUDA(cudaEventRecord(ev.b, ctx.stream));
    pt.mark(PH_FINAL);
    adopt_ids(ctx, r, g);
    r.info.output_rows = r.info.output_tuples = (i64) nout;
    finish_info(r, ctx, ev.a, ev.b, pt);
}

Run *run_program(Context &ctx, int program, const int32_t *rows, u64 n, bool on_device, const dl_options &opt) {
    auto r = new Run();
    r->ctx = &ctx;
    r->program = (dl_program) program;
    r->info.program = program;
    r->info.input_rows = (i64) n;
    ctx.run_join_total = ctx.run_join_max = 0;
    try {
        switch (program) {
            case DL_PROGRAM_TC:
                if (opt.dedup == DL_DEDUP_HASH) run_tc_hash_impl(ctx, *r, rows, n, on_device, opt);
                else run_tc_impl(ctx, *r, rows, n, on_device, opt);
                break;
            case DL_PROGRAM_SG: run_sg_impl(ctx, *r, rows, n, on_device, opt); break;
            case DL_PROGRAM_WCC: run_wcc_impl(ctx, *r, rows, n, on_device, opt); break;
            case DL_PROGRAM_SINGLE_JOIN: run_single_join_impl(ctx, *r, rows, n, on_device, opt); break;
            default: throw Error(DL_ERR_INVALID_ARGUMENT, "unknown program " + std::to_string(program));
        }
    } catch (...) {
        run_destroy(r);
        throw;
    }
    return r;
}

// Result rows [a, b) of a run into tmp + 2a (device memory). A bit-matrix
// run's rows leave by units (TC column blocks, SG matrix rows): ua/ub are
// then the units whose rows are [a, b).
static void extract_range(Context &ctx, const Run &r, int32_t *tmp, u64 a, u64 b, u64 ua, u64 ub) {
    const int32_t *ids = r.ids.as<int32_t>();
    const u64 n = b - a;
    if (r.from_bitmat) {
        bitmat_extract_rows(ctx, r, tmp, ua, ub);
        ctx.prof_add_bytes(K_BITMAP_EXTRACT, 8.0 * n);
    } else if (r.program == DL_PROGRAM_WCC) {
        DL_LAUNCH(ctx, K_PREP, 0, unpack_components_kernel<<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(
                                      r.aux.as<u32>() + a, n, ids, tmp + 2 * a));
    } else if (r.program == DL_PROGRAM_SG) {
        DL_LAUNCH(ctx, K_PREP, 0, unpack_rows_kernel<true><<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(
                                      r.words.as<u64>() + a, n, r.bits, ids, tmp + 2 * a));
    } else {
        DL_LAUNCH(ctx, K_PREP, 0, unpack_rows_kernel<false><<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(
                                      r.words.as<u64>() + a, n, r.bits, ids, tmp + 2 * a));
    }
    DL_CHECK_LAUNCH();
}

void run_copy_output(const Run &r, int32_t *dst, u64 capacity, bool dst_on_device) {
    Context &ctx = *r.ctx;
    const u64 n = (u64) r.info.output_rows;
    if (capacity < n) throw Error(DL_ERR_INVALID_ARGUMENT, "output capacity " + std::to_string(capacity) + " < " +
                                                               std::to_string(n) + " rows");
    if (n == 0) return;
    const u64 units = r.from_bitmat ? bitmat_units(r) : n;
    if (dst_on_device) {
        extract_range(ctx, r, dst, 0, n, 0, units);
        ctx.sync();
        return;
    }
    // Host destination: the rows are written to a device stage in chunks, and
    // each chunk's copy to the host runs on a second stream while the next
    // chunk is written.
    DevBuf stage;
    ctx.reserve(stage, n * 8);
    int32_t *tmp = stage.as<int32_t>();
    const int kchunks = (int) std::min<u64>(n * 8 >= (256ull << 20) ? 8 : 1, units);
    u64 *bound = ctx.host_scalars + 16;  // row bounds of the chunks (kchunks + 1 <= 9 slots)
    std::vector<u64> ubound(kchunks + 1);
    for (int k = 0; k <= kchunks; ++k) ubound[k] = units * k / kchunks;
    if (r.from_bitmat) {
        for (int k = 0; k <= kchunks; ++k) {
            const u64 idx = bitmat_unit_index(r, ubound[k]);
            if (idx >= r.bm_n) bound[k] = n;
            else DL_CUDA(cudaMemcpyAsync(bound + k, r.bm_first.as<u64>() + idx, 8, cudaMemcpyDeviceToHost, ctx.stream));
        }
        ctx.sync();
    } else {
        for (int k = 0; k <= kchunks; ++k) bound[k] = ubound[k];
    }
    std::vector<u64> rows(bound, bound + kchunks + 1);
    cudaStream_t cs = ctx.copy_stream_get();
    std::vector<cudaEvent_t> ev(kchunks, nullptr);
    try {
        for (int k = 0; k < kchunks; ++k) {
            if (rows[k + 1] <= rows[k]) continue;
            extract_range(ctx, r, tmp, rows[k], rows[k + 1], ubound[k], ubound[k + 1]);
            DL_CUDA(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
            DL_CUDA(cudaEventRecord(ev[k], ctx.stream));
            DL_CUDA(cudaStreamWaitEvent(cs, ev[k], 0));
            DL_CUDA(cudaMemcpyAsync(dst + 2 * rows[k], tmp + 2 * rows[k], (rows[k + 1] - rows[k]) * 8,
                                    cudaMemcpyDeviceToHost, cs));
        }
        DL_CUDA(cudaStreamSynchronize(cs));
    } catch (...) {
        cudaStreamSynchronize(cs);
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        ctx.give_back(stage);
        throw;
    }
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    ctx.sync();
    ctx.give_back(stage);
}

void run_copy_labels(const Run &r, int32_t *node_ids, int32_t *labels, u64 capacity) {
    Context &ctx = *r.ctx;
    if (r.program != DL_PROGRAM_WCC) throw Error(DL_ERR_INVALID_ARGUMENT, "labels exist only for WCC runs");
    const u64 n = r.n_ids;
    if (capacity < n) throw Error(DL_ERR_INVALID_ARGUMENT, "label capacity too small");
    if (n == 0) return;
    DevBuf stage;
    ctx.reserve(stage, n * 4);
    DL_LAUNCH(ctx, K_PREP, 0, unpack_labels_kernel<<<grid_for(n, T256, ctx), T256, 0, ctx.stream>>>(r.labels.as<u32>(), (u32) n,
                                                                         r.ids.as<int32_t>(), stage.as<int32_t>()));
    DL_CUDA(cudaMemcpyAsync(labels, stage.p, n * 4, cudaMemcpyDeviceToHost, ctx.stream));
    DL_CUDA(cudaMemcpyAsync(node_ids, r.ids.p, n * 4, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    ctx.give_back(stage);
}

void run_destroy(Run *r) {
    if (!r) return;
    if (r->ctx) {
        r->ctx->give_back(r->words);
        r->ctx->give_back(r->ids);
        r->ctx->give_back(r->aux);
        r->ctx->give_back(r->labels);
        r->ctx->give_back(r->bm_t);
        r->ctx->give_back(r->bm_first);
        r->ctx->give_back(r->bm_off);
        r->ctx->give_back(r->bm_live);
    }
    delete r;
}

}  // namespace dl
