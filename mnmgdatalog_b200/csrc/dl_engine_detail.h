// Engine helpers shared by the single-run drivers (dl_engine.cu) and the
// multi-instance session (dl_session.cu).
#pragma once

#include "dl_engine.h"
#include "dl_internal.h"

namespace dl {
namespace detail {

constexpr int T256 = 256;

inline unsigned grid_for(u64 n, int threads, const Context &ctx, int per_sm = 16) {
    u64 g = (n + threads - 1) / threads;
    const u64 cap = (u64) ctx.sm_count * per_sm;
    if (g > cap) g = cap;
    if (g == 0) g = 1;
    return (unsigned) g;
}

// Device-time accounting per phase (the reference's CSV breakdown).
struct PhaseTimer {
    Context &ctx;
    bool on;
    std::vector<std::pair<int, cudaEvent_t>> marks;
    explicit PhaseTimer(Context &c, bool enabled) : ctx(c), on(enabled) {}
    ~PhaseTimer() {
        for (auto &m : marks) cudaEventDestroy(m.second);
    }
    void mark(int phase) {  // a new phase starts now
        if (!on) return;
        cudaEvent_t e;
        DL_CUDA(cudaEventCreate(&e));
        DL_CUDA(cudaEventRecord(e, ctx.stream));
        marks.emplace_back(phase, e);
    }
    void finish(double out[5]) {
        for (int i = 0; i < 5; ++i) out[i] = 0;
        if (!on || marks.size() < 2) return;
        DL_CUDA(cudaEventSynchronize(marks.back().second));
        for (size_t i = 0; i + 1 < marks.size(); ++i) {
            float ms = 0;
            DL_CUDA(cudaEventElapsedTime(&ms, marks[i].second, marks[i + 1].second));
            out[marks[i].first] += ms * 1e-3;
        }
    }
};
enum { PH_INIT = 0, PH_JOIN = 1, PH_DEDUP = 2, PH_MERGE = 3, PH_FINAL = 4 };

struct Graph {
    u32 n_ids = 0;
    int bits = 1;
    int32_t *ids = nullptr;
    // ids[r] == id_base + r for every rank (the ranks cover a dense id range)
    bool ids_affine = false;
    int32_t id_base = 0;
    Csr csr;
    // Radix windows of join-output sorts; 0 = every digit of [0, 2 * bits).
    int nwin = 0;
    int win[8] = {};
};

// The full relation of TC/SG as disjoint sorted duplicate-free runs: large
// (ws.full[cur]), small (ws.small[scur]) and, when `three` is set, tiny
// (ws.tiny[tcur]). A tiny run is only non-empty while the small run is.
struct FullSet {
    int cur = 0;
    u64 nbig = 0;
    int scur = 0;
    u64 nsmall = 0;
    u64 ns = 0;
    bool sample_ok = false;
    bool three = false;       // use the tiny run
    int tcur = 0;
    u64 ntiny = 0;
    u64 nss = 0;              // sample of the small run
    bool ssample_ok = false;
    u64 size() const { return nbig + nsmall + ntiny; }
};


int bits_for(u64 n);
// Ranks over every id in [min id, max id] when that range is at most 1/8
// larger than the distinct ids (absent ids become ranks without edges):
// rank -> id is then id_base + rank, with no table lookup. Returns whether
// it did; `fits(range)` decides whether the caller can use that many ranks.
template <class Fits>
bool densify_ids(Context &ctx, Graph &g, Fits fits);
const int32_t *stage_input(Context &ctx, const int32_t *rows, u64 n, bool on_device);
void rank_nodes(Context &ctx, const int32_t *rows, u64 n, Graph &g);
u64 *sort_unique_into(Context &ctx, DevBuf &buf, DevBuf &alt, u64 n, int key_bits, u64 &n_out);
DevBuf &holder(Workspace &ws, const u64 *p);
DevBuf &other(Workspace &ws, const u64 *p);
u64 *join_and_sort(Context &ctx, const Graph &g, const u64 *probe, u64 n_probe, EmitKind kind, u64 &n_j,
                   u64 *self_pairs, PhaseTimer &pt);
u64 *join_unsorted(Context &ctx, const Graph &g, const u64 *probe, u64 n_probe, EmitKind kind, u64 &n_j,
                   PhaseTimer &pt);
u64 *absorb(Context &ctx, FullSet &F, u64 *j, u64 nj, u64 &n_delta);
void fold_tiny(Context &ctx, FullSet &F);
void settle(Context &ctx, FullSet &F);

// TC with full as an n x n bit matrix (dl_bitmap.cu).
u64 bitmat_bytes(u64 n);
// Whether a run over n node ranks keeps full as an n x n bit matrix: the
// matrix, and for TC (sg false) its result rows' column offsets, must fit.
bool bitmat_choose(Context &ctx, const dl_options &opt, u64 n, bool sg);
u64 tc_bitmap_fixpoint(Context &ctx, Run &r, const Graph &g, const u64 *edges, u64 ne, const dl_options &opt,
                       PhaseTimer &pt);
// SG with full as a bit matrix; throws DL_ERR_OVERFLOW when a step's new rows
// outgrow the buffer the device memory allows (the caller then reruns SG on
// the sorted runs).
u64 sg_bitmap_fixpoint(Context &ctx, Run &r, const Graph &g, const dl_options &opt, PhaseTimer &pt);

}  // namespace detail
}  // namespace dl
