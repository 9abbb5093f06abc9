// extern "C" boundary of libmnmgdl.so (declared in include/mnmgdl.h).
#include <cstring>
#include <memory>

#include "dl_engine.h"
#include "dl_internal.h"
#include "dl_join.cuh"
#include "dl_session.h"

struct dl_context {
    dl::Context c;
};
struct dl_hash_table {
    dl::HashTable *ht = nullptr;
    dl_context *ctx = nullptr;
};
struct dl_run {
    dl::Run *r = nullptr;
};
struct dl_session {
    dl::SessionImpl *s = nullptr;
    dl_context *ctx = nullptr;
};

namespace {

thread_local std::string g_last_error;

dl_status fail(dl_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

template <class F>
dl_status guarded(F &&f) {
    try {
        f();
        return DL_OK;
    } catch (const dl::Error &e) {
        return fail(e.status, e.what());
    } catch (const std::bad_alloc &) {
        return fail(DL_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(DL_ERR_INTERNAL, e.what());
    }
}

#define DL_REQUIRE(cond, msg)                                          \
    do {                                                               \
        if (!(cond)) return fail(DL_ERR_INVALID_ARGUMENT, (msg));      \
    } while (0)

using dl::u64;

void set_device(dl_context *ctx) { DL_CUDA(cudaSetDevice(ctx->c.device)); }

// glibc random_r TYPE_3 additive feedback generator (r[i] = r[i-3] + r[i-31],
// seeded by the Park-Miller LCG 16807 mod 2^31-1, first 310 outputs
// discarded, results r >> 1), i.e. what rand() returns after srand(seed).
struct GlibcRand {
    int32_t r[34];
    uint32_t ring[31];
    int idx = 0;
    explicit GlibcRand(uint32_t seed) {
        int32_t s = (int32_t) (seed == 0 ? 1 : seed);
        int32_t t[344];
        t[0] = s;
        for (int i = 1; i < 31; ++i) {
            const int64_t hi = t[i - 1] / 127773, lo = t[i - 1] % 127773;
            int64_t w = 16807 * lo - 2836 * hi;
            if (w < 0) w += 2147483647;
            t[i] = (int32_t) w;
        }
        for (int i = 31; i < 34; ++i) t[i] = t[i - 31];
        uint32_t u[344];
        for (int i = 0; i < 34; ++i) u[i] = (uint32_t) t[i];
        for (int i = 34; i < 344; ++i) u[i] = u[i - 31] + u[i - 3];
        for (int i = 0; i < 31; ++i) ring[i] = u[313 + i];  // u[i-31] .. u[i-1] for i = 344
        idx = 0;
    }
    int32_t next() {
        // ring holds the last 31 values, oldest at idx.
        const uint32_t v = ring[idx] + ring[(idx + 28) % 31];
        ring[idx] = v;
        idx = (idx + 1) % 31;
        return (int32_t) (v >> 1);
    }
};

}  // namespace

namespace dl {
// Error text for dl_last_error() from entry points defined in other files.
void set_last_error(const std::string &msg) { g_last_error = msg; }
}  // namespace dl

extern "C" {

DL_API const char *dl_status_string(dl_status s) {
    switch (s) {
        case DL_OK: return "ok";
        case DL_ERR_INVALID_ARGUMENT: return "invalid argument";
        case DL_ERR_CUDA: return "CUDA error";
        case DL_ERR_OUT_OF_MEMORY: return "out of device memory";
        case DL_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
        case DL_ERR_OVERFLOW: return "size overflow";
        case DL_ERR_NO_DEVICE: return "no CUDA device";
        case DL_ERR_INTERNAL: return "internal error";
    }
    return "unknown status";
}

DL_API const char *dl_last_error(void) { return g_last_error.c_str(); }

DL_API const char *dl_version(void) { return "mnmgdl 0.1 (sm_100a)"; }

DL_API dl_status dl_context_create(int32_t device, void *stream, dl_context **out) {
    DL_REQUIRE(out != nullptr, "out is NULL");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        (void) cudaGetLastError();
        return fail(DL_ERR_NO_DEVICE, "no CUDA device visible");
    }
    DL_REQUIRE(device >= 0 && device < n, "device index out of range");
    auto ctx = std::make_unique<dl_context>();
    dl_status st = guarded([&] {
        dl::Context &c = ctx->c;
        c.device = device;
        DL_CUDA(cudaSetDevice(device));
        DL_CUDA(cudaDeviceGetAttribute(&c.sm_count, cudaDevAttrMultiProcessorCount, device));
        if (stream) {
            c.stream = (cudaStream_t) stream;
        } else {
            DL_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
            c.own_stream = true;
        }
        void *p = nullptr;
        DL_CUDA(cudaMalloc(&p, sizeof(dl::Ctrl)));
        DL_CUDA(cudaMemset(p, 0, sizeof(dl::Ctrl)));
        c.ctrl = (dl::Ctrl *) p;
        DL_CUDA(cudaMallocHost((void **) &c.host_scalars, 64 * sizeof(u64)));
        std::memset(c.host_scalars, 0, 64 * sizeof(u64));
    });
    if (st != DL_OK) {
        dl_context_destroy(ctx.release());
        return st;
    }
    *out = ctx.release();
    return DL_OK;
}

DL_API dl_status dl_context_destroy(dl_context *ctx) {
    if (!ctx) return DL_OK;
    cudaSetDevice(ctx->c.device);
    if (ctx->c.stream) cudaStreamSynchronize(ctx->c.stream);
    ctx->c.release_all();
    if (ctx->c.ctrl) cudaFree(ctx->c.ctrl);
    if (ctx->c.host_scalars) cudaFreeHost(ctx->c.host_scalars);
    if (ctx->c.own_stream && ctx->c.stream) cudaStreamDestroy(ctx->c.stream);
    delete ctx;
    return DL_OK;
}

DL_API dl_status dl_context_synchronize(dl_context *ctx) {
    DL_REQUIRE(ctx, "ctx is NULL");
    return guarded([&] {
        set_device(ctx);
        ctx->c.sync();
    });
}

DL_API dl_status dl_context_release_memory(dl_context *ctx) {
    DL_REQUIRE(ctx, "ctx is NULL");
    return guarded([&] {
        set_device(ctx);
        ctx->c.sync();
        ctx->c.release_all();
    });
}

DL_API dl_status dl_free(dl_context *ctx, void *p) {
    DL_REQUIRE(ctx, "ctx is NULL");
    if (!p) return DL_OK;
    return guarded([&] {
        set_device(ctx);
        DL_CUDA(cudaStreamSynchronize(ctx->c.stream));
        DL_CUDA(cudaFree(p));
    });
}

DL_API dl_status dl_memcpy(dl_context *ctx, void *dst, const void *src, int64_t bytes) {
    DL_REQUIRE(ctx && bytes >= 0 && (bytes == 0 || (dst && src)), "invalid argument");
    return guarded([&] {
        set_device(ctx);
        if (bytes) DL_CUDA(cudaMemcpyAsync(dst, src, (size_t) bytes, cudaMemcpyDefault, ctx->c.stream));
        ctx->c.sync();
    });
}

DL_API dl_status dl_sort(dl_context *ctx, dl_entity *rel, int64_t n) {
    DL_REQUIRE(ctx && (rel || n == 0) && n >= 0, "invalid argument");
    return guarded([&] {
        set_device(ctx);
        if (n <= 1) return;
        dl::DevBuf tmp;
        ctx->c.reserve(tmp, (u64) n * 8);
        u64 *s = dl::radix_sort(ctx->c, (u64 *) rel, tmp.as<u64>(), (u64) n, dl::Codec::Entity, 0);
        if (s != (u64 *) rel) DL_CUDA(cudaMemcpyAsync(rel, s, (u64) n * 8, cudaMemcpyDeviceToDevice, ctx->c.stream));
        ctx->c.sync();
        ctx->c.give_back(tmp);
    });
}

DL_API dl_status dl_sort_unique(dl_context *ctx, dl_entity *rel, int64_t n, int64_t *n_out) {
    DL_REQUIRE(ctx && n_out && (rel || n == 0) && n >= 0, "invalid argument");
    return guarded([&] {
        set_device(ctx);
        *n_out = 0;
        if (n == 0) return;
        dl::DevBuf tmp;
        ctx->c.reserve(tmp, (u64) n * 8);
        u64 *s = dl::radix_sort(ctx->c, (u64 *) rel, tmp.as<u64>(), (u64) n, dl::Codec::Entity, 0);
        *n_out = (int64_t) dl::unique_words(ctx->c, s, (u64) n, (u64 *) rel);
        ctx->c.give_back(tmp);
    });
}

DL_API dl_status dl_set_difference(dl_context *ctx, const dl_entity *a, int64_t na, const dl_entity *b, int64_t nb,
                                   dl_entity *out, int64_t *n_out) {
    DL_REQUIRE(ctx && n_out && na >= 0 && nb >= 0 && (a || na == 0) && (b || nb == 0) && (out || na == 0),
               "invalid argument");
    return guarded([&] {
        set_device(ctx);
        // a \ b == the new words of a against the set b.
        *n_out = (int64_t) dl::diff_merge_words(ctx->c, (const u64 *) b, (u64) nb, (const u64 *) a, (u64) na, nullptr,
                                                (u64 *) out, dl::Codec::Entity);
    });
}

DL_API dl_status dl_merge(dl_context *ctx, const dl_entity *a, int64_t na, const dl_entity *b, int64_t nb,
                          dl_entity *out) {
    DL_REQUIRE(ctx && na >= 0 && nb >= 0 && (a || na == 0) && (b || nb == 0) && (out || na + nb == 0),
               "invalid argument");
    return guarded([&] {
        set_device(ctx);
        dl::merge_words(ctx->c, (const u64 *) a, (u64) na, (const u64 *) b, (u64) nb, (u64 *) out, dl::Codec::Entity);
        ctx->c.sync();
    });
}

DL_API dl_status dl_diff_merge(dl_context *ctx, const dl_entity *full, int64_t nfull, const dl_entity *j, int64_t nj,
                               dl_entity *full_out, dl_entity *delta_out, int64_t *n_delta) {
    DL_REQUIRE(ctx && n_delta && nfull >= 0 && nj >= 0 && (full || nfull == 0) && (j || nj == 0), "invalid argument");
    DL_REQUIRE(full_out || delta_out, "full_out and delta_out are both NULL");
    return guarded([&] {
        set_device(ctx);
        *n_delta = (int64_t) dl::diff_merge_words(ctx->c, (const u64 *) full, (u64) nfull, (const u64 *) j, (u64) nj,
                                                  (u64 *) full_out, (u64 *) delta_out, dl::Codec::Entity);
    });
}

DL_API dl_status dl_unique_by_key_min(dl_context *ctx, dl_entity *rel, int64_t n, int64_t *n_out) {
    DL_REQUIRE(ctx && n_out && n >= 0 && (rel || n == 0), "invalid argument");
    return guarded([&] {
        set_device(ctx);
        *n_out = (int64_t) dl::unique_words(ctx->c, (const u64 *) rel, (u64) n, (u64 *) rel, 0, dl::Codec::Entity);
    });
}

DL_API dl_status dl_remove_self_pairs(dl_context *ctx, dl_entity *rel, int64_t n, int64_t *n_out) {
    DL_REQUIRE(ctx && n_out && n >= 0 && (rel || n == 0), "invalid argument");
    return guarded([&] {
        set_device(ctx);
        *n_out = (int64_t) dl::remove_self_pairs_words(ctx->c, (const u64 *) rel, (u64) n, (u64 *) rel);
    });
}

DL_API dl_status dl_partition(dl_context *ctx, const dl_entity *rel, int64_t n, int32_t ranks, int32_t swap_columns,
                              dl_entity *out, int64_t *counts) {
    DL_REQUIRE(ctx && counts && n >= 0 && (n == 0 || (rel && out && (const void *) rel != (const void *) out)) &&
                   ranks >= 1 && (u64) ranks <= dl::kMaxPartitionRanks,
               "invalid argument");
    return guarded([&] {
        set_device(ctx);
        dl::partition_rows(ctx->c, (const int32_t *) rel, (u64) n, (uint32_t) ranks, swap_columns != 0, (int32_t *) out,
                           counts);
    });
}

DL_API dl_status dl_build_hash_table(dl_context *ctx, const dl_entity *rel, int64_t n, double load_factor,
                                     dl_hash_table **out) {
    DL_REQUIRE(ctx && out && n >= 0 && (rel || n == 0), "invalid argument");
    *out = nullptr;
    auto h = std::make_unique<dl_hash_table>();
    h->ctx = ctx;
    dl_status st = guarded([&] {
        set_device(ctx);
        h->ht = dl::hash_table_build(ctx->c, (const u64 *) rel, (u64) n, load_factor);
    });
    if (st == DL_OK) *out = h.release();
    return st;
}

DL_API dl_status dl_hash_table_info(const dl_hash_table *ht, int64_t *slots, int64_t *distinct_keys, int64_t *rows) {
    DL_REQUIRE(ht && ht->ht, "ht is NULL");
    if (slots) *slots = (int64_t) ht->ht->slots;
    if (distinct_keys) *distinct_keys = (int64_t) ht->ht->distinct;
    if (rows) *rows = (int64_t) ht->ht->rows;
    return DL_OK;
}

DL_API dl_status dl_hash_table_destroy(dl_hash_table *ht) {
    if (!ht) return DL_OK;
    if (ht->ht) {
        cudaSetDevice(ht->ctx->c.device);
        cudaStreamSynchronize(ht->ctx->c.stream);
        ht->ht->table.release();
        ht->ht->vals.release();
        delete ht->ht;
    }
    delete ht;
    return DL_OK;
}

}  // extern "C"

namespace {

template <class Count, class Emit>
dl_status join_common(dl_context *ctx, int64_t n, dl_entity **out, int64_t *n_out, Count count, Emit emit) {
    return guarded([&] {
        set_device(ctx);
        *out = nullptr;
        *n_out = 0;
        if (n == 0) return;
        dl::DevBuf offs;
        ctx->c.reserve(offs, (u64) n * 8);
        const u64 total = count(offs.as<u64>());
        if (total) {
            void *p = nullptr;
            cudaError_t e = cudaMalloc(&p, total * 8);
            if (e != cudaSuccess) {
                (void) cudaGetLastError();
                ctx->c.give_back(offs);
                throw dl::Error(DL_ERR_OUT_OF_MEMORY, "join output of " + std::to_string(total) + " rows");
            }
            emit(offs.as<u64>(), total, (u64 *) p);
            ctx->c.sync();
            *out = (dl_entity *) p;
        }
        *n_out = (int64_t) total;
        ctx->c.give_back(offs);
    });
}

}  // namespace

extern "C" {

DL_API dl_status dl_join(dl_context *ctx, const dl_hash_table *ht, const dl_entity *probe, int64_t n, dl_entity **out,
                         int64_t *n_out) {
    DL_REQUIRE(ctx && ht && ht->ht && out && n_out && n >= 0 && (probe || n == 0), "invalid argument");
    const dl::HashTable &h = *ht->ht;
    const u64 *p = (const u64 *) probe;
    return join_common(
        ctx, n, out, n_out, [&](u64 *offs) { return dl::hash_join_count(ctx->c, h, p, (u64) n, offs); },
        [&](u64 *offs, u64 total, u64 *o) { dl::hash_join_emit(ctx->c, h, p, (u64) n, offs, total, o); });
}

DL_API dl_status dl_join_sorted(dl_context *ctx, const dl_entity *rel, int64_t n_rel, const dl_entity *probe,
                                int64_t n, dl_entity **out, int64_t *n_out) {
    DL_REQUIRE(ctx && out && n_out && n >= 0 && n_rel >= 0 && (probe || n == 0) && (rel || n_rel == 0),
               "invalid argument");
    const u64 *r = (const u64 *) rel;
    const u64 *p = (const u64 *) probe;
    return join_common(
        ctx, n, out, n_out, [&](u64 *offs) { return dl::sorted_join_count(ctx->c, r, (u64) n_rel, p, (u64) n, offs); },
        [&](u64 *offs, u64 total, u64 *o) { dl::sorted_join_emit(ctx->c, r, (u64) n_rel, p, (u64) n, offs, total, o); });
}

DL_API dl_status dl_run_program(dl_context *ctx, int32_t program, const int32_t *edges, int64_t rows,
                                int32_t edges_on_device, const dl_options *opts, dl_run **out) {
    DL_REQUIRE(ctx && out && rows >= 0 && (edges || rows == 0), "invalid argument");
    DL_REQUIRE(program >= DL_PROGRAM_TC && program <= DL_PROGRAM_SINGLE_JOIN, "unknown program");
    DL_REQUIRE(rows <= (int64_t) 0x7FFFFFFF, "more than 2^31-1 input rows");
    *out = nullptr;
    dl_options o{};
    if (opts) o = *opts;
    DL_REQUIRE(o.wcc_stop == DL_WCC_STOP_REFERENCE || o.wcc_stop == DL_WCC_STOP_FIXPOINT, "unknown wcc_stop");
    DL_REQUIRE(o.dedup >= DL_DEDUP_AUTO && o.dedup <= DL_DEDUP_BITMAP, "unknown dedup mode");
    auto run = std::make_unique<dl_run>();
    dl_status st = guarded([&] {
        set_device(ctx);
        run->r = dl::run_program(ctx->c, program, edges, (u64) rows, edges_on_device != 0, o);
    });
    if (st == DL_OK) *out = run.release();
    return st;
}

DL_API dl_status dl_run_tc(dl_context *ctx, const int32_t *e, int64_t rows, int32_t on_dev, const dl_options *o,
                           dl_run **out) {
    return dl_run_program(ctx, DL_PROGRAM_TC, e, rows, on_dev, o, out);
}
DL_API dl_status dl_run_sg(dl_context *ctx, const int32_t *e, int64_t rows, int32_t on_dev, const dl_options *o,
                           dl_run **out) {
    return dl_run_program(ctx, DL_PROGRAM_SG, e, rows, on_dev, o, out);
}
DL_API dl_status dl_run_wcc(dl_context *ctx, const int32_t *e, int64_t rows, int32_t on_dev, const dl_options *o,
                            dl_run **out) {
    return dl_run_program(ctx, DL_PROGRAM_WCC, e, rows, on_dev, o, out);
}
DL_API dl_status dl_run_single_join(dl_context *ctx, const int32_t *e, int64_t rows, int32_t on_dev,
                                    const dl_options *o, dl_run **out) {
    return dl_run_program(ctx, DL_PROGRAM_SINGLE_JOIN, e, rows, on_dev, o, out);
}

DL_API dl_status dl_run_get_info(const dl_run *run, dl_run_info *info) {
    DL_REQUIRE(run && run->r && info, "invalid argument");
    *info = run->r->info;
    return DL_OK;
}

DL_API dl_status dl_run_copy_output(const dl_run *run, int32_t *dst, int64_t capacity_rows, int32_t dst_on_device) {
    DL_REQUIRE(run && run->r && capacity_rows >= 0 && (dst || run->r->info.output_rows == 0), "invalid argument");
    return guarded([&] {
        DL_CUDA(cudaSetDevice(run->r->ctx->device));
        dl::run_copy_output(*run->r, dst, (u64) capacity_rows, dst_on_device != 0);
    });
}

DL_API dl_status dl_run_copy_deltas(const dl_run *run, int64_t *dst, int64_t capacity) {
    DL_REQUIRE(run && run->r && capacity >= 0, "invalid argument");
    const auto &d = run->r->deltas;
    DL_REQUIRE((int64_t) d.size() <= capacity, "delta capacity smaller than the iteration count");
    if (!d.empty()) std::memcpy(dst, d.data(), d.size() * sizeof(int64_t));
    return DL_OK;
}

DL_API dl_status dl_run_copy_iteration_stats(const dl_run *run, int64_t *join_rows, int64_t *full_rows,
                                             int64_t capacity) {
    DL_REQUIRE(run && run->r && capacity >= 0, "invalid argument");
    const auto &j = run->r->joins;
    const auto &f = run->r->fulls;
    DL_REQUIRE((int64_t) j.size() <= capacity, "capacity smaller than the iteration count");
    if (join_rows && !j.empty()) std::memcpy(join_rows, j.data(), j.size() * sizeof(int64_t));
    if (full_rows && !f.empty()) std::memcpy(full_rows, f.data(), f.size() * sizeof(int64_t));
    return DL_OK;
}

DL_API dl_status dl_run_copy_labels(const dl_run *run, int32_t *node_ids, int32_t *labels, int64_t capacity) {
    DL_REQUIRE(run && run->r && capacity >= 0, "invalid argument");
    return guarded([&] {
        DL_CUDA(cudaSetDevice(run->r->ctx->device));
        dl::run_copy_labels(*run->r, node_ids, labels, (u64) capacity);
    });
}

DL_API dl_status dl_run_destroy(dl_run *run) {
    if (!run) return DL_OK;
    if (run->r) {
        cudaSetDevice(run->r->ctx->device);
        dl::run_destroy(run->r);
    }
    delete run;
    return DL_OK;
}

// ---- sessions (dl_session.cu) ----

DL_API dl_status dl_session_create(dl_context *ctx, int32_t program, const dl_options *opts, int64_t max_nodes,
                                   dl_session **out) {
    DL_REQUIRE(ctx && out && max_nodes >= 0, "invalid argument");
    DL_REQUIRE(program == DL_PROGRAM_TC || program == DL_PROGRAM_SG || program == DL_PROGRAM_WCC,
               "sessions run TC, SG or WCC");
    *out = nullptr;
    dl_options o{};
    if (opts) o = *opts;
    DL_REQUIRE(o.wcc_stop == DL_WCC_STOP_REFERENCE || o.wcc_stop == DL_WCC_STOP_FIXPOINT, "unknown wcc_stop");
    DL_REQUIRE(o.dedup >= DL_DEDUP_AUTO && o.dedup <= DL_DEDUP_BITMAP, "unknown dedup mode");
    auto s = std::make_unique<dl_session>();
    s->ctx = ctx;
    dl_status st = guarded([&] {
        set_device(ctx);
        s->s = dl::session_create(ctx->c, program, o, (u64) max_nodes);
    });
    if (st == DL_OK) *out = s.release();
    return st;
}

DL_API dl_status dl_session_admit(dl_session *s, const int32_t *edges, int64_t rows, int32_t edges_on_device,
                                  int64_t *instance) {
    DL_REQUIRE(s && s->s && instance && rows >= 0 && (edges || rows == 0), "invalid argument");
    DL_REQUIRE(rows <= (int64_t) 0x7FFFFFFF, "more than 2^31-1 input rows");
    return guarded([&] {
        set_device(s->ctx);
        *instance = dl::session_admit(*s->s, edges, (u64) rows, edges_on_device != 0);
        dl::session_fold_profile(*s->s, s->ctx->c);
    });
}

DL_API dl_status dl_session_admit_many(dl_session *s, const int32_t *const *edges, const int64_t *rows,
                                       int64_t count, int32_t edges_on_device, int64_t *first_instance) {
    DL_REQUIRE(s && s->s && first_instance && count >= 0 && (count == 0 || (edges && rows)), "invalid argument");
    for (int64_t i = 0; i < count; ++i)
        DL_REQUIRE(rows[i] >= 0 && rows[i] <= (int64_t) 0x7FFFFFFF && (edges[i] || rows[i] == 0),
                   "invalid edge set");
    return guarded([&] {
        set_device(s->ctx);
        std::vector<u64> n(count);
        for (int64_t i = 0; i < count; ++i) n[i] = (u64) rows[i];
        const auto ids = dl::session_admit_many(*s->s, edges, n.data(), (u64) count, edges_on_device != 0);
        *first_instance = ids.empty() ? (int64_t) dl::session_instance_count(*s->s) : ids[0];
        dl::session_fold_profile(*s->s, s->ctx->c);
    });
}

DL_API dl_status dl_session_step(dl_session *s, int64_t *active) {
    DL_REQUIRE(s && s->s, "invalid argument");
    return guarded([&] {
        set_device(s->ctx);
        const u64 a = dl::session_step(*s->s);
        dl::session_fold_profile(*s->s, s->ctx->c);
        if (active) *active = (int64_t) a;
    });
}

DL_API dl_status dl_session_poll(dl_session *s, int64_t *ids, int64_t capacity, int64_t *count) {
    DL_REQUIRE(s && s->s && count && capacity >= 0 && (ids || capacity == 0), "invalid argument");
    return guarded([&] { *count = (int64_t) dl::session_poll(*s->s, ids, (u64) capacity); });
}

DL_API dl_status dl_session_get_info(const dl_session *s, int64_t instance, dl_run_info *info) {
    DL_REQUIRE(s && s->s && info, "invalid argument");
    return guarded([&] { dl::session_info(*s->s, instance, *info); });
}

DL_API dl_status dl_session_copy_output(dl_session *s, int64_t instance, int32_t *dst, int64_t capacity_rows,
                                        int32_t dst_on_device) {
    DL_REQUIRE(s && s->s && capacity_rows >= 0, "invalid argument");
    return guarded([&] {
        set_device(s->ctx);
        if (!dst && dl::session_instance(*s->s, instance).n_result)
            throw dl::Error(DL_ERR_INVALID_ARGUMENT, "dst is NULL");
        dl::session_copy_output(*s->s, instance, dst, (u64) capacity_rows, dst_on_device != 0);
    });
}

DL_API dl_status dl_session_copy_deltas(const dl_session *s, int64_t instance, int64_t *dst, int64_t capacity) {
    DL_REQUIRE(s && s->s && capacity >= 0, "invalid argument");
    return guarded([&] {
        const auto &d = dl::session_instance(*s->s, instance).deltas;
        if ((int64_t) d.size() > capacity)
            throw dl::Error(DL_ERR_INVALID_ARGUMENT, "delta capacity smaller than the iteration count");
        if (!d.empty()) std::memcpy(dst, d.data(), d.size() * sizeof(int64_t));
    });
}

DL_API dl_status dl_session_copy_labels(dl_session *s, int64_t instance, int32_t *node_ids, int32_t *labels,
                                        int64_t capacity) {
    DL_REQUIRE(s && s->s && capacity >= 0, "invalid argument");
    return guarded([&] {
        set_device(s->ctx);
        if ((!node_ids || !labels) && dl::session_instance(*s->s, instance).n_ids)
            throw dl::Error(DL_ERR_INVALID_ARGUMENT, "node_ids/labels is NULL");
        dl::session_copy_labels(*s->s, instance, node_ids, labels, (u64) capacity);
    });
}

DL_API dl_status dl_session_release(dl_session *s, int64_t instance) {
    DL_REQUIRE(s && s->s, "invalid argument");
    return guarded([&] {
        set_device(s->ctx);
        dl::session_release(*s->s, instance);
    });
}

DL_API dl_status dl_session_memory(const dl_session *s, int64_t *device_bytes, int64_t *active) {
    DL_REQUIRE(s && s->s, "invalid argument");
    if (device_bytes) *device_bytes = (int64_t) dl::session_device_bytes(*s->s);
    if (active) *active = (int64_t) dl::session_active(*s->s);
    return DL_OK;
}

DL_API dl_status dl_session_destroy(dl_session *s) {
    if (!s) return DL_OK;
    if (s->s) {
        cudaSetDevice(s->ctx->c.device);
        dl::session_destroy(s->s);
    }
    delete s;
    return DL_OK;
}

DL_API dl_status dl_run_batch(dl_context *ctx, int32_t program, const int32_t *const *edges, const int64_t *rows,
                              int64_t count, int32_t edges_on_device, const dl_options *opts, dl_session **out) {
    DL_REQUIRE(ctx && out && count >= 0 && (count == 0 || (edges && rows)), "invalid argument");
    for (int64_t i = 0; i < count; ++i)
        DL_REQUIRE(rows[i] >= 0 && rows[i] <= (int64_t) 0x7FFFFFFF && (edges[i] || rows[i] == 0),
                   "invalid edge set");
    *out = nullptr;
    u64 nodes = 0;  // upper bound on distinct nodes: two per edge row
    for (int64_t i = 0; i < count; ++i) nodes += 2 * (u64) rows[i];
    if (program == DL_PROGRAM_WCC || nodes == 0 || nodes >= (1ull << 30)) nodes = 0;
    dl_session *s = nullptr;
    dl_status st = dl_session_create(ctx, program, opts, (int64_t) nodes, &s);
    if (st != DL_OK) return st;
    st = guarded([&] {
        set_device(ctx);
        std::vector<u64> n(count);
        for (int64_t i = 0; i < count; ++i) n[i] = (u64) rows[i];
        dl::session_admit_many(*s->s, edges, n.data(), (u64) count, edges_on_device != 0);
        while (dl::session_step(*s->s) > 0) {
        }
        dl::session_fold_profile(*s->s, ctx->c);
    });
    if (st != DL_OK) {
        dl_session_destroy(s);
        return st;
    }
    *out = s;
    return DL_OK;
}

DL_API dl_status dl_context_get_tuning(const dl_context *ctx, dl_tuning *out) {
    DL_REQUIRE(ctx && out, "invalid argument");
    const dl::Tuning &t = ctx->c.tune;
    std::memset(out, 0, sizeof(*out));
    out->sort_algorithm = t.sort_algo;
    out->sort_ranking = t.rank;
    out->sort_keys_per_thread = t.sort_kpt;
    out->dense_ratio = (int32_t) t.dense_ratio;
    out->small_ratio = (int32_t) t.small_ratio;
    out->sort_input_tma = t.sort_tma;
    out->join_first_pass = t.join_first_pass;
    out->hash_load_factor = t.hash_load;
    out->bitmap_max_gib = t.bitmap_max_gib;
    out->bitmap_unit_rows = (int32_t) t.bitmap_unit_rows;
    out->cache_max_gib = t.cache_max_gib;
    out->bitmap_result = t.bitmap_result;
    return DL_OK;
}

DL_API dl_status dl_context_set_tuning(dl_context *ctx, const dl_tuning *t) {
    DL_REQUIRE(ctx && t, "invalid argument");
    DL_REQUIRE(t->sort_algorithm == 0 || t->sort_algorithm == 1, "sort_algorithm must be 0 or 1");
    DL_REQUIRE(t->sort_ranking == 0 || t->sort_ranking == 1, "sort_ranking must be 0 or 1");
    DL_REQUIRE(t->sort_keys_per_thread == 12 || t->sort_keys_per_thread == 16, "sort_keys_per_thread must be 12 or 16");
    DL_REQUIRE(t->dense_ratio >= 1 && t->dense_ratio <= 64, "dense_ratio must be in 1..64");
    DL_REQUIRE(t->small_ratio >= 1 && t->small_ratio <= 64, "small_ratio must be in 1..64");
    DL_REQUIRE(t->sort_input_tma == 0 || t->sort_input_tma == 1, "sort_input_tma must be 0 or 1");
    DL_REQUIRE(t->join_first_pass == 0 || t->join_first_pass == 1, "join_first_pass must be 0 or 1");
    DL_REQUIRE(t->hash_load_factor > 0.0 && t->hash_load_factor < 1.0, "hash_load_factor must be in (0, 1)");
    DL_REQUIRE(t->bitmap_max_gib >= 0 && t->bitmap_max_gib <= 1024, "bitmap_max_gib must be in 0..1024");
    DL_REQUIRE(t->bitmap_unit_rows >= 1 && t->bitmap_unit_rows <= (1 << 24), "bitmap_unit_rows must be in 1..16777216");
    DL_REQUIRE(t->cache_max_gib >= 0 && t->cache_max_gib <= 1024, "cache_max_gib must be in 0..1024");
    DL_REQUIRE(t->bitmap_result >= 0 && t->bitmap_result <= 2, "bitmap_result must be 0, 1 or 2");
    dl::Tuning &o = ctx->c.tune;
    o.sort_algo = t->sort_algorithm;
    o.rank = t->sort_ranking;
    o.sort_kpt = t->sort_keys_per_thread;
    o.dense_ratio = (u64) t->dense_ratio;
    o.small_ratio = (u64) t->small_ratio;
    o.sort_tma = t->sort_input_tma;
    o.join_first_pass = t->join_first_pass;
    o.hash_load = t->hash_load_factor;
    o.bitmap_max_gib = t->bitmap_max_gib;
    o.bitmap_unit_rows = (uint32_t) t->bitmap_unit_rows;
    o.cache_max_gib = t->cache_max_gib;
    o.bitmap_result = t->bitmap_result;
    ctx->c.trim_spares();
    return DL_OK;
}

DL_API dl_status dl_profile_enable(dl_context *ctx, int32_t enabled) {
    DL_REQUIRE(ctx, "ctx is NULL");
    return guarded([&] {
        set_device(ctx);
        ctx->c.sync();
        ctx->c.prof_reset();
        ctx->c.prof_on = enabled != 0;
    });
}

DL_API dl_status dl_profile_read(dl_context *ctx, dl_kernel_stat *out, int32_t capacity, int32_t *count) {
    DL_REQUIRE(ctx && count && capacity >= 0 && (out || capacity == 0), "invalid argument");
    return guarded([&] {
        set_device(ctx);
        ctx->c.sync();
        *count = dl::K_COUNT;
        for (int k = 0; k < dl::K_COUNT && k < capacity; ++k) {
            std::memset(&out[k], 0, sizeof(dl_kernel_stat));
            std::strncpy(out[k].name, dl::kernel_name(k), sizeof(out[k].name) - 1);
            out[k].launches = (int64_t) ctx->c.kstat[k].launches;
            out[k].timed_launches = (int64_t) ctx->c.kstat[k].timed;
            out[k].seconds = ctx->c.kstat[k].seconds;
            out[k].bytes = ctx->c.kstat[k].bytes;
        }
    });
}

DL_API dl_status dl_generate_rows(int64_t rows, int32_t rand_range, uint32_t seed, int32_t *host_out) {
    DL_REQUIRE(rows >= 0 && rand_range > 0 && (host_out || rows == 0), "invalid argument");
    GlibcRand g(seed);
    for (int64_t i = 0; i < 2 * rows; ++i) host_out[i] = (g.next() % rand_range) + 1;
    return DL_OK;
}

}  // extern "C"
