// The reference's operator entry points (declared in include/mnmgdl_compat.h):
// get_hash_table / get_join / get_join_nl semantics on top of the engine,
// with the reference's ownership (caller cudaFree's every result) and error
// behaviour (print, exit(code)).
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>

struct Entity;  // the caller's type; only the extern "C" entry points are used here
#include "../../include/mnmgdl_compat.h"
#include "dl_internal.h"
#include "dl_join.cuh"

namespace {

using dl::u64;

constexpr u64 kCompatMagic = 0x4D4E4D47444C4854ull;  // "MNMGDLHT"
constexpr u64 kHeaderBytes = 256;

struct CompatHeader {
    u64 magic;
    u64 slots;
    u64 distinct;
    u64 rows;
};

std::mutex g_mu;
dl::Context *g_ctx[64];

[[noreturn]] void die(int code, const std::string &msg) {
    fprintf(stderr, "GPUassert: %s\n", msg.c_str());
    exit(code ? code : 1);
}

dl::Context &compat_context() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) die(1, "no CUDA device");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx[dev]) {
        auto *c = new dl::Context();
        c->device = dev;
        c->stream = cudaStreamLegacy;  // the reference's blocking default stream
        cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, dev);
        void *p = nullptr;
        if (cudaMalloc(&p, sizeof(dl::Ctrl)) != cudaSuccess) die(2, "cudaMalloc of the control block failed");
        cudaMemset(p, 0, sizeof(dl::Ctrl));
        c->ctrl = (dl::Ctrl *) p;
        if (cudaMallocHost((void **) &c->host_scalars, 64 * sizeof(u64)) != cudaSuccess) die(2, "cudaMallocHost failed");
        std::memset(c->host_scalars, 0, 64 * sizeof(u64));
        g_ctx[dev] = c;
    }
    return *g_ctx[dev];
}

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class F>
auto guarded_exit(F &&f) -> decltype(f()) {
    try {
        return f();
    } catch (const dl::Error &e) {
        die((int) e.status, e.what());
    } catch (const std::exception &e) {
        die(1, e.what());
    }
}

dl_entity *to_int_result(dl::Context &ctx, u64 total, int *out_n) {
    if (total > 0x7FFFFFFFull)
        die((int) DL_ERR_OVERFLOW, "join result of " + std::to_string(total) + " rows exceeds the reference's int size");
    *out_n = (int) total;
    return nullptr;
}

}  // namespace

extern "C" {

DL_API dl_entity *dl_compat_get_hash_table(int, int, dl_entity *relation, int relation_size, int *hash_table_size,
                                           double *compute_time) {
    const double t0 = now();
    dl_entity *blob = nullptr;
    if (relation_size <= 0) {  // common/hash_table.cu:30-35
        *hash_table_size = 0;
        *compute_time = now() - t0;
        return nullptr;
    }
    guarded_exit([&] {
        dl::Context &ctx = compat_context();
        dl::HashTable *ht = dl::hash_table_build(ctx, (const u64 *) relation, (u64) relation_size, 0.5);
        const u64 bytes = kHeaderBytes + ht->slots * sizeof(dl::HashSlot) + ht->rows * sizeof(uint32_t);
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) die((int) DL_ERR_OUT_OF_MEMORY, "cudaMalloc of the hash table failed");
        CompatHeader h{kCompatMagic, ht->slots, ht->distinct, ht->rows};
        char *c = (char *) p;
        DL_CUDA(cudaMemcpy(c, &h, sizeof(h), cudaMemcpyHostToDevice));
        DL_CUDA(cudaMemcpy(c + kHeaderBytes, ht->table.p, ht->slots * sizeof(dl::HashSlot), cudaMemcpyDeviceToDevice));
        DL_CUDA(cudaMemcpy(c + kHeaderBytes + ht->slots * sizeof(dl::HashSlot), ht->vals.p, ht->rows * sizeof(uint32_t),
                           cudaMemcpyDeviceToDevice));
        ht->table.release();
        ht->vals.release();
        delete ht;
        if (h.slots > 0x7FFFFFFFull) die((int) DL_ERR_OVERFLOW, "hash table exceeds the reference's int size");
        *hash_table_size = (int) h.slots;
        blob = (dl_entity *) p;
        return 0;
    });
    *compute_time = now() - t0;
    return blob;
}

DL_API dl_entity *dl_compat_get_join(int, int, dl_entity *hash_table, int hash_table_size, dl_entity *relation,
                                     int relation_size, int *join_result_size, double *compute_time) {
    const double t0 = now();
    dl_entity *result = nullptr;
    *join_result_size = 0;
    if (hash_table_size == 0 || hash_table == nullptr || relation_size <= 0) {  // common/join.cu:56-62
        *compute_time = now() - t0;
        return nullptr;
    }
    guarded_exit([&] {
        dl::Context &ctx = compat_context();
        CompatHeader h;
        DL_CUDA(cudaMemcpy(&h, hash_table, sizeof(h), cudaMemcpyDeviceToHost));
        if (h.magic != kCompatMagic || h.slots != (u64) hash_table_size)
            die((int) DL_ERR_INVALID_ARGUMENT, "get_join: not a table made by get_hash_table");
        dl::HashTable view;  // non-owning view over the blob
        view.table.p = (char *) hash_table + kHeaderBytes;
        view.vals.p = (char *) hash_table + kHeaderBytes + h.slots * sizeof(dl::HashSlot);
        view.slots = h.slots;
        view.distinct = h.distinct;
        view.rows = h.rows;
        dl::DevBuf offs;
        ctx.reserve(offs, (u64) relation_size * 8);
        const u64 total = dl::hash_join_count(ctx, view, (const u64 *) relation, (u64) relation_size, offs.as<u64>());
        to_int_result(ctx, total, join_result_size);
        if (total) {
            void *p = nullptr;
            if (cudaMalloc(&p, total * 8) != cudaSuccess) die((int) DL_ERR_OUT_OF_MEMORY, "cudaMalloc of the join result failed");
            dl::hash_join_emit(ctx, view, (const u64 *) relation, (u64) relation_size, offs.as<u64>(), total, (u64 *) p);
            ctx.sync();
            result = (dl_entity *) p;
        }
        view.table.p = view.vals.p = nullptr;
        ctx.give_back(offs);
        return 0;
    });
    *compute_time = now() - t0;
    return result;
}

DL_API dl_entity *dl_compat_get_join_nl(int, int, dl_entity *sorted_relation, int sorted_relation_size,
                                        dl_entity *relation, int relation_size, int *join_result_size,
                                        double *compute_time) {
    const double t0 = now();
    dl_entity *result = nullptr;
    *join_result_size = 0;
    if (sorted_relation_size <= 0 || relation_size <= 0) {  // common/join.cu:149-155
        *compute_time = now() - t0;
        return nullptr;
    }
    guarded_exit([&] {
        dl::Context &ctx = compat_context();
        dl::DevBuf offs;
        ctx.reserve(offs, (u64) relation_size * 8);
        const u64 total = dl::sorted_join_count(ctx, (const u64 *) sorted_relation, (u64) sorted_relation_size,
                                                (const u64 *) relation, (u64) relation_size, offs.as<u64>());
        to_int_result(ctx, total, join_result_size);
        if (total) {
            void *p = nullptr;
            if (cudaMalloc(&p, total * 8) != cudaSuccess) die((int) DL_ERR_OUT_OF_MEMORY, "cudaMalloc of the join result failed");
            dl::sorted_join_emit(ctx, (const u64 *) sorted_relation, (u64) sorted_relation_size, (const u64 *) relation,
                                 (u64) relation_size, offs.as<u64>(), total, (u64 *) p);
            ctx.sync();
            result = (dl_entity *) p;
        }
        ctx.give_back(offs);
        return 0;
    });
    *compute_time = now() - t0;
    return result;
}

}  // extern "C"
