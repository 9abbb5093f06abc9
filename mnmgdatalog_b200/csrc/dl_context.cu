// Context: device, stream, control block, grow-only scratch.
#include <chrono>

#include "dl_internal.h"

namespace dl {

namespace {
double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

void DevBuf::reserve(size_t bytes, bool zero) {
    if (bytes <= cap && p) return;
    if (fixed)
        throw Error(DL_ERR_INTERNAL, "a fixed scratch slice of " + std::to_string(cap) + " bytes cannot hold " +
                                         std::to_string(bytes) + " bytes");
    size_t want = bytes + bytes / 8 + 256;
    release();
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        cap = 0;
        (void) cudaGetLastError();
        throw Error(DL_ERR_OUT_OF_MEMORY, "cudaMalloc of " + std::to_string(want) + " bytes failed: " +
                                              cudaGetErrorString(e));
    }
    cap = want;
    if (zero) DL_CUDA(cudaMemset(p, 0, want));
}

void DevBuf::release() {
    if (fixed) return;  // not ours to free
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

void Context::reserve(DevBuf &buf, size_t bytes, bool zero) {
    if (buf.fixed) {  // a fixed slice: it fits or the request is an error
        buf.reserve(bytes);
        if (zero) DL_CUDA(cudaMemsetAsync(buf.p, 0, buf.cap, stream));
        return;
    }
    if (buf.p && buf.cap >= bytes) return;
    // A buffer that outgrows itself grows by half at least, so a relation that
    // grows every iteration is reallocated O(log) times, not at every step.
    const size_t want = buf.p ? std::max(bytes, buf.cap + buf.cap / 2) : bytes;
    // Best fit among the cached buffers, but never one far larger than the
    // request: a small result must not pin a large buffer that a growing
    // relation will need next.
    const size_t limit = std::max<size_t>(4 * bytes, bytes + (size_t(64) << 20));
    int best = -1;
    for (int i = 0; i < (int) spares.size(); ++i)
        if (spares[i].cap >= bytes && spares[i].cap <= limit && (best < 0 || spares[i].cap < spares[best].cap))
            best = i;
    if (best >= 0) {
        if (buf.p) spares.push_back(buf);
        buf = spares[best];
        spares.erase(spares.begin() + best);
        trim_spares();
        if (zero) DL_CUDA(cudaMemsetAsync(buf.p, 0, buf.cap, stream));
        return;
    }
    if (buf.p) {
        // Keep the old allocation for smaller requests later.
        spares.push_back(buf);
        buf = DevBuf();
        trim_spares();
    }
    allocate(buf, want, zero, bytes);
}

void Context::allocate(DevBuf &buf, size_t bytes, bool zero, size_t minimum) {
    if (no_alloc)
        throw Error(DL_ERR_INTERNAL, "a context without allocation was asked for a new buffer of " +
                                         std::to_string(bytes) + " bytes");
    const double t0 = now_s();
    try {
        buf.reserve(bytes, zero);
    } catch (const Error &) {
        // Out of memory: drop every cached buffer and retry once.
        for (auto &s : spares) s.release();
        spares.clear();
        buf.reserve(minimum ? minimum : bytes, zero);
    }
    KernelStat &k = kstat[K_HOST_MALLOC];
    k.launches++;
    k.timed++;
    k.seconds += now_s() - t0;
    k.bytes += (double) buf.cap;
}

void Context::trim_spares() {
    // Cache at most kSpareCount buffers and tune.cache_max_gib in total, freeing the
    // smallest first (large buffers are the expensive ones to re-create).
    size_t total = 0;
    for (const auto &s : spares) total += s.cap;
    const size_t limit = (size_t) tune.cache_max_gib << 30;
    while (!spares.empty() && (spares.size() > kSpareCount || total > limit)) {
        int small = 0;
        for (int i = 1; i < (int) spares.size(); ++i)
            if (spares[i].cap < spares[small].cap) small = i;
        total -= spares[small].cap;
        const double t0 = now_s();
        kstat[K_HOST_FREE].bytes += (double) spares[small].cap;
        spares[small].release();
        kstat[K_HOST_FREE].seconds += now_s() - t0;
        kstat[K_HOST_FREE].launches++;
        kstat[K_HOST_FREE].timed++;
        spares.erase(spares.begin() + small);
    }
}

void Context::give_back(DevBuf &buf) {
    if (!buf.p || buf.fixed) return;
    spares.push_back(buf);
    buf = DevBuf();
    trim_spares();
}

cudaStream_t Context::copy_stream_get() {
    if (!copy_stream) DL_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
    return copy_stream;
}

void Context::release_all() {
    prof_resolve();
    for (auto e : ev_pool) cudaEventDestroy(e);
    ev_pool.clear();
    if (copy_stream) {
        cudaStreamSynchronize(copy_stream);
        cudaStreamDestroy(copy_stream);
        copy_stream = nullptr;
    }
    for (auto &s : spares) s.release();
    spares.clear();
    DevBuf *all[] = {&ws.input, &ws.ids, &ws.w0, &ws.w1, &ws.csr_off, &ws.csr_val, &ws.full[0], &ws.full[1],
                     &ws.small[0], &ws.small[1], &ws.tiny[0], &ws.tiny[1], &ws.sample, &ws.sample_small,
                     &ws.jbuf[0], &ws.jbuf[1], &ws.offsets, &ws.wcc_label, &ws.wcc_flag, &ws.wcc_next,
                     &ws.bitmat[0], &ws.bitmat[1], &ws.offsets_next, &ws.bit_hasout,
                     &lookback, &sort_hist, &lbs_splits, &radix_part, &merge_splits, &bucket_cursor,
                     &part_cursor};
    for (DevBuf *b : all) b->release();
}

u32 Context::next_epoch() {
    if (epoch >= kEpochMask) {
        // Wrap: clear every word so none can carry a recycled epoch.
        if (lookback.p) DL_CUDA(cudaMemsetAsync(lookback.p, 0, lookback.cap, stream));
        epoch = 0;
    }
    return ++epoch;
}

u64 *Context::lookback_words(size_t words) {
    if (words * sizeof(u64) > lookback.cap) {
        sync();
        lookback.reserve(words * sizeof(u64), true);
    }
    return lookback.as<u64>();
}

u32 *Context::tile_counter(int slot) { return &ctrl->tile_counter[slot]; }

void Context::check_device_error() {
    u32 err = reinterpret_cast<volatile u32 *>(host_scalars)[2 * 63];
    if (err) {
        DL_CUDA(cudaMemsetAsync(&ctrl->err, 0, sizeof(u32), stream));
        DL_CUDA(cudaStreamSynchronize(stream));
        reinterpret_cast<volatile u32 *>(host_scalars)[2 * 63] = 0;
        if (err & DL_DEVERR_HASH_FULL) throw Error(DL_ERR_INTERNAL, "hash set probe sequence exceeded its capacity");
        if (err & DL_DEVERR_CAPACITY) throw Error(DL_ERR_OVERFLOW, "a device buffer was smaller than its contents");
        if (err & DL_DEVERR_LOOKBACK)
            throw Error(DL_ERR_DEVICE_TIMEOUT, "a device-side wait exceeded its limit (decoupled look-back)");
        throw Error(DL_ERR_INTERNAL, "device error flag " + std::to_string(err));
    }
}

const char *kernel_name(int kid) {
    static const char *names[K_COUNT] = {"prep", "sort_histogram", "sort_spine_scan", "sort_scatter_pass",
                                         "select_compact", "join_count_scan", "join_partition", "join_emit",
                                         "wcc_propagate", "merge_partition", "diff_merge", "merge", "hash_build",
                                         "sparse_diff", "hash_insert", "bitmap_expand", "bitmap_columns", "bitmap_extract", "host_cudaMalloc", "host_cudaFree",
                                         "host_sync"};
    return (kid >= 0 && kid < K_COUNT) ? names[kid] : "?";
}

void Context::prof_begin() {
    if (!prof_on) return;
    cudaEvent_t e;
    if (ev_pool.empty()) {
        DL_CUDA(cudaEventCreate(&e));
    } else {
        e = ev_pool.back();
        ev_pool.pop_back();
    }
    DL_CUDA(cudaEventRecord(e, stream));
    prof_open = e;
}

void Context::prof_end(int kid, double bytes) {
    kstat[kid].launches++;
    if (!prof_on || !prof_open) return;
    cudaEvent_t e;
    if (ev_pool.empty()) {
        DL_CUDA(cudaEventCreate(&e));
    } else {
        e = ev_pool.back();
        ev_pool.pop_back();
    }
    DL_CUDA(cudaEventRecord(e, stream));
    pending.push_back({kid, prof_open, e, bytes});
    prof_open = nullptr;
}

void Context::prof_add_bytes(int kid, double bytes) {
    if (prof_on) kstat[kid].bytes += bytes;
}

void Context::prof_resolve() {
    for (auto &p : pending) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            kstat[p.kid].seconds += ms * 1e-3;
            kstat[p.kid].timed++;
            kstat[p.kid].bytes += p.bytes;
        }
        ev_pool.push_back(p.a);
        ev_pool.push_back(p.b);
    }
    pending.clear();
}

void Context::prof_reset() {
    prof_resolve();
    for (auto &k : kstat) k = KernelStat();
}

void Context::sync() {
    DL_CUDA(cudaMemcpyAsync(reinterpret_cast<u32 *>(host_scalars) + 2 * 63, &ctrl->err, sizeof(u32),
                            cudaMemcpyDeviceToHost, stream));
    const double t0 = now_s();
    DL_CUDA(cudaStreamSynchronize(stream));
    KernelStat &k = kstat[K_HOST_SYNC];
    k.launches++;
    k.timed++;
    k.seconds += now_s() - t0;
    if (!pending.empty()) prof_resolve();
    check_device_error();
}

}  // namespace dl
