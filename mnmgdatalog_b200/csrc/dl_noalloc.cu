// dl_sort_unique_noalloc: sort + deduplicate without allocating any memory.
//
// Some callers of this library cannot call cudaMalloc when they sort: a host
// process whose device memory is already owned by another allocator's pool
// (a framework's caching allocator that reserved nearly all of the GPU), a
// service that must keep a fixed device footprint after start-up, or code
// that must not pay the implicit device synchronisation a cudaMalloc/cudaFree
// can cause in the middle of other work. For them this entry point runs the
// same radix sort and unique kernels as dl_sort_unique, with every scratch
// buffer carved out of one file-scope device array of fixed size.
//
// * The array below exists once per GPU that loads the library and stays
//   there until the process exits.
// * In host code `g_sort_unique_scratch` is only a host-side stand-in for the
//   symbol: its real device address is fetched with cudaGetSymbolAddress, once
//   per device, the first time the entry point runs on that device (with that
//   device current). That first call should therefore happen before any
//   stream capture begins.
// * Every call shares the array and it keeps the previous call's contents.
//   The first call on a device clears the control words and the look-back
//   words on the call's stream; after that the look-back words carry an epoch
//   so that old contents can never be taken for new ones, and the sort clears
//   its own counters. Calls whose GPU work overlaps would race on the array:
//   host calls are serialised by a lock and each call waits on its stream for
//   its own GPU work before it returns.
// * Every slice of the array is marked fixed and the context forbids new
//   buffers: should a future change make the sort ask for more scratch than
//   a slice holds, the call fails with DL_ERR_INTERNAL instead of allocating.
#include <cstring>
#include <mutex>
#include <new>
#include <stdexcept>

#include "dl_internal.h"

namespace {

using dl::u64;

constexpr u64 kNoAllocMaxRows = 1ull << 20;  // 1,048,576 rows (8 MiB of input)
constexpr size_t kTmpBytes = kNoAllocMaxRows * 8;                 // sort ping-pong buffer
constexpr size_t kPartBytes = 2ull * 256 * 256 * 8;                // per-(digit, CTA) counts and offsets
constexpr size_t kHistBytes = 2ull * 8 * 256 * 8;                  // histogram + bucket bases
constexpr size_t kLookbackBytes = 65536ull * 8;                    // look-back words
constexpr size_t kCtrlBytes = 4096;                                // control block (>= sizeof(Ctrl))
constexpr size_t kScratchBytes = kTmpBytes + kPartBytes + kHistBytes + kLookbackBytes + kCtrlBytes;
static_assert(sizeof(dl::Ctrl) <= kCtrlBytes, "control block does not fit");
// The radix sort of at most kNoAllocMaxRows keys uses at most 256 CTAs per
// pass (a 4,096-key tile each) with 256 digits, and its look-back needs one
// word per (tile, digit) of a onesweep pass: both fit their slices. A change
// that breaks this is caught at run time (fixed slices, no_alloc context).
static_assert(kPartBytes >= 2ull * 256 * ((kNoAllocMaxRows + 4095) / 4096) * 8, "radix_part slice too small");

}  // namespace

static __device__ __align__(256) unsigned char g_sort_unique_scratch[kScratchBytes];

namespace {

struct NoAllocDevice {
    bool ready = false;
    dl::Context ctx;
    u64 *tmp = nullptr;
    u64 host_words[64] = {};
};

std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc[64];

dl_status noalloc_fail(dl_status s, const std::string &m) {
    dl::set_last_error(m);  // reported by dl_last_error()
    return s;
}

// Once per device: find the array's device address and point every scratch
// buffer of a context at a slice of it.
dl_status noalloc_setup(int device, NoAllocDevice &d, cudaStream_t stream) {
    void *base = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&base, g_sort_unique_scratch);
    if (e != cudaSuccess) {
        (void) cudaGetLastError();
        return noalloc_fail(DL_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    }
    char *p = static_cast<char *>(base);
    dl::Context &c = d.ctx;
    c.device = device;
    cudaDeviceGetAttribute(&c.sm_count, cudaDevAttrMultiProcessorCount, device);
    d.tmp = reinterpret_cast<u64 *>(p);
    p += kTmpBytes;
    c.radix_part.p = p;
    c.radix_part.cap = kPartBytes;
    c.radix_part.fixed = true;
    p += kPartBytes;
    c.sort_hist.p = p;
    c.sort_hist.cap = kHistBytes;
    c.sort_hist.fixed = true;
    p += kHistBytes;
    c.lookback.p = p;
    c.lookback.cap = kLookbackBytes;
    c.lookback.fixed = true;
    p += kLookbackBytes;
    c.ctrl = reinterpret_cast<dl::Ctrl *>(p);
    c.host_scalars = d.host_words;  // pageable host words: copies into them need no allocation
    c.epoch = 0;
    c.no_alloc = true;
    e = cudaMemsetAsync(c.ctrl, 0, kCtrlBytes, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.lookback.p, 0, kLookbackBytes, stream);
    if (e != cudaSuccess) {
        (void) cudaGetLastError();
        return noalloc_fail(DL_ERR_CUDA, std::string("clearing the scratch array: ") + cudaGetErrorString(e));
    }
    d.ready = true;
    return DL_OK;
}

}  // namespace

extern "C" {

DL_API int64_t dl_sort_unique_noalloc_max_rows(void) { return (int64_t) kNoAllocMaxRows; }

DL_API dl_status dl_sort_unique_noalloc(dl_entity *rel, int64_t n, int64_t *n_out, void *stream) {
    // Every failure becomes a status code; nothing may leave this C function
    // as an exception.
    try {
        if (!n_out || n < 0 || (n > 0 && !rel)) return noalloc_fail(DL_ERR_INVALID_ARGUMENT, "invalid argument");
        if ((u64) n > kNoAllocMaxRows)
            return noalloc_fail(DL_ERR_INVALID_ARGUMENT, "dl_sort_unique_noalloc takes at most " +
                                                             std::to_string(kNoAllocMaxRows) + " rows, got " +
                                                             std::to_string(n));
        *n_out = 0;
        if (n == 0) return DL_OK;
        int device = 0;
        if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) {
            (void) cudaGetLastError();
            return noalloc_fail(DL_ERR_NO_DEVICE, "no current CUDA device");
        }
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        NoAllocDevice &d = g_noalloc[device];
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (!d.ready) {
            const dl_status st = noalloc_setup(device, d, s);
            if (st != DL_OK) return st;
        }
        d.ctx.stream = s;
        u64 *sorted = dl::radix_sort(d.ctx, reinterpret_cast<u64 *>(rel), d.tmp, (u64) n, dl::Codec::Entity, 0);
        *n_out = (int64_t) dl::unique_words(d.ctx, sorted, (u64) n, reinterpret_cast<u64 *>(rel));
        return DL_OK;
    } catch (const dl::Error &err) {
        return noalloc_fail(err.status, err.what());
    } catch (const std::bad_alloc &) {
        return noalloc_fail(DL_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception &err) {
        return noalloc_fail(DL_ERR_INTERNAL, err.what());
    }
}

}  // extern "C"
