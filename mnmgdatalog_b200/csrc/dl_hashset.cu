// Hash set of tuple words: the full relation of the TC fixpoint when the
// join output is deduplicated by hashing instead of sorting.
//
// The reference keeps full sorted and re-merges it with every delta
// (tc.cu:250-286). The sorted order is only needed for the program's output;
// the fixpoint itself needs set semantics: delta' = dedup(J) \ full and
// full' = full u delta'. Here full is an open-addressing table of 64-bit
// words; inserting every join-output word with one compare-and-swap yields
// exactly the words new to full (the first insert of a duplicate wins, the
// others see it), which are appended to the next delta. One radix sort of
// the table's words at the end gives the reference's sorted output.
#include "dl_internal.h"

namespace dl {
namespace {

constexpr u64 kEmpty = ~0ull;  // never a tuple word: ranks are below 2^31
constexpr int HS_THREADS = 256;

// splitmix64 finalizer (public-domain mixing function): every key bit
// affects every slot bit, so structured words (rank << B | rank) spread.
__device__ __forceinline__ u64 mix64(u64 z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Returns true when w was not in the table and this thread inserted it.
__device__ __forceinline__ bool insert_word(u64 *__restrict__ slots, u64 mask, u64 w, u32 *err) {
    u64 h = mix64(w) & mask;
    for (u64 probe = 0; probe <= mask; ++probe) {
        const u64 cur = slots[h];
        if (cur == w) return false;
        if (cur == kEmpty) {
            const u64 old = atomicCAS(reinterpret_cast<unsigned long long *>(slots + h), kEmpty, w);
            if (old == kEmpty) return true;
            if (old == w) return false;
        }
        h = (h + 1) & mask;
    }
    atomicOr(err, DL_DEVERR_HASH_FULL);  // cannot happen below half load; reported, not hung
    return false;
}

// Inserts in[0, n); new words are appended to fresh (warp-aggregated).
__global__ void __launch_bounds__(HS_THREADS)
wordset_insert_kernel(u64 *__restrict__ slots, u64 mask, const u64 *__restrict__ in, u64 n, u64 *__restrict__ fresh,
                      unsigned long long *__restrict__ fresh_count, u32 *err) {
    const u64 stride = (u64) gridDim.x * blockDim.x;
    const u32 lane = threadIdx.x & 31;
    // the loop bound is the same for all lanes of a warp: the ballot below sees them all
    for (u64 base = (u64) blockIdx.x * blockDim.x; base < n; base += stride) {
        const u64 i = base + threadIdx.x;
        bool is_new = false;
        u64 w = 0;
        if (i < n) {
            w = __ldcs(in + i);
            is_new = insert_word(slots, mask, w, err);
        }
        const u32 b = __ballot_sync(0xffffffffu, is_new);
        if (b) {  // warp-uniform
            unsigned long long at = 0;
            if (lane == 0) at = atomicAdd(fresh_count, (unsigned long long) __popc(b));
            if (fresh) {
                at = __shfl_sync(0xffffffffu, at, 0);
                if (is_new) fresh[at + __popc(b & ((1u << lane) - 1u))] = w;
            }
        }
    }
}

// Re-inserts every word of an old table (all distinct) into a new one.
__global__ void __launch_bounds__(HS_THREADS)
wordset_rehash_kernel(const u64 *__restrict__ old_slots, u64 old_cap, u64 *__restrict__ slots, u64 mask, u32 *err) {
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < old_cap; i += stride) {
        const u64 w = __ldcs(old_slots + i);
        if (w != kEmpty) insert_word(slots, mask, w, err);
    }
}

unsigned hs_grid(const Context &ctx, u64 n) {
    const u64 want = (n + HS_THREADS - 1) / HS_THREADS;
    const u64 cap = (u64) ctx.sm_count * 8;  // 2048 threads per SM: many probes in flight
    return (unsigned) std::max<u64>(1, std::min(want, cap));
}

}  // namespace

void wordset_reserve(Context &ctx, WordSet &s, DevBuf buf[2], u64 incoming) {
    // at most 3/4 full even if every incoming word is new (join outputs are
    // mostly duplicates, so the load stays well below that)
    const u64 need = (s.size + incoming) / 3 * 4 + 4;
    if (s.cap >= need && s.cap) return;
    u64 cap = 1ull << 16;
    while (cap < need) cap <<= 1;
    DevBuf &nb = buf[1 - s.cur];
    ctx.reserve(nb, cap * 8);
    DL_CUDA(cudaMemsetAsync(nb.p, 0xFF, cap * 8, ctx.stream));
    if (s.size) {
        DL_LAUNCH(ctx, K_HASH_INSERT, 8.0 * s.cap + 40.0 * s.size,
                  wordset_rehash_kernel<<<hs_grid(ctx, s.cap), HS_THREADS, 0, ctx.stream>>>(
                      buf[s.cur].as<u64>(), s.cap, nb.as<u64>(), cap - 1, &ctx.ctrl->err));
    }
    s.cur = 1 - s.cur;
    s.cap = cap;
}

u64 wordset_insert(Context &ctx, WordSet &s, DevBuf buf[2], const u64 *in, u64 n, u64 *fresh) {
    if (n == 0) return 0;
    if ((s.size + n) / 3 * 4 + 4 > s.cap) throw Error(DL_ERR_INTERNAL, "wordset_insert without wordset_reserve");
    u64 *cnt = &ctx.ctrl->scalar[40];
    DL_CUDA(cudaMemsetAsync(cnt, 0, sizeof(u64), ctx.stream));
    DL_LAUNCH(ctx, K_HASH_INSERT, 40.0 * n,
              wordset_insert_kernel<<<hs_grid(ctx, n), HS_THREADS, 0, ctx.stream>>>(
                  buf[s.cur].as<u64>(), s.cap - 1, in, n, fresh, (unsigned long long *) cnt, &ctx.ctrl->err));
    DL_CUDA(cudaMemcpyAsync(ctx.host_scalars + 14, cnt, sizeof(u64), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    const u64 added = ctx.host_scalars[14];
    ctx.prof_add_bytes(K_HASH_INSERT, 40.0 * added);
    s.size += added;
    return added;
}

u64 wordset_extract(Context &ctx, const WordSet &s, DevBuf buf[2], u64 *out) {
    if (s.size == 0) return 0;
    const u64 n = select_words(ctx, buf[s.cur].as<u64>(), s.cap, out, 0);  // drops the empty slots
    if (n != s.size) throw Error(DL_ERR_INTERNAL, "hash set size mismatch");
    return n;
}

}  // namespace dl
