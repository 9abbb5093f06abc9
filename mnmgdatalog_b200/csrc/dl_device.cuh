// Device-side building blocks shared by every kernel of the engine.
//
// * Tuple words: a relation is an array of 64-bit words whose unsigned order
//   is the reference's set_cmp order (common/utils.cu:114-124). Inside a
//   program run the engine uses *compact* words (key_index << B) | value_index
//   over dense node indices; at the C-ABI the reference's Entity layout
//   {int key; int value;} is converted by `entity_encode` / `entity_decode`.
// * Decoupled look-back: single-pass prefix sums publish one 64-bit word per
//   tile: [63:62] status, [61:48] epoch, [47:0] value. A word whose epoch is
//   not the launch's epoch reads as "not yet published", so the look-back
//   buffer never needs clearing between launches. Every wait is bounded: after
//   kSpinLimit polls the kernel records DL_DEVERR_LOOKBACK in the context's
//   error word and carries on (the host turns that into DL_ERR_DEVICE_TIMEOUT).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dl {

using u32 = uint32_t;
using u64 = uint64_t;
using i64 = int64_t;

constexpr u64 kStatusAgg = 1ull << 62;
constexpr u64 kStatusInc = 2ull << 62;
constexpr u64 kLbValueMask = (1ull << 48) - 1;
constexpr u32 kEpochMask = 0x3FFF;
constexpr u32 kSpinLimit = 1u << 22;

// Device error bits (ctrl->err).
constexpr u32 DL_DEVERR_LOOKBACK = 1u;
constexpr u32 DL_DEVERR_CAPACITY = 2u;
constexpr u32 DL_DEVERR_HASH_FULL = 4u;

// Control block resident in device memory, one per context.
struct Ctrl {
    u32 err;
    u32 pad0;
    u32 tile_counter[64];
    u64 scalar[64];
};

__host__ __device__ __forceinline__ u64 entity_encode(u64 raw) {
    // Entity {key, value} read as little-endian u64 is (value << 32) | key.
    // Rotate so the key is the high half and bias both halves by 2^31.
    return ((raw << 32) | (raw >> 32)) ^ 0x8000000080000000ull;
}
__host__ __device__ __forceinline__ u64 entity_decode(u64 w) {
    w ^= 0x8000000080000000ull;
    return (w << 32) | (w >> 32);
}

__device__ __forceinline__ u64 lb_word(u64 status, u32 epoch, u64 v) {
    return status | ((u64) (epoch & kEpochMask) << 48) | (v & kLbValueMask);
}

__device__ __forceinline__ void st_relaxed_u64(u64 *p, u64 v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ u64 ld_relaxed_u64(const u64 *p) {
    u64 v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ u32 lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ u32 lanemask_lt() {
    u32 m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename T>
__device__ __forceinline__ T warp_inclusive_sum(T x) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if ((int) lane_id() >= o) x += y;
    }
    return x;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Block-wide exclusive sum of one value per thread. `scratch` holds
// NWARPS+1 entries; returns the exclusive prefix and sets *total.
template <int NWARPS, typename T>
__device__ __forceinline__ T block_exclusive_sum(T x, T *scratch, T *total) {
    const int w = threadIdx.x >> 5;
    T inc = warp_inclusive_sum(x);
    if (lane_id() == 31) scratch[w] = inc;
    __syncthreads();
    if (w == 0) {
        T v = (lane_id() < NWARPS) ? scratch[lane_id()] : T(0);
        T vi = warp_inclusive_sum(v);
        if (lane_id() < NWARPS) scratch[lane_id()] = vi - v;
        if (lane_id() == NWARPS - 1) scratch[NWARPS] = vi;
    }
    __syncthreads();
    T r = scratch[w] + inc - x;
    *total = scratch[NWARPS];
    __syncthreads();
    return r;
}

// Warp-cooperative decoupled look-back for tile `tile` (> 0): returns the sum
// of all predecessor tiles' values. Must be called by all 32 lanes of ONE warp.
__device__ __forceinline__ u64 lookback_warp(const u64 *lb, u32 tile, u32 epoch, u32 *err) {
    u64 excl = 0;
    long long base = (long long) tile - 1;
    u32 spins = 0;
    const u32 lane = lane_id();
    while (true) {
        long long t = base - (long long) lane;
        u64 w = (t >= 0) ? ld_relaxed_u64(lb + t) : (kStatusInc | ((u64) (epoch & kEpochMask) << 48));
        u32 st = (u32) (w >> 62);
        if (((u32) (w >> 48) & kEpochMask) != (epoch & kEpochMask)) st = 0;
        u32 inc_mask = __ballot_sync(0xffffffffu, st == 2);
        u32 bad_mask = __ballot_sync(0xffffffffu, st == 0);
        int first_inc = inc_mask ? (__ffs(inc_mask) - 1) : 32;
        u32 relevant = (first_inc >= 31) ? 0xffffffffu : ((2u << first_inc) - 1u);
        if (bad_mask & relevant) {
            if (++spins > kSpinLimit) {
                if (lane == 0) atomicOr(err, DL_DEVERR_LOOKBACK);
                return excl;
            }
            if (spins > 64) __nanosleep(64);
            continue;
        }
        u64 v = ((int) lane <= first_inc) ? (w & kLbValueMask) : 0ull;
        excl += warp_sum(v);
        if (first_inc < 32) return excl;
        base -= 32;
    }
}

// Block-wide decoupled look-back: every thread reads one predecessor's word,
// so one round covers NWARPS*32 tiles -- more than the tiles resident on the
// GPU at a time -- and a tile typically finds an inclusive prefix in one L2
// round trip (a warp-wide window lags the inclusive frontier by many rounds
// when tiles are short). All threads of the block must call it.
struct LookbackScratch {
    u32 first_inc;
    u32 bad;
    u64 part[32];
};

template <int NWARPS>
__device__ __forceinline__ u64 lookback_block(const u64 *lb, u32 tile, u32 epoch, u32 *err, LookbackScratch &sc) {
    constexpr int NT = NWARPS * 32;
    const int tid = threadIdx.x;
    u64 excl = 0;
    long long base = (long long) tile - 1;
    u32 spins = 0;
    while (true) {
        const long long t = base - tid;
        const u64 w = (t >= 0) ? ld_relaxed_u64(lb + t) : (kStatusInc | ((u64) (epoch & kEpochMask) << 48));
        u32 st = (u32) (w >> 62);
        if (((u32) (w >> 48) & kEpochMask) != (epoch & kEpochMask)) st = 0;
        if (tid == 0) {
            sc.first_inc = NT;
            sc.bad = 0;
        }
        __syncthreads();
        if (st == 2) atomicMin(&sc.first_inc, (u32) tid);
        __syncthreads();
        const u32 fi = sc.first_inc;
        if (st == 0 && (u32) tid <= fi) sc.bad = 1;
        __syncthreads();
        if (sc.bad) {
            ++spins;
            if (spins > kSpinLimit) {
                if (tid == 0) atomicOr(err, DL_DEVERR_LOOKBACK);
                __syncthreads();
                return excl;
            }
            if (spins > 64) __nanosleep(64);
            __syncthreads();  // every thread has read sc.bad before it is reset
            continue;
        }
        u64 v = ((u32) tid <= fi) ? (w & kLbValueMask) : 0ull;
        v = warp_sum(v);
        if (lane_id() == 0) sc.part[tid >> 5] = v;
        __syncthreads();
        u64 sum = 0;
#pragma unroll
        for (int i = 0; i < NWARPS; ++i) sum += sc.part[i];
        excl += sum;
        __syncthreads();  // part[] and first_inc read before the next round
        if (fi < (u32) NT) return excl;
        base -= NT;
    }
}

// Look-back of one counter column (used per radix digit): the word of tile t
// lives at lb[t * stride]. Reads a window of 8 predecessors per round.
__device__ __forceinline__ u64 lookback_serial(const u64 *lb, u32 tile, u32 stride, u32 epoch, u32 *err) {
    constexpr int WIN = 8;
    u64 excl = 0;
    long long t = (long long) tile - 1;
    u32 spins = 0;
    while (t >= 0) {
        u64 w[WIN];
#pragma unroll
        for (int i = 0; i < WIN; ++i) w[i] = (t - i >= 0) ? ld_relaxed_u64(lb + (u64) (t - i) * stride) : 0ull;
        int consumed = 0;
        bool done = false, stall = false;
#pragma unroll
        for (int i = 0; i < WIN; ++i) {
            if (done || stall || t - i < 0) continue;
            u32 st = (u32) (w[i] >> 62);
            if (((u32) (w[i] >> 48) & kEpochMask) != (epoch & kEpochMask)) st = 0;
            if (st == 0) {
                stall = true;
                continue;
            }
            excl += w[i] & kLbValueMask;
            ++consumed;
            if (st == 2) done = true;
        }
        if (done) return excl;
        t -= consumed;
        if (stall) {
            if (++spins > kSpinLimit) {
                atomicOr(err, DL_DEVERR_LOOKBACK);
                return excl;
            }
            if (spins > 32) __nanosleep(32);
        }
    }
    return excl;
}

// ---- TMA bulk copies (cp.async.bulk) with mbarrier completion ---------------
__device__ __forceinline__ u32 smem_u32(const void *p) { return (u32) __cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(u64 *bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Arrive once and expect `bytes` of transaction on the barrier.
__device__ __forceinline__ void mbar_expect_tx(u64 *bar, u32 bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_complete_tx(u64 *bar, u32 bytes) {
    asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// 1D bulk copy global -> shared; dst, src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void tma_load_1d(void *dst, const void *src, u32 bytes, u64 *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(u64 *bar, u32 phase) {
    u32 ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// Bounded wait for a barrier phase; returns false (and flags `err`) on timeout.
__device__ __forceinline__ bool mbar_wait(u64 *bar, u32 phase, u32 *err) {
    u32 spins = 0;
    while (!mbar_try_wait(bar, phase)) {
        if (++spins > kSpinLimit) {
            atomicOr(err, DL_DEVERR_LOOKBACK);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ u32 fmix32(u32 k) {
    // MurmurHash3 finalizer; same mixing as the reference's get_position
    // (common/utils.cu:149-156).
    k ^= k >> 16;
    k *= 0x85ebca6bu;
    k ^= k >> 13;
    k *= 0xc2b2ae35u;
    k ^= k >> 16;
    return k;
}

}  // namespace dl
