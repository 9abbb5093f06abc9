// Joins: count pass + load-balanced emit pass.
//
// The reference (common/join.cu:1-87) walks the probe chain once to count,
// reduces and scans on the host side, cudaMallocs, then walks again to write,
// one thread per probe tuple, so a hub key with a million matches runs on one
// thread. Here:
//   1. count: single-pass scan kernel, offsets[i] = sum of match counts of
//      probe rows < i (64-bit), total to device memory;
//   2. emit: the output positions [0, T) and the probe rows are merged by
//      their offsets (merge path); every CTA takes JN_TILE merged slots, so work
//      per CTA is bounded whatever the skew. Consecutive threads write
//      consecutive output words (coalesced) and read consecutive matches.
// The index looked up per probe row is pluggable:
//   * CsrSrc   -- the engine's relation over dense node indices: a direct
//                 offset table, one 8-byte lookup per probe row;
//   * HashSrc  -- the C-ABI hash table (dl_build_hash_table): linear probing
//                 of 16-byte slots {key, begin, count, -} read with one
//                 128-bit load each, murmur3-finalizer start slot;
//   * SortedSrc-- binary search of a key-sorted relation (get_join_nl,
//                 common/join.cu:89-180).
// HBM traffic of the emit: 8 B per output word written + 8 B per probe row
// read; the indexed relation (a few MB at the configs) stays in L2.
#include "dl_internal.h"
#include "dl_join.cuh"
#include "dl_scan.cuh"

namespace dl {

// ---- engine joins over the CSR of dense node indices -------------------------

u64 join_count(Context &ctx, const Csr &csr, const u64 *probe, u64 n_probe, int bits, u64 *offsets) {
    return count_matches(ctx, CsrSrc<EmitKind::ZV>{csr.off, csr.val, probe, bits}, n_probe, offsets);
}

void join_emit(Context &ctx, const Csr &csr, const u64 *probe, u64 n_probe, int bits, const u64 *offsets, u64 total,
               EmitKind kind, u64 *out, u64 *hist, int hist_digits, u64 *self_pairs) {
    switch (kind) {
        case EmitKind::ZV:
            emit_matches(ctx, CsrSrc<EmitKind::ZV>{csr.off, csr.val, probe, bits}, n_probe, offsets, total, out, hist,
                         hist_digits, self_pairs);
            break;
        case EmitKind::VZ:
            emit_matches(ctx, CsrSrc<EmitKind::VZ>{csr.off, csr.val, probe, bits}, n_probe, offsets, total, out, hist,
                         hist_digits, self_pairs);
            break;
        case EmitKind::ZV_NOSELF:
            emit_matches(ctx, CsrSrc<EmitKind::ZV_NOSELF>{csr.off, csr.val, probe, bits}, n_probe, offsets, total, out,
                         hist, hist_digits, self_pairs);
            break;
    }
}

void join_emit_bucketed(Context &ctx, const Csr &csr, const u64 *probe, u64 n_probe, int bits, const u64 *offsets,
                        u64 total, u64 *out) {
    if (total == 0) return;
    if (bits < 8) throw Error(DL_ERR_INTERNAL, "bucketed emit needs 8 payload bits");
    const CsrSrc<EmitKind::ZV> src{csr.off, csr.val, probe, bits};
    ctx.reserve(ctx.bucket_cursor, 256 * sizeof(u64));
    auto *cur = ctx.bucket_cursor.as<unsigned long long>();
    DL_CUDA(cudaMemsetAsync(cur, 0, 256 * sizeof(u64), ctx.stream));
    const unsigned hg = (unsigned) std::max<u64>(1, std::min<u64>((n_probe + 255) / 256, (u64) ctx.sm_count * 8));
    DL_LAUNCH(ctx, K_JOIN_COUNT, 8.0 * n_probe,
              digit0_hist_kernel<CsrSrc<EmitKind::ZV>><<<hg, 256, 0, ctx.stream>>>(src, probe, n_probe, cur));
    DL_LAUNCH(ctx, K_JOIN_PARTITION, 0, bucket_starts_kernel<<<1, 256, 0, ctx.stream>>>(cur));
    const u64 tiles = (n_probe + total + JN_TILE - 1) / JN_TILE;
    ctx.lbs_splits.reserve((tiles + 1) * sizeof(u64));
    u64 *splits = ctx.lbs_splits.as<u64>();
    DL_LAUNCH(ctx, K_JOIN_PARTITION, 0,
              lbs_partition_kernel<<<(unsigned) ((tiles + 1 + 255) / 256), 256, 0, ctx.stream>>>(offsets, n_probe, total,
                                                                                                 tiles + 1, splits));
    auto kern = join_emit_bucket_kernel<CsrSrc<EmitKind::ZV>>;
    DL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sizeof(JoinBucketSmem)));
    DL_LAUNCH(ctx, K_JOIN_EMIT, CsrSrc<EmitKind::ZV>::prof_bytes(n_probe, total),
              kern<<<(unsigned) tiles, JN_THREADS, sizeof(JoinBucketSmem), ctx.stream>>>(src, n_probe, offsets, total,
                                                                                          splits, out, cur,
                                                                                          &ctx.ctrl->err));
}

// ---- C-ABI hash table ------------------------------------------------------

namespace {

// One slot per distinct key of the sorted relation: rows [i, i + count) of
// the sorted relation carry key `key`.
__global__ void hash_insert_kernel(const u64 *__restrict__ sorted, u64 n, HashSlot *__restrict__ slots, u64 mask,
                                   u32 *err) {
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u32 key = (u32) sorted[i];
        if (i > 0 && (u32) sorted[i - 1] == key) continue;
        // end of the run: first row with a larger key (binary search)
        u64 lo = i + 1, hi = n;
        while (lo < hi) {
            const u64 mid = (lo + hi) >> 1;
            if ((u32) sorted[mid] == key) lo = mid + 1;
            else hi = mid;
        }
        const u32 count = (u32) (lo - i);
        u64 h = fmix32(key) & mask;
        for (u64 probe = 0; probe <= mask; ++probe) {
            if (atomicCAS(&slots[h].count, 0u, count) == 0u) {
                slots[h].key = (int) key;
                slots[h].begin = (u32) i;
                break;
            }
            h = (h + 1) & mask;
        }
    }
}

__global__ void extract_values_kernel(const u64 *__restrict__ sorted, u64 n, u32 *__restrict__ vals) {
    const u64 stride = (u64) gridDim.x * blockDim.x;
    for (u64 i = (u64) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) vals[i] = (u32) (sorted[i] >> 32);
}

}  // namespace

HashTable *hash_table_build(Context &ctx, const u64 *rel, u64 n, double load_factor) {
    if (!(load_factor > 0.0 && load_factor < 1.0)) load_factor = ctx.tune.hash_load;
    if (n > 0xFFFFFFFFull) throw Error(DL_ERR_OVERFLOW, "hash table relation exceeds 2^32 rows");
    auto *ht = new HashTable();
    ht->rows = n;
    if (n == 0) return ht;
    DevBuf a, b;
    try {
        a.reserve(n * sizeof(u64));
        b.reserve(n * sizeof(u64));
        DL_CUDA(cudaMemcpyAsync(a.p, rel, n * sizeof(u64), cudaMemcpyDeviceToDevice, ctx.stream));
        u64 *sorted = radix_sort(ctx, a.as<u64>(), b.as<u64>(), n, Codec::Entity, 0);
        u64 *other = sorted == a.as<u64>() ? b.as<u64>() : a.as<u64>();
        const u64 distinct = unique_words(ctx, sorted, n, other, 0, Codec::Entity);
        ht->distinct = distinct;
        u64 slots = 1;
        while ((double) slots * load_factor < (double) distinct) slots <<= 1;
        ht->slots = slots;
        ht->table.reserve(slots * sizeof(HashSlot), true);
        ht->vals.reserve(n * sizeof(u32));
        const unsigned grid = (unsigned) std::min<u64>((n + 255) / 256, (u64) ctx.sm_count * 16);
        DL_LAUNCH(ctx, K_HASH_BUILD, 8.0 * n, hash_insert_kernel<<<grid, 256, 0, ctx.stream>>>(sorted, n, ht->table.as<HashSlot>(), slots - 1,
                                                         &ctx.ctrl->err));
        DL_LAUNCH(ctx, K_HASH_BUILD, 8.0 * n, extract_values_kernel<<<grid, 256, 0, ctx.stream>>>(sorted, n, ht->vals.as<u32>()));
        ctx.sync();
    } catch (...) {
        a.release();
        b.release();
        delete ht;
        throw;
    }
    a.release();
    b.release();
    return ht;
}

u64 hash_join_count(Context &ctx, const HashTable &ht, const u64 *probe, u64 n, u64 *offsets) {
    if (ht.distinct == 0) {
        if (n) DL_CUDA(cudaMemsetAsync(offsets, 0, n * sizeof(u64), ctx.stream));
        return 0;
    }
    return count_matches(ctx, HashSrc{ht.table.as<HashSlot>(), ht.vals.as<u32>(), ht.slots - 1, probe}, n, offsets);
}

void hash_join_emit(Context &ctx, const HashTable &ht, const u64 *probe, u64 n, const u64 *offsets, u64 total,
                    u64 *out) {
    emit_matches(ctx, HashSrc{ht.table.as<HashSlot>(), ht.vals.as<u32>(), ht.slots - 1, probe}, n, offsets, total, out,
                 nullptr, 0, nullptr);
}

u64 sorted_join_count(Context &ctx, const u64 *rel, u64 n_rel, const u64 *probe, u64 n, u64 *offsets) {
    return count_matches(ctx, SortedSrc{rel, n_rel, probe}, n, offsets);
}

void sorted_join_emit(Context &ctx, const u64 *rel, u64 n_rel, const u64 *probe, u64 n, const u64 *offsets, u64 total,
                      u64 *out) {
    emit_matches(ctx, SortedSrc{rel, n_rel, probe}, n, offsets, total, out, nullptr, 0, nullptr);
}

}  // namespace dl
