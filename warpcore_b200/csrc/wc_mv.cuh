/*
 * wc_mv.cuh -- MultiValueHashTable kernels (the reference's
 * multi_value_hash_table.cuh: insert :200-289, for_each / num_values
 * :607-663, bulk retrieve :371-520, unique keys gpu_engine.cuh:51-93).
 *
 * Every (key, value) pair takes a slot of its own.  A key's values live
 * along its bucket sequence, up to the first bucket that has a free slot:
 * insert counts them bucket by bucket (stopping at max_values_per_key) and
 * claims the first free slot of that bucket; num_values and retrieve walk
 * the same buckets and take the key's slots in slot order.  Buckets are the
 * table kernels' bucket-aligned windows, so a key's values come out in the
 * order they were inserted, as in the reference.
 *
 * One lane owns one key and reads each bucket with 16-byte vector loads;
 * these tables are not on the headline path and keep the code close to the
 * reference's semantics, one bucket at a time.
 */
#ifndef WC_MV_CUH
#define WC_MV_CUH

#include "wc_kernels.cuh"
#include <warpcore/detail/mv_ops.cuh>

namespace warpcore {
namespace b200 {

/* resident 256-thread blocks per SM the multi-value kernels (multi-value,
 * multi-bucket, bucket-list) are built for: 4 measured best; 6 and 8
 * (42 and 32 registers) ran 0-10 % slower on the mv32 / mb32 / bl32
 * workloads, the register cap costing more than the extra warps bring */
#ifndef WC_MULTI_MIN_BLOCKS
#define WC_MULTI_MIN_BLOCKS 4
#endif

struct MvArgs {
    TableView t;
    const void *keys;
    const void *values;               /* insert */
    void *values_out;                 /* retrieve */
    const unsigned long long *begin;  /* retrieve: begin offsets */
    const unsigned long long *end;    /* retrieve: end offsets (overlap check) */
    unsigned long long *counts_out;   /* num_values: per key, or NULL */
    unsigned long long *total;        /* num_values: sum of the counts */
    unsigned long long *num_keys;     /* insert: keys that got their first value */
    void *status_out;
    uint64_t n;
    uint64_t max_windows;
    uint64_t max_values;
    uint32_t bool_mask;
    int handler;
};

__device__ __forceinline__ void mv_write_status(const MvArgs &a, uint64_t i, uint32_t st)
{
    if (!a.status_out) return;
    if (a.handler == kHandlerStatus)
        reinterpret_cast<uint32_t *>(a.status_out)[i] = st;
    else if (a.handler == kHandlerBoolean)
        reinterpret_cast<unsigned char *>(a.status_out)[i] = (unsigned char)((st & a.bool_mask) != 0);
}

template <class L, int W>
__global__ void __launch_bounds__(256, WC_MULTI_MIN_BLOCKS) mv_insert_kernel(const MvArgs a)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    uint32_t join = 0;
    unsigned long long new_keys = 0;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        bool fresh = false;
        const uint32_t st = mv_insert_one<L, W>(a.t, reinterpret_cast<const K *>(a.keys)[i],
                                                reinterpret_cast<const V *>(a.values)[i],
                                                a.max_windows, a.max_values, fresh);
        /* the reference joins every status but the plain duplicate_key of
         * a successful insert (:266-268) */
        if (st != kStNone && st != kStDuplicateKey) join |= st;
        new_keys += fresh;
        mv_write_status(a, i, st);
    }
    /* every lane of the warp arrives here (no early exits) */
    const unsigned long long nk = __reduce_add_sync(kFull, unsigned(new_keys));
    const uint32_t wj = __reduce_or_sync(kFull, join);
    if ((threadIdx.x & 31) == 0) {
        if (nk) atomicAdd(a.num_keys, nk);
        join_status(a.t.status, wj);
    }
}

/* num_values (values_out == NULL) or retrieve of each key's values */
template <class L, int W, bool kValues>
__global__ void __launch_bounds__(256, WC_MULTI_MIN_BLOCKS) mv_find_kernel(const MvArgs a)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    uint32_t join = 0;
    unsigned long long total = 0;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        uint64_t num = 0;
        if constexpr (kValues) {
            /* The counting pass walked every key to its end and wrote its
             * status; this pass only reads values.  A key counted at 0
             * needs no walk, and a walk ends at the window where the
             * counted values are read (its value limit).  Values are
             * written inside the key's own segment only. */
            const uint64_t room = a.end[i] - a.begin[i];
            if (room == 0) continue;
            V *const out = reinterpret_cast<V *>(a.values_out) + a.begin[i];
            mv_for_each_one<L, W>(a.t, reinterpret_cast<const K *>(a.keys)[i], a.max_windows,
                                  room < a.max_values ? room : a.max_values, num,
                                  [&](V v, uint64_t j) {
                                      if (j < room) out[j] = v;
                                  });
        } else {
            const uint32_t st = mv_for_each_one<L, W>(a.t, reinterpret_cast<const K *>(a.keys)[i],
                                                      a.max_windows, a.max_values, num,
                                                      [](V, uint64_t) {});
            join |= st;
            if (a.counts_out) a.counts_out[i] = num;
            total += num;
            mv_write_status(a, i, st);
        }
    }
    /* every lane of the warp arrives here (no early exits) */
    const uint32_t wj = __reduce_or_sync(kFull, join);
    const unsigned long long sum = warp_sum_u64(total);
    if ((threadIdx.x & 31) == 0) {
        if (a.total && sum) atomicAdd(a.total, sum);
        join_status(a.t.status, wj);
    }
}

/* retrieve_all_keys: slot `gid` emits its key when it is the key's first
 * entry along its bucket sequence (lowest slot of the first bucket holding
 * the key), compacted by block tiles (wc_compact.cuh) */
template <class L, int W>
__global__ void __launch_bounds__(256) mv_unique_keys_kernel(TableView t, uint64_t capacity,
                                                             void *keys_out,
                                                             unsigned long long *count)
{
    using K = typename L::key_t;
    constexpr int SB = L::kSlotBytes;
    const K empty = K(t.empty_key), tomb = K(t.tombstone_key);
    const unsigned char *const slots = reinterpret_cast<const unsigned char *>(t.slots);
    compact_tiles<K, K>(capacity, reinterpret_cast<K *>(keys_out), nullptr, count,
                        [&](uint64_t gid, K &key, K &) {
                            key = *reinterpret_cast<const K *>(slots + gid * SB);
                            if (key == empty || key == tomb) return false;
                            uint64_t b = probe_begin<K>(t, key), step = 0;
                            for (uint64_t w = 0; w < t.num_buckets; ++w) {
                                uint32_t hits, emp;
                                mv_bucket<L, W>(t, b, key, hits, emp,
                                                [](int, const LaneWords &, int) {});
                                if (hits) return b * W + uint64_t(__ffs(hits) - 1) == gid;
                                if (w == 0) step = probe_step<K>(t, key);
                                b = probe_next(t, b, step);
                            }
                            return false;
                        });
}

/* ---- inclusive scan of per-key counts into end offsets, begin offsets
 * one behind (the reference uses cub::DeviceScan::InclusiveSum) ---- */
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr uint64_t kScanTile = uint64_t(kScanThreads) * kScanItems;

/* block-wide exclusive scan of one value per thread; returns the block total */
__device__ __forceinline__ unsigned long long block_exclusive_scan(unsigned long long v,
                                                                   unsigned long long &excl)
{
    __shared__ unsigned long long warp_sums[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned long long w = lane < int(blockDim.x >> 5) ? warp_sums[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, w, o);
            if (lane >= o) w += y;
        }
        warp_sums[lane] = w; /* inclusive over warps */
    }
    __syncthreads();
    const unsigned long long warp_base = wid ? warp_sums[wid - 1] : 0ull;
    excl = warp_base + x - v;
    const unsigned long long total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return total;
}

template <int kUnused = 0>
__global__ void __launch_bounds__(kScanThreads) scan_tile_sums_kernel(
    const unsigned long long *counts, uint64_t n, unsigned long long *tile_sums)
{
    const uint64_t t0 = uint64_t(blockIdx.x) * kScanTile;
    unsigned long long s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const uint64_t i = t0 + uint64_t(threadIdx.x) * kScanItems + j;
        if (i < n) s += counts[i];
    }
    unsigned long long excl;
    const unsigned long long total = block_exclusive_scan(s, excl);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

/* one block: exclusive scan of the tile sums, in place */
template <int kUnused = 0>
__global__ void __launch_bounds__(kScanThreads) scan_tile_offsets_kernel(unsigned long long *tile_sums,
                                                                         uint64_t ntiles)
{
    const uint64_t per = (ntiles + kScanThreads - 1) / kScanThreads;
    const uint64_t b = uint64_t(threadIdx.x) * per;
    unsigned long long s = 0;
    for (uint64_t k = 0; k < per && b + k < ntiles; ++k) s += tile_sums[b + k];
    unsigned long long excl;
    block_exclusive_scan(s, excl);
    for (uint64_t k = 0; k < per && b + k < ntiles; ++k) {
        const unsigned long long c = tile_sums[b + k];
        tile_sums[b + k] = excl;
        excl += c;
    }
}

/* counts (in end) -> end = inclusive prefix sums, begin = end - count.
 * write_begin 0 leaves begin alone: the caller passed end == begin + 1 (the
 * reference's offsets_out, offsets_out + 1 idiom), where begin[i + 1] is
 * end[i] already and writing it would race with the block reading it. */
template <int kUnused = 0>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(unsigned long long *end,
                                                                  unsigned long long *begin,
                                                                  uint64_t n,
                                                                  const unsigned long long *tile_offsets,
                                                                  int write_begin)
{
    const uint64_t t0 = uint64_t(blockIdx.x) * kScanTile;
    unsigned long long c[kScanItems];
    unsigned long long s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const uint64_t i = t0 + uint64_t(threadIdx.x) * kScanItems + j;
        c[j] = i < n ? end[i] : 0ull;
        s += c[j];
    }
    unsigned long long excl;
    block_exclusive_scan(s, excl);
    unsigned long long run = tile_offsets[blockIdx.x] + excl;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const uint64_t i = t0 + uint64_t(threadIdx.x) * kScanItems + j;
        if (i < n) {
            if (write_begin) begin[i] = run;
            run += c[j];
            end[i] = run;
        }
    }
}

/* dry run of retrieve: every key's status is dry_run */
template <int kUnused = 0>
__global__ void __launch_bounds__(256) mv_dry_status_kernel(void *status_out, uint64_t n,
                                                            int handler, uint32_t bool_mask)
{
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (handler == kHandlerStatus)
            reinterpret_cast<uint32_t *>(status_out)[i] = kStDryRun;
        else if (handler == kHandlerBoolean)
            reinterpret_cast<unsigned char *>(status_out)[i] =
                (unsigned char)((kStDryRun & bool_mask) != 0);
    }
}

} // namespace b200
} // namespace warpcore

#endif /* WC_MV_CUH */
