/*
 * mv_ops.cuh -- per-key MultiValueHashTable operations shared by the bulk
 * kernels (warpcore_b200/csrc/wc_mv.cuh) and the device per-key methods of
 * the C++ drop-in (include/warpcore/multi_value_hash_table.cuh).
 *
 * Reference semantics (multi_value_hash_table.cuh): every (key, value) pair
 * takes a slot of its own.  A key's values live along its bucket sequence,
 * up to the first bucket that has a free slot.  Insert (:200-289) counts the
 * key's values bucket by bucket, stops with duplicate_key +
 * max_values_for_key_reached at max_values_per_key, and claims the first
 * free slot of the first bucket that has one; an equal key claiming a slot
 * first counts as one more value.  for_each (:607-663) takes the key's
 * slots in slot order until a bucket has a free slot or the count reaches
 * max_values_per_key.  Buckets are the bulk kernels' bucket-aligned
 * windows, so a key's values come out in the order they were inserted.
 */
#ifndef WARPCORE_B200_MV_OPS_CUH
#define WARPCORE_B200_MV_OPS_CUH

#include "b200_core.cuh"

namespace warpcore {
namespace b200 {

/* one bucket: bit s of hits / empties = slot s holds key / is empty; on_hit
 * gets (slot index in the bucket, the 16-byte words read, slot within them)
 * for every hit, in slot order */
template <class L, int W, class OnHit>
__device__ __forceinline__ void mv_bucket(const TableView &t, uint64_t bucket,
                                          typename L::key_t key, uint32_t &hits,
                                          uint32_t &empties, OnHit on_hit)
{
    using K = typename L::key_t;
    constexpr int SB = L::kSlotBytes;
    constexpr int WB = W * SB;
    constexpr int LB = WB < 16 ? WB : 16;
    constexpr int NV = WB / LB;
    constexpr int SPL = LB / SB;
    const K empty = K(t.empty_key);
    const unsigned char *const base =
        reinterpret_cast<const unsigned char *>(t.slots) + bucket * uint64_t(WB);
    hits = 0;
    empties = 0;
#pragma unroll 4
    for (int v = 0; v < NV; ++v) {
        const LaneWords lw = load_lane<LB>(base + v * LB);
#pragma unroll
        for (int s = 0; s < SPL; ++s) {
            const K k = slot_key<L>(lw, s);
            const int idx = v * SPL + s;
            if (k == key) {
                hits |= 1u << idx;
                on_hit(idx, lw, s);
            }
            if (k == empty) empties |= 1u << idx;
        }
    }
}

/* insert one (key, value); returns the per-key status (the caller joins
 * the error bits into the table status) and sets new_key when the key got
 * its first value */
template <class L, int W>
__device__ uint32_t mv_insert_one(const TableView &t, typename L::key_t key,
                                  typename L::val_t val, uint64_t max_windows,
                                  uint64_t max_values, bool &new_key)
{
    using K = typename L::key_t;
    constexpr int SB = L::kSlotBytes;
    const K empty = K(t.empty_key), tomb = K(t.tombstone_key);
    unsigned char *const slots = reinterpret_cast<unsigned char *>(t.slots);
    new_key = false;
    if (key == empty || key == tomb) return kStInvalidKey;
    uint64_t b = probe_begin<K>(t, key), step = 0, wins = 0, num = 0;
    for (;;) {
        uint32_t hits, emp;
        mv_bucket<L, W>(t, b, key, hits, emp, [](int, const LaneWords &, int) {});
        num += __popc(hits);
        if (num >= max_values) return kStDuplicateKey | kStMaxValuesReached;
        while (emp) {
            const int s = __ffs(emp) - 1;
            unsigned char *const sp = slots + (b * W + uint64_t(s)) * SB;
            K old;
            if (claim_slot<L>(sp, empty, key, val, old)) {
                new_key = num == 0;
                return num ? kStDuplicateKey : kStNone;
            }
            if (old == key && ++num >= max_values) return kStDuplicateKey | kStMaxValuesReached;
            emp &= emp - 1u;
        }
        if (++wins >= max_windows)
            return kStProbingLengthExceeded | (num ? kStDuplicateKey : kStNone);
        if (wins == 1) step = probe_step<K>(t, key);
        b = probe_next(t, b, step);
    }
}

/* for_each over one key's values: f(value, index) in insertion order;
 * returns the status (none, key_not_found, probing_length_exceeded,
 * invalid_key) and the count in num */
template <class L, int W, class F>
__device__ uint32_t mv_for_each_one(const TableView &t, typename L::key_t key,
                                    uint64_t max_windows, uint64_t max_values, uint64_t &num, F f)
{
    using K = typename L::key_t;
    const K empty = K(t.empty_key), tomb = K(t.tombstone_key);
    num = 0;
    if (key == empty || key == tomb) return kStInvalidKey;
    uint64_t b = probe_begin<K>(t, key), step = 0, wins = 0;
    for (;;) {
        uint32_t hits, emp;
        mv_bucket<L, W>(t, b, key, hits, emp, [&](int, const LaneWords &lw, int s) {
            f(slot_val<L>(lw, s), num);
            ++num;
        });
        if (emp || num >= max_values) return num ? kStNone : kStKeyNotFound;
        if (++wins >= max_windows) return kStProbingLengthExceeded;
        if (wins == 1) step = probe_step<K>(t, key);
        b = probe_next(t, b, step);
    }
}

} // namespace b200
} // namespace warpcore

#endif /* WARPCORE_B200_MV_OPS_CUH */
