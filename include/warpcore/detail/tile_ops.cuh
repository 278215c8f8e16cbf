/*
 * tile_ops.cuh -- per-key device operations for a cooperative group of
 * cg_size threads (the reference's device API: insert_impl / retrieve /
 * erase, single_value_hash_table.cuh:211-468, 743-823; hash_set.cuh:193-462;
 * counting_hash_table.cuh:142-225).  Thread r of the group inspects slot r of
 * the key's bucket-aligned window, so these calls find the keys the bulk
 * kernels stored and vice versa.
 */
#ifndef WARPCORE_B200_TILE_OPS_CUH
#define WARPCORE_B200_TILE_OPS_CUH

#include <cooperative_groups.h>
#include <warpcore/detail/b200_core.cuh>

namespace warpcore {
namespace b200 {

template <class L>
__device__ __forceinline__ typename L::key_t tile_slot_key(const void *sp)
{
    using K = typename L::key_t;
    return __ldcg(reinterpret_cast<const K *>(sp));
}

/* Insert (op 0), counting insert (op 1) or erase (op 3) of one key by the
 * tile.  Returns the per-key status and joins the table status like the
 * bulk kernels. */
template <class L, class Tile>
__device__ uint32_t tile_modify(const TableView &t, const Tile &g, typename L::key_t key,
                                typename L::val_t val, int op, uint64_t probing_length)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    constexpr int SB = L::kSlotBytes;
    const K empty = K(t.empty_key), tomb = K(t.tombstone_key);
    const unsigned W = g.size();
    const unsigned r = g.thread_rank();
    unsigned char *const slots = reinterpret_cast<unsigned char *>(t.slots);
    uint32_t st = kStNone, join = 0;
    if (key == empty || key == tomb) {
        st = join = kStInvalidKey;
    } else {
        uint64_t b = probe_begin<K>(t, key), step = 0, wins = 0;
        const uint64_t maxw = max_windows(probing_length, W, t.num_buckets);
        for (;;) {
            unsigned char *const sp = slots + (b * W + r) * SB;
            const K sk = tile_slot_key<L>(sp);
            const unsigned hit = g.ballot(sk == key);
            if (hit) {
                const unsigned leader = __ffs(hit) - 1;
                if (op == 3) {
                    if (r == leader && erase_slot<L>(sp, key, tomb)) {
                        fp_store(t, b * W + r, kFpTomb);
                        live_add(t, -1);
                    }
                    st = kStNone;
                } else {
                    st = kStDuplicateKey;
                    join = kStDuplicateKey;
                    if (r == leader) {
                        if (op == 0) put_value<L>(t, sp, b * W + r, val);
                        else if constexpr (L::kHasValue) count_add<L>(sp, 1u, t.max_count, st, join);
                    }
                    st = g.shfl(st, leader);
                    join = g.shfl(join, leader);
                }
                break;
            }
            unsigned emp = g.ballot(sk == empty);
            if (op == 3 && emp) {
                st = kStKeyNotFound;
                break;
            }
            bool done = false;
            while (emp) {
                const unsigned leader = __ffs(emp) - 1;
                int outcome = 0; /* 1 claimed, 2 duplicate */
                if (r == leader) {
                    K old_key;
                    const V payload = op == 1 ? V(1) : val;
                    if (claim_slot<L>(sp, empty, key, payload, old_key)) {
                        fp_store(t, b * W + r, fingerprint(key));
                        if constexpr (is_soa<L>::value) put_value<L>(t, sp, b * W + r, val);
                        live_add(t, 1);
                        outcome = 1;
                    } else if (old_key == key) {
                        outcome = 2;
                        uint32_t s2 = kStDuplicateKey, j2 = kStDuplicateKey;
                        if (op == 0) put_value<L>(t, sp, b * W + r, val);
                        else if constexpr (L::kHasValue) count_add<L>(sp, 1u, t.max_count, s2, j2);
                        st = s2;
                        join = j2;
                    }
                }
                outcome = g.shfl(outcome, leader);
                if (outcome == 1) {
                    st = kStNone;
                    done = true;
                    break;
                }
                if (outcome == 2) {
                    st = g.shfl(st, leader);
                    join = g.shfl(join, leader);
                    done = true;
                    break;
                }
                emp &= emp - 1u;
            }
            if (done) break;
            if (++wins >= maxw) {
                st = kStProbingLengthExceeded;
                if (op != 3) join = kStProbingLengthExceeded;
                break;
            }
            if (wins == 1) step = probe_step<K>(t, key);
            b = probe_next(t, b, step);
        }
    }
    if (join && r == 0) join_status(t.status, join);
    return st;
}

/* Retrieve one key: status none and the value (or found = true for sets);
 * key_not_found (sets: none with found = false); probing_length_exceeded */
template <class L, class Tile>
__device__ uint32_t tile_find(const TableView &t, const Tile &g, typename L::key_t key,
                              typename L::val_t &value_out, bool &found, bool is_set,
                              uint64_t probing_length)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    constexpr int SB = L::kSlotBytes;
    const K empty = K(t.empty_key), tomb = K(t.tombstone_key);
    const unsigned W = g.size();
    const unsigned r = g.thread_rank();
    const unsigned char *const slots = reinterpret_cast<const unsigned char *>(t.slots);
    uint32_t st, join = 0;
    found = false;
    if (key == empty || key == tomb) {
        st = join = kStInvalidKey;
    } else {
        uint64_t b = probe_begin<K>(t, key), step = 0, wins = 0;
        const uint64_t maxw = max_windows(probing_length, W, t.num_buckets);
        for (;;) {
            const unsigned char *const sp = slots + (b * W + r) * SB;
            const K sk = tile_slot_key<L>(sp);
            const unsigned hit = g.ballot(sk == key);
            if (hit) {
                const unsigned leader = __ffs(hit) - 1;
                V v = 0;
                if constexpr (is_soa<L>::value) {
                    if (r == leader) v = get_soa_value<L>(t, b * W + r);
                } else if (L::kHasValue && r == leader) {
                    v = *slot_value_ptr<L>(const_cast<unsigned char *>(sp));
                }
                value_out = g.shfl(v, leader);
                if (uint64_t(value_out) > t.max_count) value_out = V(t.max_count);
                found = true;
                st = kStNone;
                break;
            }
            if (g.any(sk == empty)) {
                st = is_set ? kStNone : kStKeyNotFound;
                join = st;
                break;
            }
            if (++wins >= maxw) {
                st = join = kStProbingLengthExceeded;
                break;
            }
            if (wins == 1) step = probe_step<K>(t, key);
            b = probe_next(t, b, step);
        }
    }
    if (join && r == 0) join_status(t.status, join);
    return st;
}

} // namespace b200
} // namespace warpcore

#endif
