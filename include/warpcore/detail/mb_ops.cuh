/*
 * mb_ops.cuh -- per-key MultiBucketHashTable operations shared by the bulk
 * kernels (warpcore_b200/csrc/wc_multibucket.cu) and the device per-key
 * methods of the C++ drop-in (include/warpcore/multi_bucket_hash_table.cuh).
 *
 * Reference semantics (multi_bucket_hash_table.cuh): a slot holds a key and
 * a bucket of `bucket` values, the empty value marking a free place.  A
 * key's slots lie along its probe sequence.  Insert (:343-517) notes the
 * last slot that holds the key and counts `bucket` values per such slot;
 * in the first window with a free slot it first tries to put the value in
 * that last bucket (insert_into_bucket, :262-330), and claims the free slot
 * only when the bucket is full, writing the value to the new bucket's first
 * place.  max_values_per_key caps the count (duplicate_key +
 * max_values_for_key_reached).  for_each (:786-846) walks the same windows
 * and hands out each hit slot's non-empty values.
 *
 * Layout (B200): keys and buckets are two arrays (structure of arrays).  A
 * probe window is `cg_size` consecutive keys of one bucket-aligned window,
 * 32 bytes for u32 keys at CG 8, read with 16-byte loads; a key's values
 * are read only for the slots that hold it.
 */
#ifndef WARPCORE_B200_MB_OPS_CUH
#define WARPCORE_B200_MB_OPS_CUH

#include "b200_core.cuh"

namespace warpcore {
namespace b200 {

constexpr uint32_t kStInvalidValue = 1u << 12;

/* a MultiBucketHashTable on the device: t.slots is the key array */
struct MbView {
    TableView t;
    void *vals;                      /* capacity * bucket values */
    uint64_t empty_value;
    uint64_t max_values;
    uint32_t bucket;                 /* values per slot, 1 .. cg_size */
    unsigned long long *num_keys;    /* keys that got a first slot */
    unsigned long long *num_occupied;/* claimed slots */
};

/* kW / kB: the window width (cg_size) and bucket size when known at
 * compile time, 0 to take them from the view.  The bulk kernels are built
 * for CG 8 with buckets of 1, 2, 4 and 8 and for any shape at run time. */
template <int kW>
__device__ __forceinline__ uint32_t mb_w(const MbView &m)
{
    return kW ? uint32_t(kW) : m.t.cg_size;
}
template <int kB>
__device__ __forceinline__ uint32_t mb_b(const MbView &m)
{
    return kB ? uint32_t(kB) : m.bucket;
}

/* one window of keys: bit s of hits / empties = key s equals `key` / is empty */
template <class K, int kW>
__device__ __forceinline__ void mb_window(const K *kw, uint32_t W, K key, K empty, uint32_t &hits,
                                          uint32_t &empties)
{
    hits = 0;
    empties = 0;
    const uint32_t bytes = W * uint32_t(sizeof(K));
    if (bytes >= 16) {
#pragma unroll
        for (uint32_t v = 0; v < (kW ? kW * sizeof(K) / 16 : bytes / 16); ++v) {
            const uint4 q = __ldcg(reinterpret_cast<const uint4 *>(kw) + v);
            if constexpr (sizeof(K) == 4) {
                const uint32_t s = v * 4;
                hits |= (uint32_t(q.x == key) | uint32_t(q.y == key) << 1 |
                         uint32_t(q.z == key) << 2 | uint32_t(q.w == key) << 3) << s;
                empties |= (uint32_t(q.x == empty) | uint32_t(q.y == empty) << 1 |
                            uint32_t(q.z == empty) << 2 | uint32_t(q.w == empty) << 3) << s;
            } else {
                const uint32_t s = v * 2;
                const K a = K(q.x) | (K(q.y) << 32), c = K(q.z) | (K(q.w) << 32);
                hits |= (uint32_t(a == key) | uint32_t(c == key) << 1) << s;
                empties |= (uint32_t(a == empty) | uint32_t(c == empty) << 1) << s;
            }
        }
    } else {
        for (uint32_t s = 0; s < W; ++s) {
            const K k = __ldcg(kw + s);
            if (k == key) hits |= 1u << s;
            if (k == empty) empties |= 1u << s;
        }
    }
}

/* bit r of the result: place r of a bucket holds the empty value.  With a
 * compile-time bucket of 8, 16 or 32 bytes (or more, in 16-byte pieces)
 * the places come in vector loads. */
template <class V, int kB>
__device__ __forceinline__ uint32_t mb_bucket_empties(const V *b, uint32_t B, V ev, V *vals_out)
{
    uint32_t e = 0;
    if constexpr (kB > 0 && (kB * sizeof(V)) % 8 == 0 && ((kB * sizeof(V)) & (kB * sizeof(V) - 1)) == 0) {
        constexpr int bytes = kB * int(sizeof(V));
        V v[kB];
        if constexpr (bytes == 8) {
            const uint2 q = __ldcg(reinterpret_cast<const uint2 *>(b));
            memcpy(v, &q, 8);
        } else {
#pragma unroll
            for (int c = 0; c < bytes / 16; ++c) {
                const uint4 q = __ldcg(reinterpret_cast<const uint4 *>(b) + c);
                memcpy(reinterpret_cast<char *>(v) + 16 * c, &q, 16);
            }
        }
#pragma unroll
        for (int r = 0; r < kB; ++r) {
            if (vals_out) vals_out[r] = v[r];
            e |= uint32_t(v[r] == ev) << r;
        }
    } else {
        for (uint32_t r = 0; r < B; ++r) {
            const V x = __ldcg(b + r);
            if (vals_out) vals_out[r] = x;
            e |= uint32_t(x == ev) << r;
        }
    }
    return e;
}

template <class V>
__device__ __forceinline__ V mb_cas(V *p, V expect, V desired)
{
    if constexpr (sizeof(V) == 8)
        return V(atomicCAS(reinterpret_cast<unsigned long long *>(p), (unsigned long long)expect,
                           (unsigned long long)desired));
    else
        return V(atomicCAS(reinterpret_cast<unsigned int *>(p), (unsigned int)expect,
                           (unsigned int)desired));
}

/* insert_into_bucket (:262-330): place 0 counts as full (its value is
 * written right after the slot's claim); the count grows by the full
 * places; the value goes to the first free place that a compare-and-swap
 * wins.  Returns true when the insert is decided (stored, or capped). */
template <class K, class V, int kB>
__device__ bool mb_into_bucket(const MbView &m, uint64_t slot, V value, uint64_t num_values,
                               uint32_t &st)
{
    const uint32_t B = mb_b<kB>(m);
    V *const b = reinterpret_cast<V *>(m.vals) + slot * B;
    const V ev = V(m.empty_value);
    uint32_t empties = mb_bucket_empties<V, kB>(b, B, ev, nullptr) & ~1u;
    num_values += B - uint32_t(__popc(empties));
    if (num_values >= m.max_values) {
        st = kStDuplicateKey | kStMaxValuesReached;
        return true;
    }
    while (empties) {
        const int r = __ffs(empties) - 1;
        if (mb_cas<V>(b + r, ev, value) == ev) {
            st = num_values > 0 ? kStDuplicateKey : kStNone;
            return true;
        }
        if (++num_values >= m.max_values) {
            st = kStDuplicateKey | kStMaxValuesReached;
            return true;
        }
        empties &= empties - 1u;
    }
    return false;
}

/* insert one (key, value).  Returns the per-key status; `claimed` /
 * `fresh` tell whether a slot was claimed and whether it was the key's
 * first.  The caller joins every status but none and the plain
 * duplicate_key of a stored value into the table status. */
template <class K, class V, int kW = 0, int kB = 0>
__device__ uint32_t mb_insert_one(const MbView &m, K key, V value, uint64_t max_windows,
                                  bool &claimed, bool &fresh)
{
    const TableView &t = m.t;
    const uint32_t W = mb_w<kW>(m), B = mb_b<kB>(m);
    const K empty = K(t.empty_key), tomb = K(t.tombstone_key);
    K *const keys = reinterpret_cast<K *>(t.slots);
    claimed = false;
    fresh = false;
    if (key == empty || key == tomb) return kStInvalidKey;
    if (value == V(m.empty_value)) return kStInvalidValue;
    uint64_t b = probe_begin<K>(t, key), step = 0, num = 0;
    uint64_t last = ~0ull;
    uint32_t st = kStUnknownError;
    for (uint64_t w = 0; w < max_windows; ++w) {
        uint32_t hits, emp;
        mb_window<K, kW>(keys + b * W, W, key, empty, hits, emp);
        if (hits) last = b * W + uint64_t(31 - __clz(hits));
        num += uint64_t(B) * uint64_t(__popc(hits));
        if (num >= m.max_values) {
            if (B == 1) return kStDuplicateKey | kStMaxValuesReached;
            mb_into_bucket<K, V, kB>(m, last, value, num - B, st);
            return st;
        }
        while (emp) {
            if (B > 1 && last != ~0ull && mb_into_bucket<K, V, kB>(m, last, value, num - B, st))
                return st;
            const int s = __ffs(emp) - 1;
            const uint64_t slot = b * W + uint64_t(s);
            const K old = mb_cas<K>(keys + slot, empty, key);
            if (old == empty) {
                /* the bucket's first place, after the key (:446-449) */
                reinterpret_cast<V *>(m.vals)[slot * B] = value;
                claimed = true;
                fresh = num == 0;
                return num > 0 ? kStDuplicateKey : kStNone;
            }
            if (old == key) {
                num += B;
                if (B == 1 && num >= m.max_values) return kStDuplicateKey | kStMaxValuesReached;
                last = slot;
            }
            emp &= emp - 1u;
        }
        if (w == 0) step = probe_step<K>(t, key);
        b = probe_next(t, b, step);
    }
    if (B > 1 && last != ~0ull && mb_into_bucket<K, V, kB>(m, last, value, num - B, st)) return st;
    return kStProbingLengthExceeded | (num > 0 ? kStDuplicateKey : kStNone);
}

/* for_each over one key's values (:786-846): f(value, index) when kValues;
 * returns the status (none, key_not_found, probing_length_exceeded,
 * invalid_key) and the count in num.  The count takes bucket values per
 * hit slot less the empty places of each window's last hit slot, so a
 * count-only walk reads that one bucket per window.  A walk that already
 * knows the key's count passes it as stop_at and ends at the window where
 * that many values are read (status none). */
template <class K, class V, int kW = 0, int kB = 0, bool kValues = true, class F>
__device__ uint32_t mb_for_each_one(const MbView &m, K key, uint64_t max_windows, uint64_t &num,
                                    F f, uint64_t stop_at = ~uint64_t(0))
{
    const TableView &t = m.t;
    const uint32_t W = mb_w<kW>(m), B = mb_b<kB>(m);
    const K empty = K(t.empty_key), tomb = K(t.tombstone_key);
    const K *const keys = reinterpret_cast<const K *>(t.slots);
    const V *const vals = reinterpret_cast<const V *>(m.vals);
    const V ev = V(m.empty_value);
    num = 0;
    if (key == empty || key == tomb) return kStInvalidKey;
    uint64_t b = probe_begin<K>(t, key), step = 0;
    for (uint64_t w = 0; w < max_windows; ++w) {
        uint32_t hits, emp;
        mb_window<K, kW>(keys + b * W, W, key, empty, hits, emp);
        if (hits) {
            const int last = 31 - __clz(hits);
            uint32_t le;
            if constexpr (kValues) {
                /* hit slots in ascending order: the last one read is the
                 * window's last bucket, whose free places the count needs */
                uint64_t j = num;
                uint32_t e = 0;
                for (uint32_t x = hits; x; x &= x - 1u) {
                    const uint64_t slot = b * W + uint64_t(__ffs(x) - 1);
                    V v[kB ? kB : 32];
                    e = mb_bucket_empties<V, kB>(vals + slot * B, B, ev, v);
                    for (uint32_t r = 0; r < (kB ? uint32_t(kB) : B); ++r)
                        if (!((e >> r) & 1u)) f(v[r], j + r);
                    j += B;
                }
                le = __popc(e);
            } else {
                le = __popc(mb_bucket_empties<V, kB>(vals + (b * W + uint64_t(last)) * B, B, ev,
                                                     nullptr));
            }
            num += uint64_t(B) * uint64_t(__popc(hits)) - le;
            if (num >= stop_at) return kStNone;
        }
        if (emp || num >= m.max_values) return num ? kStNone : kStKeyNotFound;
        if (w == 0) step = probe_step<K>(t, key);
        b = probe_next(t, b, step);
    }
    return kStProbingLengthExceeded;
}

} // namespace b200
} // namespace warpcore

#endif /* WARPCORE_B200_MB_OPS_CUH */
