/*
 * bl_ops.cuh -- per-key BucketListHashTable operations shared by the bulk
 * kernels (warpcore_b200/csrc/wc_bucketlist.cu) and the device per-key
 * methods of the C++ drop-in (include/warpcore/bucket_list_hash_table.cuh).
 *
 * Reference semantics (bucket_list_hash_table.cuh over BucketListStore,
 * storage.cuh:651-1454): a single-value table maps each key to a 64-bit
 * handle of a list of value buckets in a shared pool.  The first bucket
 * holds min_bucket_size values and no header; every later bucket starts
 * with a header {previous bucket, size}, its size the previous one times
 * grow_factor (float, rounded up) up to max_bucket_size.  A handle is
 * {state, bucket index, value count, values in the newest bucket}; states
 * uninitialized / initialized / blocking (a thread is allocating) / full
 * (the pool ran out).  Appends take a free place of the newest bucket by a
 * compare-and-swap of the handle, or block the handle, allocate the next
 * bucket from the pool's bump counter and publish it.  Lists are read
 * newest bucket first, each bucket from its first place.
 *
 * Layout (B200): keys, handles and the pool are three arrays.  A probe
 * window is cg_size keys (32 bytes for u32 at CG 8); the handle is read
 * only at the key's slot.  The wait on a blocked handle is bounded.
 */
#ifndef WARPCORE_B200_BL_OPS_CUH
#define WARPCORE_B200_BL_OPS_CUH

#include "mb_ops.cuh"

namespace warpcore {
namespace b200 {

enum : uint32_t { kBlUninit = 0, kBlInit = 1, kBlBlocking = 2, kBlFull = 3 };

/* polls of a blocked handle before an append gives up with unknown_error;
 * the thread holding it only allocates and publishes, so the wait is short */
constexpr uint32_t kBlSpinLimit = 1u << 22;

struct BlView {
    TableView t;                     /* t.slots: key array */
    unsigned long long *handles;     /* one per key slot */
    unsigned long long *pool;        /* value_capacity elements: value or header */
    unsigned long long *next_free;   /* the pool's bump counter */
    uint64_t capacity;               /* pool elements */
    uint64_t min_bucket, max_bucket, max_values;
    float grow;
    uint32_t ib, cb, sb;             /* bucket index, counter and size bits */
};

struct BlHandle {
    uint32_t state;
    uint64_t index, count, tail;
};

__host__ __device__ __forceinline__ uint64_t bl_head(uint32_t ib) { return (1ull << ib) - 1; }

__host__ __device__ __forceinline__ unsigned long long bl_pack(const BlView &v, uint32_t state,
                                                               uint64_t index, uint64_t count,
                                                               uint64_t tail)
{
    return (unsigned long long)state | (index << 2) | (count << (2 + v.ib)) |
           (tail << (2 + v.ib + v.cb));
}

__host__ __device__ __forceinline__ BlHandle bl_unpack(const BlView &v, unsigned long long h)
{
    BlHandle r;
    r.state = uint32_t(h & 3u);
    r.index = (h >> 2) & ((1ull << v.ib) - 1);
    r.count = (h >> (2 + v.ib)) & ((1ull << v.cb) - 1);
    r.tail = (h >> (2 + v.ib + v.cb)) & ((1ull << v.sb) - 1);
    return r;
}

/* a bucket header in a pool element: previous bucket and size */
__device__ __forceinline__ unsigned long long bl_header(const BlView &v, uint64_t prev,
                                                        uint64_t size)
{
    return (unsigned long long)prev | ((unsigned long long)size << v.ib);
}
__device__ __forceinline__ uint64_t bl_header_prev(const BlView &v, unsigned long long e)
{
    return e & ((1ull << v.ib) - 1);
}
__device__ __forceinline__ uint64_t bl_header_size(const BlView &v, unsigned long long e)
{
    return (e >> v.ib) & ((1ull << v.sb) - 1);
}

__device__ __forceinline__ unsigned long long bl_load(const unsigned long long *p)
{
    return *reinterpret_cast<const volatile unsigned long long *>(p);
}

/* the key's slot in the key table: hit (duplicate_key) or a claimed empty
 * slot (none), as the single-value table's insert (single_value_hash_table
 * .cuh:743-823); ~0 with probing_length_exceeded or invalid_key */
template <class K, int kW>
__device__ uint64_t bl_claim(const BlView &v, K key, uint64_t max_windows, uint32_t &st)
{
    const TableView &t = v.t;
    const uint32_t W = kW ? uint32_t(kW) : t.cg_size;
    const K empty = K(t.empty_key), tomb = K(t.tombstone_key);
    K *const keys = reinterpret_cast<K *>(t.slots);
    if (key == empty || key == tomb) {
        st = kStInvalidKey;
        return ~0ull;
    }
    uint64_t b = probe_begin<K>(t, key), step = 0;
    for (uint64_t w = 0; w < max_windows; ++w) {
        uint32_t hits, emp;
        mb_window<K, kW>(keys + b * W, W, key, empty, hits, emp);
        if (hits) {
            st = kStDuplicateKey;
            return b * W + uint64_t(__ffs(hits) - 1);
        }
        while (emp) {
            const int s = __ffs(emp) - 1;
            const uint64_t slot = b * W + uint64_t(s);
            const K old = mb_cas<K>(keys + slot, empty, key);
            if (old == empty) {
                st = kStNone;
                return slot;
            }
            if (old == key) {
                st = kStDuplicateKey;
                return slot;
            }
            emp &= emp - 1u;
        }
        if (w == 0) step = probe_step<K>(t, key);
        b = probe_next(t, b, step);
    }
    st = kStProbingLengthExceeded;
    return ~0ull;
}

/* the key's slot for reads (single_value_hash_table.cuh:268-307): none,
 * key_not_found (a window with an empty slot), probing_length_exceeded,
 * invalid_key */
template <class K, int kW>
__device__ uint64_t bl_find(const BlView &v, K key, uint64_t max_windows, uint32_t &st)
{
    const TableView &t = v.t;
    const uint32_t W = kW ? uint32_t(kW) : t.cg_size;
    const K empty = K(t.empty_key), tomb = K(t.tombstone_key);
    const K *const keys = reinterpret_cast<const K *>(t.slots);
    if (key == empty || key == tomb) {
        st = kStInvalidKey;
        return ~0ull;
    }
    uint64_t b = probe_begin<K>(t, key), step = 0;
    for (uint64_t w = 0; w < max_windows; ++w) {
        uint32_t hits, emp;
        mb_window<K, kW>(keys + b * W, W, key, empty, hits, emp);
        if (hits) {
            st = kStNone;
            return b * W + uint64_t(__ffs(hits) - 1);
        }
        if (emp) {
            st = kStKeyNotFound;
            return ~0ull;
        }
        if (w == 0) step = probe_step<K>(t, key);
        b = probe_next(t, b, step);
    }
    st = kStProbingLengthExceeded;
    return ~0ull;
}

/* pool allocation of `size` elements by the bump counter.  The lanes of a
 * warp that allocate together share one atomicAdd (the counter is a single
 * address that every list of the table grows through) and take
 * consecutive ranges in lane order; the counter ends where separate adds
 * would leave it, so a pool that runs out fails the same requests' worth
 * of elements. */
__device__ __forceinline__ unsigned long long bl_alloc(const BlView &v, uint64_t size)
{
    const unsigned m = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    unsigned long long before = 0, total = 0;
    for (unsigned rest = m; rest; rest &= rest - 1u) {
        const int src = __ffs(rest) - 1;
        const unsigned long long s = __shfl_sync(m, (unsigned long long)size, src);
        if (src < lane) before += s;
        total += s;
    }
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(v.next_free, total);
    base = __shfl_sync(m, base, leader);
    return base + before;
}

/* append (storage.cuh:1108-1285) of one value to the list of handle h */
template <class V>
__device__ uint32_t bl_append(const BlView &v, unsigned long long *h, V value,
                             unsigned long long cur)
{
    /* cur: the handle as the caller read it.  Every step is checked by a
     * compare-and-swap, whose result is the handle's current value, so a
     * stale cur costs one retry and the handle is reloaded only after
     * waiting on a list that another thread is growing. */
    const uint64_t head = bl_head(v.ib);
    if (bl_unpack(v, cur).state == kBlUninit) {
        const unsigned long long blocked = bl_pack(v, kBlBlocking, head, 0, 0);
        const unsigned long long old = atomicCAS(h, cur, blocked);
        if (old == cur) {
            /* this thread allocates the first bucket */
            const unsigned long long alloc = bl_alloc(v, v.min_bucket);
            if (alloc + v.min_bucket <= v.capacity) {
                v.pool[alloc] = (unsigned long long)value;
                __threadfence();
                atomicExch(h, bl_pack(v, kBlInit, alloc, 1, 1));
                return kStNone;
            }
            atomicExch(h, bl_pack(v, kBlFull, head, 0, 0));
            return kStOutOfMemory;
        }
        cur = old;
    }
    for (uint32_t spin = 0; spin < kBlSpinLimit; ++spin) {
        const BlHandle c = bl_unpack(v, cur);
        if (c.state == kBlBlocking || c.state == kBlUninit) {
            __nanosleep(32);
            cur = bl_load(h);
            continue;
        }
        if (c.state == kBlFull) return kStOutOfMemory;
        if (c.count == v.max_values) return kStMaxValuesReached;
        const uint64_t size =
            c.count <= v.min_bucket ? v.min_bucket : bl_header_size(v, bl_load(v.pool + c.index));
        if (c.tail == size) {
            /* the newest bucket is full: block the handle, allocate the next */
            const unsigned long long old =
                atomicCAS(h, cur, bl_pack(v, kBlBlocking, c.index, c.count, c.tail));
            if (old != cur) {
                cur = old;
                continue;
            }
            const float grown = ceilf(float(size) * v.grow);
            const float cap = float(v.max_bucket);
            const uint64_t nsize = uint64_t(cap < grown ? cap : grown);
            const unsigned long long alloc = bl_alloc(v, nsize + 1);
            if (alloc + nsize + 1 <= v.capacity) {
                v.pool[alloc + 1] = (unsigned long long)value;
                v.pool[alloc] = bl_header(v, c.index, nsize);
                __threadfence();
                atomicExch(h, bl_pack(v, kBlInit, alloc, c.count + 1, 1));
                return kStNone;
            }
            atomicExch(h, bl_pack(v, kBlFull, c.index, c.count, c.tail));
            return kStOutOfMemory;
        }
        const unsigned long long old =
            atomicCAS(h, cur, bl_pack(v, kBlInit, c.index, c.count + 1, c.tail + 1));
        if (old == cur) {
            const uint64_t j = c.count + 1 <= v.min_bucket ? c.tail : c.tail + 1;
            v.pool[c.index + j] = (unsigned long long)value;
            return kStNone;
        }
        cur = old;
    }
    return kStUnknownError;
}

/* insert one (key, value) (:187-222, 235-326): the key's slot, then the
 * append unless the list holds max_values_per_key values */
template <class K, class V, int kW = 0>
__device__ uint32_t bl_insert_one(const BlView &v, K key, V value, uint64_t max_windows,
                                  uint32_t &join)
{
    uint32_t st = kStUnknownError;
    const uint64_t slot = bl_claim<K, kW>(v, key, max_windows, st);
    join = st == kStNone ? 0u : st; /* the key table joins what it reports */
    if (slot == ~0ull) return st;
    unsigned long long *const h = v.handles + slot;
    uint32_t ast;
    const unsigned long long cur = bl_load(h);
    if (bl_unpack(v, cur).count >= v.max_values) ast = kStMaxValuesReached;
    else ast = bl_append<V>(v, h, value, cur);
    join |= ast;
    return st | ast;
}

/* the values of handle h in list order: f(value, index) */
template <class V, class F>
__device__ void bl_walk(const BlView &v, unsigned long long h, F f)
{
    const BlHandle c = bl_unpack(v, h);
    if (c.state != kBlInit || c.index == bl_head(v.ib)) return;
    uint64_t ptr = c.index;
    uint64_t off = c.count <= v.min_bucket ? 0 : 1;
    uint64_t g = 0;
    /* (every pool index is checked against the capacity: a list is only
     * read once its handle was published after its headers, but a read
     * that overlaps an insert must not leave the pool) */
    if (ptr + off + c.tail > v.capacity) return;
    for (uint64_t l = 0; l < c.tail; ++l, ++g) f(V(v.pool[ptr + l + off]), g);
    while (g < c.count) {
        ptr = bl_header_prev(v, v.pool[ptr]);
        if (ptr >= v.capacity) return;
        const bool last = g >= c.count - v.min_bucket;
        const uint64_t size = last ? v.min_bucket : bl_header_size(v, v.pool[ptr]);
        off = last ? 0 : 1;
        if (ptr + off + size > v.capacity) return;
        for (uint64_t l = 0; l < size && g < c.count; ++l, ++g) f(V(v.pool[ptr + l + off]), g);
    }
}

/* retrieve / num_values of one key (:342-371, 740-757): the status of the
 * key table's lookup; num = the list's count (0 when not found) */
template <class K, class V, int kW = 0, bool kValues = true, class F>
__device__ uint32_t bl_for_each_one(const BlView &v, K key, uint64_t max_windows, uint64_t &num,
                                    F f)
{
    uint32_t st = kStUnknownError;
    num = 0;
    const uint64_t slot = bl_find<K, kW>(v, key, max_windows, st);
    if (slot == ~0ull) return st;
    const unsigned long long h = v.handles[slot];
    num = bl_unpack(v, h).count;
    if constexpr (kValues) bl_walk<V>(v, h, f);
    return st;
}

} // namespace b200
} // namespace warpcore

#endif /* WARPCORE_B200_BL_OPS_CUH */
