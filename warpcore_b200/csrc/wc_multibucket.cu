/*
 * wc_multibucket.cu -- MultiBucketHashTable (the reference's
 * multi_bucket_hash_table.cuh): kernels and the wc_mbht_* C ABI.
 *
 * Layout: the key array (capacity keys, bucket-aligned probe windows of
 * cg_size keys) and the bucket array (capacity x bucket values) are
 * separate; the reference keeps {key, value[bucket]} structures (AoSStore).
 * A probe window then costs cg_size keys (32 bytes for u32 at CG 8) whatever
 * the bucket size, and a key's values are read only where the key is.
 * Every kernel runs one key per lane (detail/mb_ops.cuh).
 */
#include <warpcore_b200.h>

#include "wc_internal.h"
#include "wc_compact.cuh"
#include <warpcore/detail/mb_ops.cuh>

#include <cstdio>
#include <cstring>

using namespace warpcore::b200;

struct wc_mbht {
    wc_table_config cfg{};
    uint32_t bucket = 1;
    uint64_t empty_value = 0;
    uint64_t capacity = 0, num_buckets = 0, seed = 0, max_values = ~0ull;
    void *keys = nullptr;
    void *vals = nullptr;
    uint32_t *status = nullptr;           /* device Status word */
    unsigned long long *counters = nullptr; /* device: num_keys, num_occupied, scratch */
    void *scan = nullptr;                 /* scan tile sums, grown on demand */
    uint64_t scan_bytes = 0;
    bool initialized = false;
};

namespace {

#define MB_CUDA(call)                                                          \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) return host_cuda_fail(e_, #call);               \
    } while (0)

constexpr int kBlock = 256;

int mb_fail(int code, const char *msg) { return host_fail(code, msg); }

uint64_t kmask(uint32_t bytes) { return bytes == 4 ? 0xffffffffull : ~0ull; }

struct MbArgs {
    MbView m;
    const void *keys;
    const void *values;              /* insert */
    void *values_out;                /* retrieve */
    const unsigned long long *begin; /* retrieve */
    const unsigned long long *end;
    unsigned long long *counts_out;  /* num_values: per key, or NULL */
    unsigned long long *total;       /* num_values: sum */
    void *status_out;
    uint64_t n;
    uint64_t max_windows;
    uint32_t bool_mask;
    int handler;
};

__device__ __forceinline__ void mb_write_status(const MbArgs &a, uint64_t i, uint32_t st)
{
    if (!a.status_out) return;
    if (a.handler == kHandlerStatus)
        reinterpret_cast<uint32_t *>(a.status_out)[i] = st;
    else if (a.handler == kHandlerBoolean)
        reinterpret_cast<unsigned char *>(a.status_out)[i] = (unsigned char)((st & a.bool_mask) != 0);
}

/* warp sums of two counters and the joined status, one atomic each per warp */
__device__ __forceinline__ void mb_flush(const MbView &m, uint32_t join, unsigned claimed,
                                         unsigned fresh)
{
    const uint32_t wj = __reduce_or_sync(0xffffffffu, join);
    const unsigned c = __reduce_add_sync(0xffffffffu, claimed);
    const unsigned f = __reduce_add_sync(0xffffffffu, fresh);
    if ((threadIdx.x & 31) == 0) {
        if (c) atomicAdd(m.num_occupied, (unsigned long long)c);
        if (f) atomicAdd(m.num_keys, (unsigned long long)f);
        join_status(m.t.status, wj);
    }
}

template <class K, class V, int kW, int kB>
__global__ void __launch_bounds__(256, WC_MULTI_MIN_BLOCKS) mb_insert_kernel(const MbArgs a)
{
    uint32_t join = 0;
    unsigned claimed = 0, fresh = 0;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        bool c = false, f = false;
        const uint32_t st = mb_insert_one<K, V, kW, kB>(a.m, reinterpret_cast<const K *>(a.keys)[i],
                                                reinterpret_cast<const V *>(a.values)[i],
                                                a.max_windows, c, f);
        /* every status but a stored value's none / duplicate_key is joined */
        if (st != kStNone && st != kStDuplicateKey) join |= st;
        claimed += c;
        fresh += f;
        mb_write_status(a, i, st);
    }
    mb_flush(a.m, join, claimed, fresh); /* every lane arrives (no early exit) */
}

/* num_values (kValues false) or retrieve of each key's values */
template <class K, class V, int kW, int kB, bool kValues>
__global__ void __launch_bounds__(256, WC_MULTI_MIN_BLOCKS) mb_find_kernel(const MbArgs a)
{
    uint32_t join = 0;
    unsigned long long total = 0;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        uint64_t num = 0;
        const K key = reinterpret_cast<const K *>(a.keys)[i];
        if constexpr (kValues) {
            /* The counting pass walked every key to its end and wrote its
             * status; this pass only reads values.  A key counted at 0
             * needs no walk, and a walk ends once the counted values are
             * read.  Values go inside the key's own segment only. */
            const uint64_t room = a.end[i] - a.begin[i];
            if (room == 0) continue;
            V *const out = reinterpret_cast<V *>(a.values_out) + a.begin[i];
            mb_for_each_one<K, V, kW, kB, true>(
                a.m, key, a.max_windows, num, [&](V v, uint64_t j) {
                    if (j < room) out[j] = v;
                },
                room);
        } else {
            const uint32_t st = mb_for_each_one<K, V, kW, kB, false>(a.m, key, a.max_windows, num,
                                                                     [](V, uint64_t) {});
            join |= st;
            if (a.counts_out) a.counts_out[i] = num;
            total += num;
            mb_write_status(a, i, st);
        }
    }
    const uint32_t wj = __reduce_or_sync(0xffffffffu, join);
    const unsigned long long sum = warp_sum_u64(total);
    if ((threadIdx.x & 31) == 0) {
        if (a.total && sum) atomicAdd(a.total, sum);
        join_status(a.m.t.status, wj);
    }
}

/* retrieve_all_keys (gpu_engine.cuh:51-93): slot `gid` emits its key when
 * it is the lowest slot of the first window holding the key; compacted by
 * block tiles (wc_compact.cuh) */
template <class K>
__global__ void __launch_bounds__(256) mb_unique_keys_kernel(const MbView m, uint64_t capacity,
                                                             void *keys_out,
                                                             unsigned long long *count)
{
    const TableView &t = m.t;
    const K empty = K(t.empty_key), tomb = K(t.tombstone_key);
    const K *const keys = reinterpret_cast<const K *>(t.slots);
    compact_tiles<K, K>(capacity, reinterpret_cast<K *>(keys_out), nullptr, count,
                        [&](uint64_t gid, K &key, K &) {
                            key = keys[gid];
                            if (key == empty || key == tomb) return false;
                            uint64_t b = probe_begin<K>(t, key), step = 0;
                            for (uint64_t w = 0; w < t.num_buckets; ++w) {
                                uint32_t hits, emp;
                                mb_window<K, 0>(keys + b * t.cg_size, t.cg_size, key, empty,
                                                hits, emp);
                                if (hits) return b * t.cg_size + uint64_t(__ffs(hits) - 1) == gid;
                                if (w == 0) step = probe_step<K>(t, key);
                                b = probe_next(t, b, step);
                            }
                            return false;
                        });
}

/* size (gpu_engine.cuh:419-464): non-empty values of slots with a valid key */
template <class K, class V>
__global__ void __launch_bounds__(256) mb_size_kernel(const MbView m, uint64_t capacity,
                                                      unsigned long long *count)
{
    const K empty = K(m.t.empty_key), tomb = K(m.t.tombstone_key);
    const V ev = V(m.empty_value);
    const K *const keys = reinterpret_cast<const K *>(m.t.slots);
    const V *const vals = reinterpret_cast<const V *>(m.vals);
    unsigned long long c = 0;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < capacity; i += stride) {
        const K k = keys[i];
        if (k == empty || k == tomb) continue;
        for (uint32_t r = 0; r < m.bucket; ++r) c += vals[i * m.bucket + r] != ev;
    }
    const unsigned s = __reduce_add_sync(0xffffffffu, unsigned(c));
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(count, (unsigned long long)s);
}

struct MbKernels {
    const void *insert, *count, *values, *unique, *size;
};

template <class K, class V, int kW, int kB>
MbKernels mb_kernels_of()
{
    return {reinterpret_cast<const void *>(mb_insert_kernel<K, V, kW, kB>),
            reinterpret_cast<const void *>(mb_find_kernel<K, V, kW, kB, false>),
            reinterpret_cast<const void *>(mb_find_kernel<K, V, kW, kB, true>),
            reinterpret_cast<const void *>(mb_unique_keys_kernel<K>),
            reinterpret_cast<const void *>(mb_size_kernel<K, V>)};
}

/* CG 8 (the reference's default) with buckets of 1, 2, 4 or 8 runs kernels
 * built for that shape; every other shape runs the run-time ones */
template <class K, class V>
MbKernels mb_kernels_kv(uint32_t cg, uint32_t bucket)
{
    if (cg == 8) {
        switch (bucket) {
        case 1: return mb_kernels_of<K, V, 8, 1>();
        case 2: return mb_kernels_of<K, V, 8, 2>();
        case 4: return mb_kernels_of<K, V, 8, 4>();
        case 8: return mb_kernels_of<K, V, 8, 8>();
        default: break;
        }
    }
    return mb_kernels_of<K, V, 0, 0>();
}

MbKernels mb_kernels(const wc_mbht *t)
{
    using U32 = unsigned int;
    using U64 = unsigned long long;
    const uint32_t cg = t->cfg.cg_size, b = t->bucket;
    if (t->cfg.key_bytes == 4)
        return t->cfg.value_bytes == 4 ? mb_kernels_kv<U32, U32>(cg, b) : mb_kernels_kv<U32, U64>(cg, b);
    return t->cfg.value_bytes == 4 ? mb_kernels_kv<U64, U32>(cg, b) : mb_kernels_kv<U64, U64>(cg, b);
}

MbView view_of(const wc_mbht *t)
{
    MbView m{};
    TableView &v = m.t;
    v.slots = t->keys;
    v.status = t->status;
    v.fps = nullptr;
    v.num_buckets = t->num_buckets;
    v.seed = t->seed;
    v.empty_key = t->cfg.empty_key;
    v.tombstone_key = t->cfg.tombstone_key;
    v.max_count = ~0ull;
    v.magic_nb = barrett_magic(t->num_buckets);
    v.magic_nb1 = barrett_magic(t->num_buckets > 1 ? t->num_buckets - 1 : 1);
    v.probing = t->cfg.probing;
    v.hasher1 = t->cfg.hasher1;
    v.hasher2 = t->cfg.hasher2;
    v.cg_size = t->cfg.cg_size;
    m.vals = t->vals;
    m.empty_value = t->empty_value;
    m.max_values = t->max_values;
    m.bucket = t->bucket;
    m.num_keys = t->counters;
    m.num_occupied = t->counters + 1;
    return m;
}

int check(const wc_mbht *t)
{
    if (!t) return mb_fail(WC_ERR_INVALID_ARGUMENT, "table is NULL");
    if (!t->initialized) return mb_fail(WC_ERR_NOT_INITIALIZED, "table is not initialized");
    return WC_OK;
}

MbArgs args_of(const wc_mbht *t, const void *keys, uint64_t n, uint64_t probing_length, bool find,
               void *status_out, int handler, uint32_t ignore)
{
    MbArgs a{};
    a.m = view_of(t);
    a.keys = keys;
    a.n = n;
    /* for_each caps the probing length at the capacity (:802) */
    const uint64_t pl = find && probing_length > t->capacity ? t->capacity : probing_length;
    a.max_windows = max_windows(pl, t->cfg.cg_size, t->num_buckets);
    a.status_out = handler == WC_HANDLER_NOTHING ? nullptr : status_out;
    a.handler = handler;
    a.bool_mask = (~ignore) ^ 0xFFFu; /* ~Status(Ignore), status.cuh:142-146 */
    return a;
}

int launch(const void *k, uint64_t items, MbArgs &a, cudaStream_t s)
{
    void *args[] = {&a};
    MB_CUDA(cudaLaunchKernel(k, dim3(host_grid(k, kBlock, items, kBlock)), dim3(kBlock), args, 0, s));
    note_launches(1);
    return WC_OK;
}

int read_counter(const unsigned long long *d, cudaStream_t s, uint64_t *out)
{
    return host_read_counter(d, s, out);
}

/* per-key counts (and their sum, read back) */
int count(wc_mbht *t, const void *keys, uint64_t n, uint64_t *counts_dev, uint64_t *total,
          cudaStream_t s, uint64_t probing_length, void *status_out, int handler, uint32_t ignore)
{
    unsigned long long *tmp = t->counters + 2;
    MB_CUDA(cudaMemsetAsync(tmp, 0, sizeof(unsigned long long), s));
    MbArgs a = args_of(t, keys, n, probing_length, true, status_out, handler, ignore);
    a.counts_out = reinterpret_cast<unsigned long long *>(counts_dev);
    a.total = tmp;
    int rc = launch(mb_kernels(t).count, n, a, s);
    if (rc) return rc;
    return read_counter(tmp, s, total);
}

/* counts in end -> end = inclusive prefix sums, begin = exclusive ones */
int scan(wc_mbht *t, uint64_t *begin, uint64_t *end, uint64_t n, cudaStream_t s)
{
    return host_offsets_scan(&t->scan, &t->scan_bytes, begin, end, n, s);
}

/* host join of status bits into the table's Status word */
int join_host(wc_mbht *t, uint32_t bits, cudaStream_t s)
{
    return host_join_status(t->status, bits, s);
}

/* fill `bytes` (a multiple of 4) with a repeated 4- or 8-byte word */
int fill(void *p, uint64_t bytes, uint64_t word, uint32_t word_bytes, cudaStream_t s)
{
    uint32_t w[4];
    if (word_bytes == 4) {
        w[0] = w[1] = w[2] = w[3] = uint32_t(word);
    } else {
        w[0] = w[2] = uint32_t(word);
        w[1] = w[3] = uint32_t(word >> 32);
    }
    uint4 pat = make_uint4(w[0], w[1], w[2], w[3]);
    uint32_t *dst = reinterpret_cast<uint32_t *>(p);
    uint64_t n = bytes / 4;
    const void *kfn = reinterpret_cast<const void *>(fill_kernel<0>);
    void *args[] = {&dst, &n, &pat};
    MB_CUDA(cudaLaunchKernel(kfn, dim3(host_grid(kfn, kBlock, n / 4, kBlock)), dim3(kBlock), args, 0,
                             s));
    note_launches(1);
    return WC_OK;
}

} // namespace

extern "C" {

int wc_mbht_create(const wc_table_config *cfg, uint32_t bucket_size, uint64_t empty_value,
                   uint64_t min_capacity, uint64_t seed, uint64_t max_values_per_key, int no_init,
                   wc_mbht **out)
{
    if (!out) return mb_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!cfg) return mb_fail(WC_ERR_INVALID_ARGUMENT, "config is NULL");
    if (cfg->key_bytes != 4 && cfg->key_bytes != 8)
        return mb_fail(WC_ERR_UNSUPPORTED, "key_bytes must be 4 or 8");
    if (cfg->value_bytes != 4 && cfg->value_bytes != 8)
        return mb_fail(WC_ERR_UNSUPPORTED, "value_bytes must be 4 or 8");
    const uint32_t cg = cfg->cg_size;
    if (!(cg == 1 || cg == 2 || cg == 4 || cg == 8 || cg == 16 || cg == 32))
        return mb_fail(WC_ERR_INVALID_ARGUMENT, "cg_size must be 1, 2, 4, 8, 16 or 32");
    if (bucket_size == 0 || bucket_size > cg)
        return mb_fail(WC_ERR_UNSUPPORTED, "bucket_size must be 1 .. cg_size");
    if (cfg->probing > WC_PROBING_QUADRATIC || cfg->hasher1 > WC_HASH_IDENTITY64 ||
        cfg->hasher2 > WC_HASH_IDENTITY64)
        return mb_fail(WC_ERR_INVALID_ARGUMENT, "unknown probing scheme or hasher");
    const uint64_t km = kmask(cfg->key_bytes);
    if ((cfg->empty_key & km) == (cfg->tombstone_key & km))
        return mb_fail(WC_ERR_INVALID_ARGUMENT, "empty key and tombstone key must differ");
    const uint64_t cap = host_valid_capacity(min_capacity, cg);
    if (cap == 0) return mb_fail(WC_ERR_INVALID_ARGUMENT, "min_capacity exceeds the largest capacity");
    auto *t = new wc_mbht();
    t->cfg = *cfg;
    t->cfg.empty_key &= km;
    t->cfg.tombstone_key &= km;
    t->bucket = bucket_size;
    t->empty_value = empty_value & kmask(cfg->value_bytes);
    t->capacity = cap;
    t->num_buckets = cap / cg;
    t->seed = seed & km;
    t->max_values = max_values_per_key;
    const uint64_t kbytes = (cap * cfg->key_bytes + 255) & ~uint64_t(255);
    const uint64_t vbytes = cap * bucket_size * cfg->value_bytes;
    cudaError_t e = cudaMalloc(&t->keys, kbytes + vbytes);
    if (e == cudaSuccess) e = cudaMalloc(&t->status, 256);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (t->keys) cudaFree(t->keys);
        delete t;
        return host_cuda_fail(e, "cudaMalloc (multi-bucket table)");
    }
    t->vals = static_cast<char *>(t->keys) + kbytes;
    t->counters = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(t->status) + 64);
    *out = t;
    if (!no_init) {
        const int rc = wc_mbht_init(t, nullptr);
        if (rc) {
            wc_mbht_destroy(t);
            *out = nullptr;
            return rc;
        }
    }
    return WC_OK;
}

int wc_mbht_destroy(wc_mbht *t)
{
    if (!t) return WC_OK;
    if (t->keys) cudaFree(t->keys);
    if (t->status) cudaFree(t->status);
    if (t->scan) cudaFree(t->scan);
    delete t;
    return WC_OK;
}

int wc_mbht_init(wc_mbht *t, wc_stream_t stream)
{
    if (!t) return mb_fail(WC_ERR_INVALID_ARGUMENT, "table is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int rc = fill(t->keys, t->capacity * t->cfg.key_bytes, t->cfg.empty_key, t->cfg.key_bytes, s);
    if (rc) return rc;
    rc = fill(t->vals, t->capacity * t->bucket * t->cfg.value_bytes, t->empty_value,
              t->cfg.value_bytes, s);
    if (rc) return rc;
    MB_CUDA(cudaMemsetAsync(t->status, 0, 256, s));
    MB_CUDA(cudaStreamSynchronize(s));
    t->initialized = true;
    return WC_OK;
}

int wc_mbht_insert(wc_mbht *t, const void *keys_in, const void *values_in, uint64_t num_in,
                   wc_stream_t stream, uint64_t probing_length, void *status_out,
                   int status_handler, uint32_t ignore)
{
    int rc = check(t);
    if (rc) return rc;
    if (status_handler < WC_HANDLER_NOTHING || status_handler > WC_HANDLER_BOOLEAN)
        return mb_fail(WC_ERR_INVALID_ARGUMENT, "unknown status handler");
    if (num_in == 0) return WC_OK;
    if (!keys_in || !values_in) return mb_fail(WC_ERR_INVALID_ARGUMENT, "keys_in / values_in is NULL");
    MbArgs a = args_of(t, keys_in, num_in, probing_length, false, status_out, status_handler, ignore);
    a.values = values_in;
    return launch(mb_kernels(t).insert, num_in, a, reinterpret_cast<cudaStream_t>(stream));
}

int wc_mbht_num_values(wc_mbht *t, const void *keys_in, uint64_t num_in, uint64_t *num_out,
                       uint64_t *num_per_key_out, wc_stream_t stream, uint64_t probing_length,
                       void *status_out, int status_handler, uint32_t ignore)
{
    int rc = check(t);
    if (rc) return rc;
    if (!num_out) return mb_fail(WC_ERR_INVALID_ARGUMENT, "num_out is NULL");
    *num_out = 0;
    if (num_in == 0) return WC_OK;
    if (!keys_in) return mb_fail(WC_ERR_INVALID_ARGUMENT, "keys_in is NULL");
    return count(t, keys_in, num_in, num_per_key_out, num_out,
                 reinterpret_cast<cudaStream_t>(stream), probing_length, status_out,
                 status_handler, ignore);
}

int wc_mbht_retrieve(wc_mbht *t, const void *keys_in, uint64_t num_in,
                     uint64_t *begin_offsets_out, uint64_t *end_offsets_out, void *values_out,
                     uint64_t *num_out, wc_stream_t stream, uint64_t probing_length,
                     void *status_out, int status_handler, uint32_t ignore)
{
    int rc = check(t);
    if (rc) return rc;
    if (!num_out) return mb_fail(WC_ERR_INVALID_ARGUMENT, "num_out is NULL");
    *num_out = 0;
    if (num_in == 0) return WC_OK;
    if (!keys_in || !end_offsets_out || (values_out && !begin_offsets_out))
        return mb_fail(WC_ERR_INVALID_ARGUMENT, "NULL buffer");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    /* pass 1: counts per key into end_offsets, and each key's status (the
     * values pass reads values only) */
    rc = count(t, keys_in, num_in, end_offsets_out, num_out, s, probing_length,
               values_out ? status_out : nullptr, values_out ? status_handler : WC_HANDLER_NOTHING,
               ignore);
    if (rc) return rc;
    if (!values_out) {
        /* dry run: per-key counts, status dry_run for every key */
        rc = host_dry_run_status(status_out, num_in, status_handler, ignore, s);
        if (rc) return rc;
        return join_host(t, kStDryRun, s);
    }
    /* pass 2: offsets; pass 3: values at each key's begin offset */
    rc = scan(t, begin_offsets_out, end_offsets_out, num_in, s);
    if (rc) return rc;
    MbArgs a = args_of(t, keys_in, num_in, probing_length, true, status_out, status_handler, ignore);
    a.values_out = values_out;
    a.begin = reinterpret_cast<const unsigned long long *>(begin_offsets_out);
    a.end = reinterpret_cast<const unsigned long long *>(end_offsets_out);
    return launch(mb_kernels(t).values, num_in, a, s);
}

int wc_mbht_retrieve_all_keys(wc_mbht *t, void *keys_out, uint64_t *num_out, wc_stream_t stream)
{
    int rc = check(t);
    if (rc) return rc;
    if (!num_out) return mb_fail(WC_ERR_INVALID_ARGUMENT, "num_out is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!keys_out) {
        rc = read_counter(t->counters, s, num_out);
        if (rc) return rc;
        return join_host(t, kStDryRun, s);
    }
    unsigned long long *tmp = t->counters + 2;
    MB_CUDA(cudaMemsetAsync(tmp, 0, sizeof(unsigned long long), s));
    MbView v = view_of(t);
    uint64_t cap = t->capacity;
    const MbKernels k = mb_kernels(t);
    void *args[] = {&v, &cap, &keys_out, &tmp};
    MB_CUDA(cudaLaunchKernel(k.unique, dim3(host_grid(k.unique, kBlock, cap, kBlock)), dim3(kBlock),
                             args, 0, s));
    note_launches(1);
    return read_counter(tmp, s, num_out);
}

int wc_mbht_num_keys(wc_mbht *t, wc_stream_t stream, uint64_t *out)
{
    int rc = check(t);
    if (rc) return rc;
    if (!out) return mb_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    return read_counter(t->counters, reinterpret_cast<cudaStream_t>(stream), out);
}

int wc_mbht_num_occupied(wc_mbht *t, wc_stream_t stream, uint64_t *out)
{
    int rc = check(t);
    if (rc) return rc;
    if (!out) return mb_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    return read_counter(t->counters + 1, reinterpret_cast<cudaStream_t>(stream), out);
}

int wc_mbht_size(wc_mbht *t, wc_stream_t stream, uint64_t *out)
{
    int rc = check(t);
    if (rc) return rc;
    if (!out) return mb_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    unsigned long long *tmp = t->counters + 2;
    MB_CUDA(cudaMemsetAsync(tmp, 0, sizeof(unsigned long long), s));
    MbView v = view_of(t);
    uint64_t cap = t->capacity;
    const MbKernels k = mb_kernels(t);
    void *args[] = {&v, &cap, &tmp};
    MB_CUDA(cudaLaunchKernel(k.size, dim3(host_grid(k.size, kBlock, cap, kBlock)), dim3(kBlock), args,
                             0, s));
    note_launches(1);
    return read_counter(tmp, s, out);
}

int wc_mbht_peek_status(wc_mbht *t, wc_stream_t stream, uint32_t *out)
{
    if (!t || !out) return mb_fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    MB_CUDA(cudaMemcpyAsync(out, t->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    return WC_OK;
}

int wc_mbht_pop_status(wc_mbht *t, wc_stream_t stream, uint32_t *out)
{
    int rc = wc_mbht_peek_status(t, stream, out);
    if (rc) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    MB_CUDA(cudaMemsetAsync(t->status, 0, sizeof(uint32_t), s));
    MB_CUDA(cudaStreamSynchronize(s));
    return WC_OK;
}

int wc_mbht_get_info(const wc_mbht *t, wc_mbht_info *info)
{
    if (!t || !info) return mb_fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memset(info, 0, sizeof(*info));
    info->key_bytes = t->cfg.key_bytes;
    info->value_bytes = t->cfg.value_bytes;
    info->bucket_size = t->bucket;
    info->cg_size = t->cfg.cg_size;
    info->probing = t->cfg.probing;
    info->hasher1 = t->cfg.hasher1;
    info->hasher2 = t->cfg.hasher2;
    info->capacity = t->capacity;
    info->value_capacity = t->capacity * t->bucket;
    info->num_buckets = t->num_buckets;
    info->seed = t->seed;
    info->empty_key = t->cfg.empty_key;
    info->tombstone_key = t->cfg.tombstone_key;
    info->empty_value = t->empty_value;
    info->max_values_per_key = t->max_values;
    info->bytes_total = t->capacity * (t->cfg.key_bytes + uint64_t(t->bucket) * t->cfg.value_bytes) +
                        sizeof(uint64_t);
    info->keys = t->keys;
    info->values = t->vals;
    info->status = t->status;
    info->num_keys = t->counters;
    info->num_occupied = t->counters + 1;
    info->is_initialized = t->initialized ? 1 : 0;
    return WC_OK;
}

} // extern "C"
