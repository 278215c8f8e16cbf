/*
 * wc_bucketlist.cu -- BucketListHashTable (the reference's
 * bucket_list_hash_table.cuh over BucketListStore, storage.cuh:651-1454):
 * kernels and the wc_blht_* C ABI.
 *
 * Layout: keys, handles (one 64-bit list handle per key slot) and the
 * value pool are three arrays; the reference keeps {key, handle} pairs and
 * a pool of value/header unions.  Every kernel runs one key per lane
 * (detail/bl_ops.cuh): the key's window, then its handle, then its list.
 */
#include <warpcore_b200.h>

#include "wc_internal.h"
#include "wc_compact.cuh"
#include <warpcore/detail/bl_ops.cuh>

#include <cstring>

using namespace warpcore::b200;

struct wc_blht {
    wc_table_config cfg{};
    uint64_t capacity = 0, num_buckets = 0, seed = 0;
    uint64_t value_capacity = 0, min_bucket = 1, max_bucket = 1, max_values = 1;
    float grow = 1.1f;
    uint32_t ib = 32, cb = 20, sb = 10;
    void *keys = nullptr;
    unsigned long long *handles = nullptr;
    unsigned long long *pool = nullptr;
    uint32_t *status = nullptr;             /* device Status word */
    unsigned long long *counters = nullptr; /* device: next free pool element, scratch */
    void *scan = nullptr;
    uint64_t scan_bytes = 0;
    bool initialized = false;
};

namespace {

#define BL_CUDA(call)                                                          \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) return host_cuda_fail(e_, #call);               \
    } while (0)

constexpr int kBlock = 256;

int bl_fail(int code, const char *msg) { return host_fail(code, msg); }

uint64_t kmask(uint32_t bytes) { return bytes == 4 ? 0xffffffffull : ~0ull; }

struct BlArgs {
    BlView v;
    const void *keys;
    const void *values;              /* insert */
    void *values_out;                /* retrieve */
    const unsigned long long *begin;
    const unsigned long long *end;
    unsigned long long *counts_out;
    unsigned long long *total;
    void *status_out;
    uint64_t n;
    uint64_t max_windows;
    uint32_t bool_mask;
    int handler;
};

__device__ __forceinline__ void bl_write_status(const BlArgs &a, uint64_t i, uint32_t st)
{
    if (!a.status_out) return;
    if (a.handler == kHandlerStatus)
        reinterpret_cast<uint32_t *>(a.status_out)[i] = st;
    else if (a.handler == kHandlerBoolean)
        reinterpret_cast<unsigned char *>(a.status_out)[i] = (unsigned char)((st & a.bool_mask) != 0);
}

/* bulk insert (:235-326).  Unlike the reference kernel, which leaves the
 * status of a key without a slot (invalid key, probing length exceeded)
 * unwritten, every key gets its status. */
template <class K, class V, int kW>
__global__ void __launch_bounds__(256, WC_MULTI_MIN_BLOCKS) bl_insert_kernel(const BlArgs a)
{
    uint32_t join = 0;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        uint32_t j = 0;
        const uint32_t st = bl_insert_one<K, V, kW>(a.v, reinterpret_cast<const K *>(a.keys)[i],
                                                    reinterpret_cast<const V *>(a.values)[i],
                                                    a.max_windows, j);
        join |= j;
        bl_write_status(a, i, st);
    }
    const uint32_t wj = __reduce_or_sync(0xffffffffu, join); /* every lane arrives */
    if ((threadIdx.x & 31) == 0) join_status(a.v.t.status, wj);
}

/* num_values (kValues false) or retrieve (gpu_engine.cuh:305-346) */
template <class K, class V, int kW, bool kValues>
__global__ void __launch_bounds__(256, WC_MULTI_MIN_BLOCKS) bl_find_kernel(const BlArgs a)
{
    uint32_t join = 0;
    unsigned long long total = 0;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        uint64_t num = 0;
        const K key = reinterpret_cast<const K *>(a.keys)[i];
        if constexpr (kValues) {
            /* The counting pass looked every key up and wrote its status;
             * this pass only reads lists.  A key counted at 0 needs no
             * lookup.  Values go inside the key's own segment only. */
            const uint64_t room = a.end[i] - a.begin[i];
            if (room == 0) continue;
            V *const out = reinterpret_cast<V *>(a.values_out) + a.begin[i];
            bl_for_each_one<K, V, kW, true>(a.v, key, a.max_windows, num, [&](V x, uint64_t j) {
                if (j < room) out[j] = x;
            });
        } else {
            const uint32_t st = bl_for_each_one<K, V, kW, false>(a.v, key, a.max_windows, num,
                                                                 [](V, uint64_t) {});
            join |= st;
            if (a.counts_out) a.counts_out[i] = num;
            total += num;
            bl_write_status(a, i, st);
        }
    }
    const uint32_t wj = __reduce_or_sync(0xffffffffu, join);
    const unsigned long long sum = warp_sum_u64(total);
    if ((threadIdx.x & 31) == 0) {
        if (a.total && sum) atomicAdd(a.total, sum);
        join_status(a.v.t.status, wj);
    }
}

/* init: keys empty, handles uninitialized, pool headers {head, min}, next free 0 */
template <class K>
__global__ void __launch_bounds__(256) bl_init_kernel(const BlView v, uint64_t capacity)
{
    const unsigned long long u = bl_pack(v, kBlUninit, bl_head(v.ib), 0, 0);
    const unsigned long long hdr = bl_header(v, bl_head(v.ib), v.min_bucket);
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t tid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    for (uint64_t i = tid; i < capacity; i += stride) {
        reinterpret_cast<K *>(v.t.slots)[i] = K(v.t.empty_key);
        v.handles[i] = u;
    }
    for (uint64_t i = tid; i < v.capacity; i += stride) v.pool[i] = hdr;
    if (tid == 0) *v.next_free = 0;
}

/* num_keys (valid keys), num_values (sum of list counts) and the keys,
 * compacted by block tiles (wc_compact.cuh) */
template <class K>
__global__ void __launch_bounds__(256) bl_scan_keys_kernel(const BlView v, uint64_t capacity,
                                                           void *keys_out,
                                                           unsigned long long *num_keys,
                                                           unsigned long long *num_values)
{
    const K empty = K(v.t.empty_key), tomb = K(v.t.tombstone_key);
    const K *const keys = reinterpret_cast<const K *>(v.t.slots);
    unsigned long long vals = 0;
    compact_tiles<K, K>(capacity, reinterpret_cast<K *>(keys_out), nullptr, num_keys,
                        [&](uint64_t i, K &k, K &) {
                            k = keys[i];
                            if (k == empty || k == tomb) return false;
                            vals += bl_unpack(v, v.handles[i]).count;
                            return true;
                        });
    vals = warp_sum_u64(vals);
    if ((threadIdx.x & 31) == 0 && vals) atomicAdd(num_values, vals);
}

struct BlKernels {
    const void *insert, *count, *values, *init, *scan;
};

template <class K, class V, int kW>
BlKernels bl_kernels_of()
{
    return {reinterpret_cast<const void *>(bl_insert_kernel<K, V, kW>),
            reinterpret_cast<const void *>(bl_find_kernel<K, V, kW, false>),
            reinterpret_cast<const void *>(bl_find_kernel<K, V, kW, true>),
            reinterpret_cast<const void *>(bl_init_kernel<K>),
            reinterpret_cast<const void *>(bl_scan_keys_kernel<K>)};
}

template <class K, class V>
BlKernels bl_kernels_kv(uint32_t cg)
{
    return cg == 8 ? bl_kernels_of<K, V, 8>() : bl_kernels_of<K, V, 0>();
}

BlKernels bl_kernels(const wc_blht *t)
{
    using U32 = unsigned int;
    using U64 = unsigned long long;
    const uint32_t cg = t->cfg.cg_size;
    if (t->cfg.key_bytes == 4)
        return t->cfg.value_bytes == 4 ? bl_kernels_kv<U32, U32>(cg) : bl_kernels_kv<U32, U64>(cg);
    return t->cfg.value_bytes == 4 ? bl_kernels_kv<U64, U32>(cg) : bl_kernels_kv<U64, U64>(cg);
}

BlView view_of(const wc_blht *t)
{
    BlView v{};
    TableView &tv = v.t;
    tv.slots = t->keys;
    tv.status = t->status;
    tv.fps = nullptr;
    tv.num_buckets = t->num_buckets;
    tv.seed = t->seed;
    tv.empty_key = t->cfg.empty_key;
    tv.tombstone_key = t->cfg.tombstone_key;
    tv.max_count = ~0ull;
    tv.magic_nb = barrett_magic(t->num_buckets);
    tv.magic_nb1 = barrett_magic(t->num_buckets > 1 ? t->num_buckets - 1 : 1);
    tv.probing = t->cfg.probing;
    tv.hasher1 = t->cfg.hasher1;
    tv.hasher2 = t->cfg.hasher2;
    tv.cg_size = t->cfg.cg_size;
    v.handles = t->handles;
    v.pool = t->pool;
    v.next_free = t->counters;
    v.capacity = t->value_capacity;
    v.min_bucket = t->min_bucket;
    v.max_bucket = t->max_bucket;
    v.max_values = t->max_values;
    v.grow = t->grow;
    v.ib = t->ib;
    v.cb = t->cb;
    v.sb = t->sb;
    return v;
}

int check(const wc_blht *t)
{
    if (!t) return bl_fail(WC_ERR_INVALID_ARGUMENT, "table is NULL");
    if (!t->initialized) return bl_fail(WC_ERR_NOT_INITIALIZED, "table is not initialized");
    return WC_OK;
}

BlArgs args_of(const wc_blht *t, const void *keys, uint64_t n, uint64_t probing_length,
               void *status_out, int handler, uint32_t ignore)
{
    BlArgs a{};
    a.v = view_of(t);
    a.keys = keys;
    a.n = n;
    a.max_windows = max_windows(probing_length, t->cfg.cg_size, t->num_buckets);
    a.status_out = handler == WC_HANDLER_NOTHING ? nullptr : status_out;
    a.handler = handler;
    a.bool_mask = (~ignore) ^ 0xFFFu;
    return a;
}

int launch(const void *k, uint64_t items, BlArgs &a, cudaStream_t s)
{
    void *args[] = {&a};
    BL_CUDA(cudaLaunchKernel(k, dim3(host_grid(k, kBlock, items, kBlock)), dim3(kBlock), args, 0, s));
    note_launches(1);
    return WC_OK;
}

int read_counter(const unsigned long long *d, cudaStream_t s, uint64_t *out)
{
    return host_read_counter(d, s, out);
}

int count(wc_blht *t, const void *keys, uint64_t n, uint64_t *counts_dev, uint64_t *total,
          cudaStream_t s, uint64_t probing_length, void *status_out, int handler, uint32_t ignore)
{
    unsigned long long *tmp = t->counters + 1;
    BL_CUDA(cudaMemsetAsync(tmp, 0, sizeof(unsigned long long), s));
    BlArgs a = args_of(t, keys, n, probing_length, status_out, handler, ignore);
    a.counts_out = reinterpret_cast<unsigned long long *>(counts_dev);
    a.total = tmp;
    int rc = launch(bl_kernels(t).count, n, a, s);
    if (rc) return rc;
    return read_counter(tmp, s, total);
}

int scan(wc_blht *t, uint64_t *begin, uint64_t *end, uint64_t n, cudaStream_t s)
{
    return host_offsets_scan(&t->scan, &t->scan_bytes, begin, end, n, s);
}

int join_host(wc_blht *t, uint32_t bits, cudaStream_t s)
{
    return host_join_status(t->status, bits, s);
}

/* valid keys (into keys_out if not NULL) and the sum of their list counts */
int scan_keys(wc_blht *t, void *keys_out, uint64_t *num_keys, uint64_t *num_values,
              cudaStream_t s)
{
    unsigned long long *nk = t->counters + 2, *nv = t->counters + 3;
    BL_CUDA(cudaMemsetAsync(nk, 0, 2 * sizeof(unsigned long long), s));
    BlView v = view_of(t);
    uint64_t cap = t->capacity;
    const void *k = bl_kernels(t).scan;
    void *args[] = {&v, &cap, &keys_out, &nk, &nv};
    BL_CUDA(cudaLaunchKernel(k, dim3(host_grid(k, kBlock, cap, kBlock)), dim3(kBlock), args, 0, s));
    note_launches(1);
    unsigned long long h[2] = {0, 0};
    BL_CUDA(cudaMemcpyAsync(h, nk, sizeof(h), cudaMemcpyDeviceToHost, s));
    BL_CUDA(cudaStreamSynchronize(s));
    if (num_keys) *num_keys = h[0];
    if (num_values) *num_values = h[1];
    return WC_OK;
}

} // namespace

extern "C" {

int wc_blht_create(const wc_table_config *cfg, uint64_t key_capacity, uint64_t value_capacity,
                   uint64_t seed, float grow_factor, uint64_t min_bucket_size,
                   uint64_t max_bucket_size, uint64_t max_values_per_key, uint32_t index_bits,
                   uint32_t counter_bits, uint32_t size_bits, int no_init, wc_blht **out)
{
    if (!out) return bl_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!cfg) return bl_fail(WC_ERR_INVALID_ARGUMENT, "config is NULL");
    if (cfg->key_bytes != 4 && cfg->key_bytes != 8)
        return bl_fail(WC_ERR_UNSUPPORTED, "key_bytes must be 4 or 8");
    if (cfg->value_bytes != 4 && cfg->value_bytes != 8)
        return bl_fail(WC_ERR_UNSUPPORTED, "value_bytes must be 4 or 8");
    const uint32_t cg = cfg->cg_size;
    if (!(cg == 1 || cg == 2 || cg == 4 || cg == 8 || cg == 16 || cg == 32))
        return bl_fail(WC_ERR_INVALID_ARGUMENT, "cg_size must be 1, 2, 4, 8, 16 or 32");
    if (cfg->probing > WC_PROBING_QUADRATIC || cfg->hasher1 > WC_HASH_IDENTITY64 ||
        cfg->hasher2 > WC_HASH_IDENTITY64)
        return bl_fail(WC_ERR_INVALID_ARGUMENT, "unknown probing scheme or hasher");
    const uint64_t km = kmask(cfg->key_bytes);
    if ((cfg->empty_key & km) == (cfg->tombstone_key & km))
        return bl_fail(WC_ERR_INVALID_ARGUMENT, "empty key and tombstone key must differ");
    if (index_bits == 0 || counter_bits == 0 || size_bits == 0 ||
        uint64_t(index_bits) + counter_bits + size_bits + 2 > 64 || index_bits + size_bits > 64)
        return bl_fail(WC_ERR_INVALID_ARGUMENT, "bit widths must be positive and fit in 62 bits");
    /* the store's configuration check (storage.cuh:990-1014) */
    const uint64_t head = (1ull << index_bits) - 1, max_size = (1ull << size_bits) - 1;
    if (!(value_capacity < head && grow_factor >= 1.0f && min_bucket_size >= 1 &&
          max_bucket_size >= min_bucket_size && max_bucket_size <= max_size))
        return bl_fail(WC_ERR_INVALID_ARGUMENT,
                       "invalid bucket list configuration (value capacity, grow factor, bucket sizes)");
    const uint64_t cap = host_valid_capacity(key_capacity, cg);
    if (cap == 0) return bl_fail(WC_ERR_INVALID_ARGUMENT, "key_capacity exceeds the largest capacity");
    auto *t = new wc_blht();
    t->cfg = *cfg;
    t->cfg.empty_key &= km;
    t->cfg.tombstone_key &= km;
    t->capacity = cap;
    t->num_buckets = cap / cg;
    t->seed = seed & km;
    t->value_capacity = value_capacity;
    t->grow = grow_factor;
    t->min_bucket = min_bucket_size;
    t->max_bucket = max_bucket_size;
    const uint64_t max_count = (1ull << counter_bits) - 1;
    t->max_values = max_values_per_key < max_count ? max_values_per_key : max_count;
    t->ib = index_bits;
    t->cb = counter_bits;
    t->sb = size_bits;
    const uint64_t kbytes = (cap * cfg->key_bytes + 255) & ~uint64_t(255);
    const uint64_t hbytes = cap * 8;
    const uint64_t pbytes = (value_capacity ? value_capacity : 1) * 8;
    void *mem = nullptr;
    cudaError_t e = cudaMalloc(&mem, kbytes + hbytes + pbytes);
    if (e == cudaSuccess) e = cudaMalloc(&t->status, 256);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (mem) cudaFree(mem);
        delete t;
        return host_cuda_fail(e, "cudaMalloc (bucket list table)");
    }
    t->keys = mem;
    t->handles = reinterpret_cast<unsigned long long *>(static_cast<char *>(mem) + kbytes);
    t->pool = reinterpret_cast<unsigned long long *>(static_cast<char *>(mem) + kbytes + hbytes);
    t->counters = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(t->status) + 64);
    *out = t;
    if (!no_init) {
        const int rc = wc_blht_init(t, t->seed, nullptr);
        if (rc) {
            wc_blht_destroy(t);
            *out = nullptr;
            return rc;
        }
    }
    return WC_OK;
}

int wc_blht_destroy(wc_blht *t)
{
    if (!t) return WC_OK;
    if (t->keys) cudaFree(t->keys);
    if (t->status) cudaFree(t->status);
    if (t->scan) cudaFree(t->scan);
    delete t;
    return WC_OK;
}

int wc_blht_init(wc_blht *t, uint64_t seed, wc_stream_t stream)
{
    if (!t) return bl_fail(WC_ERR_INVALID_ARGUMENT, "table is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    t->seed = seed & kmask(t->cfg.key_bytes);
    BL_CUDA(cudaMemsetAsync(t->status, 0, 256, s));
    BlView v = view_of(t);
    uint64_t cap = t->capacity;
    const void *k = bl_kernels(t).init;
    const uint64_t items = cap > t->value_capacity ? cap : t->value_capacity;
    void *args[] = {&v, &cap};
    BL_CUDA(cudaLaunchKernel(k, dim3(host_grid(k, kBlock, items, kBlock)), dim3(kBlock), args, 0, s));
    note_launches(1);
    BL_CUDA(cudaStreamSynchronize(s));
    t->initialized = true;
    return WC_OK;
}

int wc_blht_insert(wc_blht *t, const void *keys_in, const void *values_in, uint64_t num_in,
                   wc_stream_t stream, uint64_t probing_length, void *status_out,
                   int status_handler, uint32_t ignore)
{
    int rc = check(t);
    if (rc) return rc;
    if (status_handler < WC_HANDLER_NOTHING || status_handler > WC_HANDLER_BOOLEAN)
        return bl_fail(WC_ERR_INVALID_ARGUMENT, "unknown status handler");
    if (num_in == 0) return WC_OK;
    if (!keys_in || !values_in) return bl_fail(WC_ERR_INVALID_ARGUMENT, "keys_in / values_in is NULL");
    BlArgs a = args_of(t, keys_in, num_in, probing_length, status_out, status_handler, ignore);
    a.values = values_in;
    return launch(bl_kernels(t).insert, num_in, a, reinterpret_cast<cudaStream_t>(stream));
}

int wc_blht_num_values(wc_blht *t, const void *keys_in, uint64_t num_in, uint64_t *num_out,
                       uint64_t *num_per_key_out, wc_stream_t stream, uint64_t probing_length,
                       void *status_out, int status_handler, uint32_t ignore)
{
    int rc = check(t);
    if (rc) return rc;
    if (!num_out) return bl_fail(WC_ERR_INVALID_ARGUMENT, "num_out is NULL");
    *num_out = 0;
    if (num_in == 0) return WC_OK;
    if (!keys_in) return bl_fail(WC_ERR_INVALID_ARGUMENT, "keys_in is NULL");
    return count(t, keys_in, num_in, num_per_key_out, num_out,
                 reinterpret_cast<cudaStream_t>(stream), probing_length, status_out,
                 status_handler, ignore);
}

int wc_blht_retrieve(wc_blht *t, const void *keys_in, uint64_t num_in,
                     uint64_t *begin_offsets_out, uint64_t *end_offsets_out, void *values_out,
                     uint64_t *num_out, wc_stream_t stream, uint64_t probing_length,
                     void *status_out, int status_handler, uint32_t ignore)
{
    int rc = check(t);
    if (rc) return rc;
    if (!num_out) return bl_fail(WC_ERR_INVALID_ARGUMENT, "num_out is NULL");
    *num_out = 0;
    if (num_in == 0) return WC_OK;
    if (!keys_in || !end_offsets_out || (values_out && !begin_offsets_out))
        return bl_fail(WC_ERR_INVALID_ARGUMENT, "NULL buffer");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    /* pass 1: counts, and each key's status (the values pass reads lists only) */
    rc = count(t, keys_in, num_in, end_offsets_out, num_out, s, probing_length,
               values_out ? status_out : nullptr, values_out ? status_handler : WC_HANDLER_NOTHING,
               ignore);
    if (rc) return rc;
    if (!values_out) {
        rc = host_dry_run_status(status_out, num_in, status_handler, ignore, s);
        if (rc) return rc;
        return join_host(t, kStDryRun, s);
    }
    rc = scan(t, begin_offsets_out, end_offsets_out, num_in, s);
    if (rc) return rc;
    BlArgs a = args_of(t, keys_in, num_in, probing_length, status_out, status_handler, ignore);
    a.values_out = values_out;
    a.begin = reinterpret_cast<const unsigned long long *>(begin_offsets_out);
    a.end = reinterpret_cast<const unsigned long long *>(end_offsets_out);
    return launch(bl_kernels(t).values, num_in, a, s);
}

int wc_blht_retrieve_all_keys(wc_blht *t, void *keys_out, uint64_t *num_out, wc_stream_t stream)
{
    int rc = check(t);
    if (rc) return rc;
    if (!num_out) return bl_fail(WC_ERR_INVALID_ARGUMENT, "num_out is NULL");
    return scan_keys(t, keys_out, num_out, nullptr, reinterpret_cast<cudaStream_t>(stream));
}

int wc_blht_num_keys(wc_blht *t, wc_stream_t stream, uint64_t *out)
{
    int rc = check(t);
    if (rc) return rc;
    if (!out) return bl_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    return scan_keys(t, nullptr, out, nullptr, reinterpret_cast<cudaStream_t>(stream));
}

int wc_blht_total_values(wc_blht *t, wc_stream_t stream, uint64_t *out)
{
    int rc = check(t);
    if (rc) return rc;
    if (!out) return bl_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    return scan_keys(t, nullptr, nullptr, out, reinterpret_cast<cudaStream_t>(stream));
}

int wc_blht_pool_used(wc_blht *t, wc_stream_t stream, uint64_t *out)
{
    int rc = check(t);
    if (rc) return rc;
    if (!out) return bl_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    return read_counter(t->counters, reinterpret_cast<cudaStream_t>(stream), out);
}

int wc_blht_peek_status(wc_blht *t, wc_stream_t stream, uint32_t *out)
{
    if (!t || !out) return bl_fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    BL_CUDA(cudaMemcpyAsync(out, t->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    BL_CUDA(cudaStreamSynchronize(s));
    return WC_OK;
}

int wc_blht_pop_status(wc_blht *t, wc_stream_t stream, uint32_t *out)
{
    int rc = wc_blht_peek_status(t, stream, out);
    if (rc) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    BL_CUDA(cudaMemsetAsync(t->status, 0, sizeof(uint32_t), s));
    BL_CUDA(cudaStreamSynchronize(s));
    return WC_OK;
}

int wc_blht_get_info(const wc_blht *t, wc_blht_info *info)
{
    if (!t || !info) return bl_fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memset(info, 0, sizeof(*info));
    info->key_bytes = t->cfg.key_bytes;
    info->value_bytes = t->cfg.value_bytes;
    info->cg_size = t->cfg.cg_size;
    info->probing = t->cfg.probing;
    info->hasher1 = t->cfg.hasher1;
    info->hasher2 = t->cfg.hasher2;
    info->index_bits = t->ib;
    info->counter_bits = t->cb;
    info->size_bits = t->sb;
    info->grow_factor = t->grow;
    info->key_capacity = t->capacity;
    info->value_capacity = t->value_capacity;
    info->num_buckets = t->num_buckets;
    info->seed = t->seed;
    info->empty_key = t->cfg.empty_key;
    info->tombstone_key = t->cfg.tombstone_key;
    info->min_bucket_size = t->min_bucket;
    info->max_bucket_size = t->max_bucket;
    info->max_values_per_key = t->max_values;
    info->bytes_total = t->capacity * (t->cfg.key_bytes + 8) + t->value_capacity * 8 + 8;
    info->keys = t->keys;
    info->handles = t->handles;
    info->pool = t->pool;
    info->next_free = t->counters;
    info->status = t->status;
    info->is_initialized = t->initialized ? 1 : 0;
    return WC_OK;
}

} // extern "C"
