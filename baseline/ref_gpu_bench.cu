/*
 * Timing harness for the REFERENCE warpcore compiled for sm_100a (the GPU
 * baseline that the B200 library is compared with).  Built by
 * baseline/build_ref_gpu.sh from the reference's own headers, with the
 * hpc_helpers stand-in of oracle/ref/, into baseline/_ref/ (git-ignored).
 *
 * Each entry point takes device buffers that the caller already filled,
 * builds the reference structure with its own constructor, and times its
 * own bulk methods with cudaEvents on the legacy default stream, as the
 * reference's benchmark driver does (benchmark_common.cuh:116-199): the
 * table is re-initialised untimed before every insert.  Times are the
 * minimum over `reps`.  Return value: 0, or a CUDA error code.
 */
#include <warpcore/single_value_hash_table.cuh>
#include <warpcore/hash_set.cuh>
#include <warpcore/counting_hash_table.cuh>
#include <warpcore/bloom_filter.cuh>
#include <warpcore/multi_value_hash_table.cuh>
#include <warpcore/multi_bucket_hash_table.cuh>
#include <warpcore/bucket_list_hash_table.cuh>

#include <cfloat>
#include <cstring>
#include <cstdint>

namespace wc = warpcore;

namespace {

struct Timer {
    cudaEvent_t a, b;
    Timer() { cudaEventCreate(&a); cudaEventCreate(&b); }
    ~Timer() { cudaEventDestroy(a); cudaEventDestroy(b); }
    void start() { cudaEventRecord(a, 0); }
    float stop()
    {
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
};

template <class Set>
__global__ void set_contains(const typename Set::key_type *keys, uint64_t n, bool *flags, Set s)
{
    namespace cg = cooperative_groups;
    const uint64_t tid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    const uint64_t gid = tid / Set::cg_size();
    const auto group = cg::tiled_partition<Set::cg_size()>(cg::this_thread_block());
    if (gid < n) {
        bool f = false;
        const wc::Status st = s.retrieve(keys[gid], f, group);
        if (group.thread_rank() == 0 && !st.has_any()) flags[gid] = f;
    }
}

/* After the timed repetitions, `status_out` (if not null) receives the
 * per-key statuses of one more, untimed retrieve with the ReturnStatus
 * handler (single_value_hash_table.cuh:318-337), so that the caller can
 * compare them with its own. */
template <class Table, class K, class V>
int run_table(const K *keys, const V *vals, uint64_t n, const K *q, uint64_t nq, V *out,
              uint64_t min_cap, int reps, float *ms_insert, float *ms_retrieve,
              uint64_t *capacity, uint32_t *status_out)
{
    Table t(min_cap);
    *capacity = t.capacity();
    Timer tm;
    float bi = FLT_MAX, br = FLT_MAX;
    for (int r = 0; r < reps; ++r) {
        t.init();
        cudaDeviceSynchronize();
        tm.start();
        t.insert(keys, vals, n);
        bi = fminf(bi, tm.stop());
        tm.start();
        t.retrieve(q, nq, out);
        br = fminf(br, tm.stop());
    }
    if (status_out)
        t.template retrieve<wc::status_handlers::ReturnStatus>(
            q, nq, out, 0, wc::defaults::probing_length(),
            reinterpret_cast<wc::Status *>(status_out));
    *ms_insert = bi;
    *ms_retrieve = br;
    return int(cudaDeviceSynchronize());
}

} // namespace

/* MultiBucketHashTable<u32,u32> with AoSStore<u32, ArrayBucket<u32, B>>
 * (the reference's multi_bucket benchmark types), B = 1, 2, 4 or 8: bulk
 * insert, then the two-phase bulk retrieve */
template <uint32_t B>
static int ref_mb32(const uint32_t *keys, const uint32_t *vals, uint64_t n, const uint32_t *q,
                    uint64_t nq, uint64_t *begin, uint64_t *end, uint32_t *values_out,
                    uint64_t *num_out, uint64_t min_cap, int reps, float *ms_insert,
                    float *ms_retrieve, uint64_t *capacity)
{
    using Table = wc::MultiBucketHashTable<
        uint32_t, uint32_t, wc::defaults::empty_key<uint32_t>(),
        wc::defaults::tombstone_key<uint32_t>(), wc::defaults::empty_key<uint32_t>(),
        wc::defaults::probing_scheme_t<uint32_t, 8>,
        wc::storage::key_value::AoSStore<uint32_t, wc::ArrayBucket<uint32_t, B>>>;
    Table t(min_cap);
    *capacity = t.capacity();
    Timer tm;
    float bi = FLT_MAX, br = FLT_MAX;
    for (int r = 0; r < reps; ++r) {
        t.init();
        cudaDeviceSynchronize();
        tm.start();
        t.insert(keys, vals, n);
        bi = fminf(bi, tm.stop());
        wc::index_t num = 0;
        tm.start();
        t.retrieve(q, nq, (wc::index_t *)begin, (wc::index_t *)end, values_out, num);
        br = fminf(br, tm.stop());
        *num_out = num;
    }
    *ms_insert = bi;
    *ms_retrieve = br;
    return int(cudaDeviceSynchronize());
}

extern "C" {

int ref_svht64_run(const uint64_t *keys, const uint64_t *vals, uint64_t n, const uint64_t *q,
                   uint64_t nq, uint64_t *out, uint64_t min_cap, int reps, float *ms_insert,
                   float *ms_retrieve, uint64_t *capacity, uint32_t *status_out)
{
    return run_table<wc::SingleValueHashTable<uint64_t, uint64_t>>(
        keys, vals, n, q, nq, out, min_cap, reps, ms_insert, ms_retrieve, capacity, status_out);
}

/* the same table stored as a struct of arrays (storage.cuh:218-432) */
int ref_svht64_soa_run(const uint64_t *keys, const uint64_t *vals, uint64_t n, const uint64_t *q,
                       uint64_t nq, uint64_t *out, uint64_t min_cap, int reps, float *ms_insert,
                       float *ms_retrieve, uint64_t *capacity, uint32_t *status_out)
{
    using Soa = wc::SingleValueHashTable<uint64_t, uint64_t, wc::defaults::empty_key<uint64_t>(),
                                         wc::defaults::tombstone_key<uint64_t>(),
                                         wc::defaults::probing_scheme_t<uint64_t, 8>,
                                         wc::storage::key_value::SoAStore<uint64_t, uint64_t>>;
    return run_table<Soa>(keys, vals, n, q, nq, out, min_cap, reps, ms_insert, ms_retrieve,
                          capacity, status_out);
}

int ref_svht32_run(const uint32_t *keys, const uint32_t *vals, uint64_t n, const uint32_t *q,
                   uint64_t nq, uint32_t *out, uint64_t min_cap, int reps, float *ms_insert,
                   float *ms_retrieve, uint64_t *capacity, uint32_t *status_out)
{
    return run_table<wc::SingleValueHashTable<uint32_t, uint32_t>>(
        keys, vals, n, q, nq, out, min_cap, reps, ms_insert, ms_retrieve, capacity, status_out);
}

int ref_svht32_soa_run(const uint32_t *keys, const uint32_t *vals, uint64_t n, const uint32_t *q,
                       uint64_t nq, uint32_t *out, uint64_t min_cap, int reps, float *ms_insert,
                       float *ms_retrieve, uint64_t *capacity, uint32_t *status_out)
{
    using Soa = wc::SingleValueHashTable<uint32_t, uint32_t, wc::defaults::empty_key<uint32_t>(),
                                         wc::defaults::tombstone_key<uint32_t>(),
                                         wc::defaults::probing_scheme_t<uint32_t, 8>,
                                         wc::storage::key_value::SoAStore<uint32_t, uint32_t>>;
    return run_table<Soa>(keys, vals, n, q, nq, out, min_cap, reps, ms_insert, ms_retrieve,
                          capacity, status_out);
}

/* HashSet<u64>: the host bulk retrieve does not compile (hash_set.cuh:356),
 * so contains runs the device method from this harness's own kernel */
int ref_hashset64_run(const uint64_t *keys, uint64_t n, const uint64_t *q, uint64_t nq,
                      bool *flags, uint64_t min_cap, int reps, float *ms_insert,
                      float *ms_retrieve, uint64_t *capacity)
{
    using Set = wc::HashSet<uint64_t>;
    Set s(min_cap);
    *capacity = s.capacity();
    Timer tm;
    float bi = FLT_MAX, br = FLT_MAX;
    for (int r = 0; r < reps; ++r) {
        s.init();
        cudaDeviceSynchronize();
        tm.start();
        s.insert(keys, n);
        bi = fminf(bi, tm.stop());
        tm.start();
        const uint64_t threads = nq * Set::cg_size();
        set_contains<Set><<<(threads + 1023) / 1024, 1024>>>(q, nq, flags, s);
        br = fminf(br, tm.stop());
    }
    *ms_insert = bi;
    *ms_retrieve = br;
    return int(cudaDeviceSynchronize());
}

int ref_counting32_run(const uint32_t *keys, uint64_t n, const uint32_t *q, uint64_t nq,
                       uint32_t *out, uint64_t min_cap, int reps, float *ms_insert,
                       float *ms_retrieve, uint64_t *capacity, uint32_t *status_out)
{
    using Table = wc::CountingHashTable<uint32_t, uint32_t>;
    Table t(min_cap);
    *capacity = t.capacity();
    Timer tm;
    float bi = FLT_MAX, br = FLT_MAX;
    for (int r = 0; r < reps; ++r) {
        t.init();
        cudaDeviceSynchronize();
        tm.start();
        t.insert(keys, n);
        bi = fminf(bi, tm.stop());
        tm.start();
        t.retrieve(q, nq, out);
        br = fminf(br, tm.stop());
    }
    if (status_out)
        t.template retrieve<wc::status_handlers::ReturnStatus>(
            q, nq, out, 0, wc::defaults::probing_length(),
            reinterpret_cast<wc::Status *>(status_out));
    *ms_insert = bi;
    *ms_retrieve = br;
    return int(cudaDeviceSynchronize());
}

/* BloomFilter<u64, MurmurHash<u64>, u64, 8>.  After the timed repetitions
 * (each re-initialises the filter, so it ends holding exactly the inserted
 * keys), `words_out` (if not null, num_slots() words of device memory)
 * receives the filter's bit vector and *num_slots its length. */
int ref_bloom64_run(const uint64_t *keys, uint64_t n, const uint64_t *q, uint64_t nq,
                    bool *flags, uint64_t num_bits, uint64_t k, int reps, float *ms_insert,
                    float *ms_retrieve, uint64_t *words_out, uint64_t *num_slots)
{
    using Filter = wc::BloomFilter<uint64_t, wc::hashers::MurmurHash<uint64_t>, uint64_t, 8>;
    Filter f(num_bits, k);
    *num_slots = f.num_slots();
    Timer tm;
    float bi = FLT_MAX, br = FLT_MAX;
    for (int r = 0; r < reps; ++r) {
        f.init();
        cudaDeviceSynchronize();
        tm.start();
        f.insert(keys, n);
        bi = fminf(bi, tm.stop());
        tm.start();
        f.retrieve(q, nq, flags);
        br = fminf(br, tm.stop());
    }
    if (words_out) {
        /* BloomFilter keeps its bit vector private and has no accessor; the
         * device pointer is its first data member (bloom_filter.cuh:410) */
        uint64_t *words_d = nullptr;
        std::memcpy(&words_d, &f, sizeof(words_d));
        cudaMemcpy(words_out, words_d, sizeof(uint64_t) * f.num_slots(), cudaMemcpyDeviceToDevice);
    }
    *ms_insert = bi;
    *ms_retrieve = br;
    return int(cudaDeviceSynchronize());
}

/* MultiValueHashTable<u32,u32>: bulk insert, then the two-phase bulk
 * retrieve (counts, scan, values; it synchronises) into caller buffers of
 * at least the number of values */
int ref_mv32_run(const uint32_t *keys, const uint32_t *vals, uint64_t n, const uint32_t *q,
                 uint64_t nq, uint64_t *begin, uint64_t *end, uint32_t *values_out,
                 uint64_t *num_out, uint64_t min_cap, int reps, float *ms_insert,
                 float *ms_retrieve, uint64_t *capacity)
{
    using Table = wc::MultiValueHashTable<uint32_t, uint32_t>;
    Table t(min_cap);
    *capacity = t.capacity();
    Timer tm;
    float bi = FLT_MAX, br = FLT_MAX;
    for (int r = 0; r < reps; ++r) {
        t.init();
        cudaDeviceSynchronize();
        tm.start();
        t.insert(keys, vals, n);
        bi = fminf(bi, tm.stop());
        wc::index_t num = 0;
        tm.start();
        t.retrieve(q, nq, (wc::index_t *)begin, (wc::index_t *)end, values_out, num);
        br = fminf(br, tm.stop());
        *num_out = num;
    }
    *ms_insert = bi;
    *ms_retrieve = br;
    return int(cudaDeviceSynchronize());
}

int ref_mb32_run(const uint32_t *keys, const uint32_t *vals, uint64_t n, const uint32_t *q,
                 uint64_t nq, uint64_t *begin, uint64_t *end, uint32_t *values_out,
                 uint64_t *num_out, uint64_t min_cap, uint32_t bucket, int reps, float *ms_insert,
                 float *ms_retrieve, uint64_t *capacity)
{
    switch (bucket) {
    case 1: return ref_mb32<1>(keys, vals, n, q, nq, begin, end, values_out, num_out, min_cap, reps, ms_insert, ms_retrieve, capacity);
    case 2: return ref_mb32<2>(keys, vals, n, q, nq, begin, end, values_out, num_out, min_cap, reps, ms_insert, ms_retrieve, capacity);
    case 4: return ref_mb32<4>(keys, vals, n, q, nq, begin, end, values_out, num_out, min_cap, reps, ms_insert, ms_retrieve, capacity);
    case 8: return ref_mb32<8>(keys, vals, n, q, nq, begin, end, values_out, num_out, min_cap, reps, ms_insert, ms_retrieve, capacity);
    default: return -1;
    }
}

/* BucketListHashTable<u32, u32> over BucketListStore<u32, 29, 18, 15> (the
 * reference's bucket_list benchmark types), grow factor 1.1, first bucket
 * 1: bulk insert (n a multiple of 128, the insert kernel's groups per
 * block), then the two-phase bulk retrieve */
int ref_bl32_run(const uint32_t *keys, const uint32_t *vals, uint64_t n, const uint32_t *q,
                 uint64_t nq, uint64_t *begin, uint64_t *end, uint32_t *values_out,
                 uint64_t *num_out, uint64_t key_cap, uint64_t value_cap, int reps,
                 float *ms_insert, float *ms_retrieve, uint64_t *capacity)
{
    if (n % 128) return -1;
    using Store = wc::storage::multi_value::BucketListStore<uint32_t, 29, 18, 15>;
    using Table = wc::BucketListHashTable<uint32_t, uint32_t, wc::defaults::empty_key<uint32_t>(),
                                          wc::defaults::tombstone_key<uint32_t>(), Store,
                                          wc::defaults::probing_scheme_t<uint32_t, 8>>;
    Table t(key_cap, value_cap, wc::defaults::seed<uint32_t>(), 1.1f, 1);
    *capacity = t.key_capacity();
    Timer tm;
    float bi = FLT_MAX, br = FLT_MAX;
    for (int r = 0; r < reps; ++r) {
        t.init();
        cudaDeviceSynchronize();
        tm.start();
        t.insert(keys, vals, n);
        bi = fminf(bi, tm.stop());
        wc::index_t num = 0;
        tm.start();
        t.retrieve(q, nq, (wc::index_t *)begin, (wc::index_t *)end, values_out, num);
        br = fminf(br, tm.stop());
        *num_out = num;
    }
    *ms_insert = bi;
    *ms_retrieve = br;
    return int(cudaDeviceSynchronize());
}

} // extern "C"
