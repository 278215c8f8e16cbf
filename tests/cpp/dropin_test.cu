/*
 * Drop-in check of the C++ front end: code written against warpcore's C++
 * API (host bulk methods, device per-key methods in user kernels, for_each
 * with a device lambda, status handlers) compiles against include/warpcore
 * and gives the reference's answers.  Exit code 0 on success.
 */
#include <warpcore/warpcore.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <numeric>
#include <random>
#include <unordered_map>
#include <vector>

namespace wc = warpcore;
namespace cg = cooperative_groups;

static int g_fail = 0;
#define CHECK(c)                                                                       \
    do {                                                                               \
        if (!(c)) {                                                                    \
            std::fprintf(stderr, "CHECK failed: %s (line %d)\n", #c, __LINE__);      \
            g_fail = 1;                                                                \
        }                                                                              \
    } while (0)

template <class T>
static T *dcopy(const std::vector<T> &h)
{
    T *d = nullptr;
    cudaMalloc(&d, sizeof(T) * std::max<size_t>(h.size(), 1));
    cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
    return d;
}

template <class T>
static std::vector<T> hcopy(const T *d, size_t n)
{
    std::vector<T> h(n);
    cudaDeviceSynchronize();
    cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost);
    return h;
}

template <class K>
static std::vector<K> distinct_keys(size_t n, unsigned seed)
{
    std::mt19937_64 rng(seed);
    std::vector<K> v;
    std::unordered_map<K, int> seen;
    while (v.size() < n) {
        const K k = K(rng());
        if (k == K(0) || k == K(~K(0)) || seen.count(k)) continue;
        seen[k] = 1;
        v.push_back(k);
    }
    return v;
}

/* device-side insert of (key, value) pairs, one tile of cg_size() per key */
template <class Table>
__global__ void device_insert(Table t, const typename Table::key_type *k,
                              const typename Table::value_type *v, uint64_t n, wc::Status *st)
{
    const auto g = cg::tiled_partition<Table::cg_size()>(cg::this_thread_block());
    const uint64_t gid = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / Table::cg_size();
    if (gid < n) {
        const wc::Status s = t.insert(k[gid], v[gid], g);
        if (g.thread_rank() == 0) st[gid] = s;
    }
}

template <class Table>
__global__ void device_retrieve(Table t, const typename Table::key_type *k, uint64_t n,
                                typename Table::value_type *out, wc::Status *st)
{
    const auto g = cg::tiled_partition<Table::cg_size()>(cg::this_thread_block());
    const uint64_t gid = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / Table::cg_size();
    if (gid < n) {
        typename Table::value_type v = 0;
        const wc::Status s = t.retrieve(k[gid], v, g);
        if (g.thread_rank() == 0) {
            st[gid] = s;
            if (!s.has_any()) out[gid] = v;
        }
    }
}

template <class Set>
__global__ void device_contains(Set s, const typename Set::key_type *k, uint64_t n, bool *flags)
{
    const auto g = cg::tiled_partition<Set::cg_size()>(cg::this_thread_block());
    const uint64_t gid = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / Set::cg_size();
    if (gid < n) {
        bool f = false;
        const wc::Status st = s.retrieve(k[gid], f, g);
        if (g.thread_rank() == 0 && !st.has_any()) flags[gid] = f;
    }
}

template <class Counter>
__global__ void device_count(Counter c, const typename Counter::key_type *k, uint64_t n)
{
    const auto g = cg::tiled_partition<Counter::cg_size()>(cg::this_thread_block());
    const uint64_t gid = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / Counter::cg_size();
    if (gid < n) c.insert(k[gid], g);
}

template <class Filter>
__global__ void device_query(Filter f, const typename Filter::key_type *k, uint64_t n, bool *out)
{
    const auto g = cg::tiled_partition<Filter::cg_size()>(cg::this_thread_block());
    const uint64_t gid = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / Filter::cg_size();
    if (gid < n) {
        const bool r = f.retrieve(k[gid], g);
        if (g.thread_rank() == 0) out[gid] = r;
    }
}

template <class Filter>
__global__ void device_insert_and_query(Filter f, const typename Filter::key_type *k, uint64_t n,
                                        bool *out)
{
    const auto g = cg::tiled_partition<1>(cg::this_thread_block());
    const uint64_t gid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (gid < n) out[gid] = f.insert_and_query(k[gid], g);
}

static unsigned blocks_for(uint64_t n, uint64_t cg) { return unsigned((n * cg + 255) / 256); }

static void test_svht_u32()
{
    using Table = wc::SingleValueHashTable<uint32_t, uint32_t>;
    const uint64_t n = 100000;
    auto keys = distinct_keys<uint32_t>(2 * n, 1);
    std::vector<uint32_t> ins(keys.begin(), keys.begin() + n), vals(n);
    for (uint64_t i = 0; i < n; ++i) vals[i] = uint32_t(i * 2654435761u);
    Table t(uint64_t(n / 0.8));
    CHECK(t.capacity() == wc::detail::get_valid_capacity(uint64_t(n / 0.8), 8));
    CHECK(t.size() == 0);
    CHECK(t.peek_status() == wc::Status::none());
    uint32_t *dk = dcopy(ins), *dv = dcopy(vals), *dq = dcopy(keys);
    uint32_t *dout;
    cudaMalloc(&dout, sizeof(uint32_t) * 2 * n);
    cudaMemset(dout, 0xff, sizeof(uint32_t) * 2 * n);
    wc::Status *dst;
    cudaMalloc(&dst, sizeof(wc::Status) * 2 * n);
    t.insert(dk, dv, n);
    CHECK(t.size() == n);
    t.retrieve<wc::status_handlers::ReturnStatus>(dq, 2 * n, dout, 0, wc::defaults::probing_length(), dst);
    auto out = hcopy(dout, 2 * n);
    auto st = hcopy(reinterpret_cast<uint32_t *>(dst), 2 * n);
    for (uint64_t i = 0; i < n; ++i) {
        CHECK(out[i] == vals[i]);
        CHECK(st[i] == 0);
        CHECK(out[n + i] == 0xffffffffu);
        CHECK(st[n + i] == wc::Status::key_not_found().base());
    }
    CHECK(t.pop_status().has_key_not_found());
    /* ReturnBoolean<none>: the reference's flag of key_not_found is false */
    bool *dflag;
    cudaMalloc(&dflag, 2 * n);
    t.retrieve<wc::status_handlers::ReturnBoolean<>>(dq, 2 * n, dout, 0, wc::defaults::probing_length(), dflag);
    auto fl = hcopy(reinterpret_cast<uint8_t *>(dflag), 2 * n);
    CHECK(std::count(fl.begin(), fl.end(), 1) == 0);
    /* for_each with a device lambda counts every pair */
    unsigned long long *dc;
    cudaMalloc(&dc, 8);
    cudaMemset(dc, 0, 8);
    t.for_each([=] __device__(uint32_t k, uint32_t v) { atomicAdd(dc, 1ull); });
    CHECK(hcopy(dc, 1)[0] == n);
    /* retrieve_all */
    uint32_t *ak, *av;
    cudaMalloc(&ak, sizeof(uint32_t) * t.capacity());
    cudaMalloc(&av, sizeof(uint32_t) * t.capacity());
    wc::index_t num = 0;
    t.retrieve_all(ak, av, num);
    CHECK(num == n);
    /* erase then size */
    t.erase(dk, n / 2);
    CHECK(t.size() == n - n / 2);
    cudaFree(dk); cudaFree(dv); cudaFree(dq); cudaFree(dout); cudaFree(dst); cudaFree(dflag);
    cudaFree(dc); cudaFree(ak); cudaFree(av);
}

static void test_svht_u64_device_api()
{
    using Table = wc::SingleValueHashTable<uint64_t, uint64_t>;
    const uint64_t n = 50000;
    auto keys = distinct_keys<uint64_t>(2 * n, 2);
    std::vector<uint64_t> a(keys.begin(), keys.begin() + n), b(keys.begin() + n, keys.end());
    std::vector<uint64_t> va(n), vb(n);
    for (uint64_t i = 0; i < n; ++i) { va[i] = i + 1; vb[i] = ~i; }
    Table t(4 * n);
    uint64_t *da = dcopy(a), *dva = dcopy(va), *db = dcopy(b), *dvb = dcopy(vb);
    wc::Status *dst;
    cudaMalloc(&dst, sizeof(wc::Status) * n);
    /* half inserted by the bulk kernel, half by a user kernel */
    t.insert(da, dva, n);
    device_insert<<<blocks_for(n, Table::cg_size()), 256>>>(t, db, dvb, n, dst);
    auto st = hcopy(reinterpret_cast<uint32_t *>(dst), n);
    CHECK(std::all_of(st.begin(), st.end(), [](uint32_t s) { return s == 0; }));
    CHECK(t.size() == 2 * n);
    /* the bulk path finds the device-inserted keys and vice versa */
    uint64_t *dout;
    cudaMalloc(&dout, sizeof(uint64_t) * n);
    t.retrieve(db, n, dout);
    auto o1 = hcopy(dout, n);
    CHECK(o1 == vb);
    device_retrieve<<<blocks_for(n, Table::cg_size()), 256>>>(t, da, n, dout, dst);
    auto o2 = hcopy(dout, n);
    CHECK(o2 == va);
    /* duplicates through the device API overwrite and report duplicate_key */
    device_insert<<<blocks_for(n, Table::cg_size()), 256>>>(t, da, dvb, n, dst);
    st = hcopy(reinterpret_cast<uint32_t *>(dst), n);
    CHECK(std::all_of(st.begin(), st.end(), [](uint32_t s) { return s == wc::Status::duplicate_key().base(); }));
    t.retrieve(da, n, dout);
    CHECK(hcopy(dout, n) == vb);
    cudaFree(da); cudaFree(dva); cudaFree(db); cudaFree(dvb); cudaFree(dst); cudaFree(dout);
}

/* SingleValueHashTable with SoAStore: keys and values in two arrays, the
 * same answers through the bulk and the device API */
template <class K, class V>
static void test_svht_soa(unsigned seed)
{
    using Store = wc::storage::key_value::SoAStore<K, V>;
    using Table = wc::SingleValueHashTable<K, V, wc::defaults::empty_key<K>(),
                                           wc::defaults::tombstone_key<K>(),
                                           wc::defaults::probing_scheme_t<K, 8>, Store>;
    const uint64_t n = 40000;
    auto keys = distinct_keys<K>(2 * n, seed);
    std::vector<K> a(keys.begin(), keys.begin() + n), b(keys.begin() + n, keys.end());
    std::vector<V> va(n), vb(n);
    for (uint64_t i = 0; i < n; ++i) { va[i] = V(i + 7); vb[i] = V(~i); }
    Table t(uint64_t(2 * n / 0.9));
    K *da = dcopy(a), *db = dcopy(b);
    V *dva = dcopy(va), *dvb = dcopy(vb);
    wc::Status *dst;
    cudaMalloc(&dst, sizeof(wc::Status) * n);
    t.insert(da, dva, n);
    device_insert<<<blocks_for(n, Table::cg_size()), 256>>>(t, db, dvb, n, dst);
    auto st = hcopy(reinterpret_cast<uint32_t *>(dst), n);
    CHECK(std::all_of(st.begin(), st.end(), [](uint32_t s) { return s == 0; }));
    CHECK(t.size() == 2 * n);
    V *dout;
    cudaMalloc(&dout, sizeof(V) * n);
    t.retrieve(db, n, dout);
    CHECK(hcopy(dout, n) == vb);
    device_retrieve<<<blocks_for(n, Table::cg_size()), 256>>>(t, da, n, dout, dst);
    CHECK(hcopy(dout, n) == va);
    /* duplicates overwrite the value array's element */
    device_insert<<<blocks_for(n, Table::cg_size()), 256>>>(t, da, dvb, n, dst);
    st = hcopy(reinterpret_cast<uint32_t *>(dst), n);
    CHECK(std::all_of(st.begin(), st.end(), [](uint32_t s) { return s == wc::Status::duplicate_key().base(); }));
    t.retrieve(da, n, dout);
    CHECK(hcopy(dout, n) == vb);
    /* the memory is a key array and a value array: key slot i holds a key,
     * value i its value */
    const auto &view = t.device_view();
    CHECK(view.values != nullptr);
    const auto hk = hcopy(reinterpret_cast<const K *>(view.slots), t.capacity());
    const auto hv = hcopy(reinterpret_cast<const V *>(view.values), t.capacity());
    std::unordered_map<K, V> expect;
    for (uint64_t i = 0; i < n; ++i) { expect[a[i]] = vb[i]; expect[b[i]] = vb[i]; }
    uint64_t seen = 0;
    for (uint64_t i = 0; i < t.capacity(); ++i) {
        if (!Table::is_valid_key(hk[i])) continue;
        ++seen;
        CHECK(expect.count(hk[i]) == 1 && expect[hk[i]] == hv[i]);
    }
    CHECK(seen == 2 * n);
    /* for_each and retrieve_all read the value array */
    unsigned long long *dc;
    cudaMalloc(&dc, 16);
    cudaMemset(dc, 0, 16);
    t.for_each([=] __device__(K k, V v) {
        atomicAdd(dc, 1ull);
        atomicAdd(dc + 1, (unsigned long long)v);
    });
    const auto c = hcopy(dc, 2);
    unsigned long long vsum = 0;
    for (uint64_t i = 0; i < n; ++i) vsum += 2ull * (unsigned long long)vb[i];
    CHECK(c[0] == 2 * n && c[1] == vsum);
    K *ak;
    V *av;
    cudaMalloc(&ak, sizeof(K) * t.capacity());
    cudaMalloc(&av, sizeof(V) * t.capacity());
    wc::index_t num = 0;
    t.retrieve_all(ak, av, num);
    CHECK(num == 2 * n);
    const auto rk = hcopy(ak, num);
    const auto rv = hcopy(av, num);
    for (uint64_t i = 0; i < num; ++i) CHECK(expect.count(rk[i]) == 1 && expect[rk[i]] == rv[i]);
    /* erase leaves tombstones in the key array */
    t.erase(da, n);
    CHECK(t.size() == n);
    t.retrieve(db, n, dout);
    CHECK(hcopy(dout, n) == vb);
    cudaFree(da); cudaFree(db); cudaFree(dva); cudaFree(dvb); cudaFree(dst); cudaFree(dout);
    cudaFree(dc); cudaFree(ak); cudaFree(av);
}

static void test_hash_set()
{
    using Set = wc::HashSet<uint64_t>;
    const uint64_t n = 60000;
    auto keys = distinct_keys<uint64_t>(2 * n, 3);
    Set s(uint64_t(n / 0.9));
    CHECK(Set::cg_size() == 16);
    uint64_t *dk = dcopy(keys);
    s.insert(dk, n);
    CHECK(s.size() == n);
    bool *df;
    cudaMalloc(&df, 2 * n);
    s.retrieve(dk, 2 * n, df); /* the host form that does not compile in the reference */
    auto f = hcopy(reinterpret_cast<uint8_t *>(df), 2 * n);
    for (uint64_t i = 0; i < 2 * n; ++i) CHECK(f[i] == (i < n ? 1 : 0));
    cudaMemset(df, 7, 2 * n);
    device_contains<<<blocks_for(2 * n, Set::cg_size()), 256>>>(s, dk, 2 * n, df);
    auto f2 = hcopy(reinterpret_cast<uint8_t *>(df), 2 * n);
    CHECK(f2 == f);
    cudaFree(dk); cudaFree(df);
}

static void test_counting()
{
    using Counter = wc::CountingHashTable<uint32_t, uint32_t>;
    const uint64_t distinct = 5000;
    auto keys = distinct_keys<uint32_t>(distinct, 4);
    std::vector<uint32_t> occ;
    for (uint64_t i = 0; i < distinct; ++i)
        for (uint64_t j = 0; j < 1 + (i % 7); ++j) occ.push_back(keys[i]);
    std::shuffle(occ.begin(), occ.end(), std::mt19937(5));
    Counter c(2 * distinct);
    uint32_t *docc = dcopy(occ), *dk = dcopy(keys), *dout;
    cudaMalloc(&dout, sizeof(uint32_t) * distinct);
    c.insert(docc, occ.size());                                            /* bulk */
    device_count<<<blocks_for(occ.size(), Counter::cg_size()), 256>>>(c, docc, occ.size()); /* device */
    c.retrieve(dk, distinct, dout);
    auto out = hcopy(dout, distinct);
    for (uint64_t i = 0; i < distinct; ++i) CHECK(out[i] == 2 * (1 + (i % 7)));
    /* for_each visits every key once with its count */
    unsigned long long *dacc;
    cudaMalloc(&dacc, 2 * sizeof(unsigned long long));
    cudaMemset(dacc, 0, 2 * sizeof(unsigned long long));
    c.for_each([=] __device__(uint32_t k, uint32_t n) {
        atomicAdd(dacc, 1ull);
        atomicAdd(dacc + 1, (unsigned long long)n);
    });
    auto acc = hcopy(dacc, 2);
    CHECK(acc[0] == distinct);
    CHECK(acc[1] == 2 * occ.size());
    CHECK(Counter::is_empty_key(0) && Counter::is_tombstone_key(~0u) && !Counter::is_empty_key(5));
    cudaFree(dacc);
    Counter capped(2 * distinct, wc::defaults::seed<uint32_t>(), 3);
    capped.insert(docc, occ.size());
    capped.retrieve(dk, distinct, dout);
    out = hcopy(dout, distinct);
    for (uint64_t i = 0; i < distinct; ++i) CHECK(out[i] == std::min<uint32_t>(3, 1 + (i % 7)));
    cudaFree(docc); cudaFree(dk); cudaFree(dout);
}

static void test_bloom()
{
    using Filter = wc::BloomFilter<uint64_t, wc::hashers::MurmurHash<uint64_t>, uint64_t, 8>;
    const uint64_t n = 100000;
    auto keys = distinct_keys<uint64_t>(2 * n, 6);
    Filter f(16 * n, 8);
    CHECK(f.num_slots() == 16 * n / 64);
    uint64_t *dk = dcopy(keys);
    bool *dflag;
    cudaMalloc(&dflag, 2 * n);
    f.insert(dk, n);
    f.retrieve(dk, 2 * n, dflag);
    auto a = hcopy(reinterpret_cast<uint8_t *>(dflag), 2 * n);
    for (uint64_t i = 0; i < n; ++i) CHECK(a[i] == 1);
    device_query<<<blocks_for(2 * n, 8), 256>>>(f, dk, 2 * n, dflag);
    auto b = hcopy(reinterpret_cast<uint8_t *>(dflag), 2 * n);
    CHECK(a == b); /* device and bulk queries agree bit for bit */
    uint64_t fp = 0;
    for (uint64_t i = n; i < 2 * n; ++i) fp += a[i];
    CHECK(fp < n / 100);
    /* CG 1: insert_and_query reports prior membership */
    wc::BloomFilter<uint64_t> f1(1 << 22, 6);
    device_insert_and_query<<<blocks_for(n, 1), 256>>>(f1, dk, n, dflag);
    auto c = hcopy(reinterpret_cast<uint8_t *>(dflag), n);
    uint64_t before = 0;
    for (auto v : c) before += v;
    CHECK(before < n / 10);
    device_insert_and_query<<<blocks_for(n, 1), 256>>>(f1, dk, n, dflag);
    auto d = hcopy(reinterpret_cast<uint8_t *>(dflag), n);
    CHECK(std::all_of(d.begin(), d.end(), [](uint8_t x) { return x == 1; }));
    cudaFree(dk); cudaFree(dflag);
}

/* The reference's filtered-histogram example (examples/src/
 * advanced_usage_from_device.cu), in this test's words: a CG-1 Bloom
 * filter's insert_and_query tells whether a key was seen before, and the
 * keys seen before are counted in a CountingHashTable<u32, u64>, one key at
 * a time by the counting table's tile. */
template <class Filter, class Counter>
__global__ void filtered_histogram(const uint32_t *keys, uint64_t n, Filter f, Counter c)
{
    const auto fg = cg::tiled_partition<1>(cg::this_thread_block());
    const auto tg = cg::tiled_partition<Counter::cg_size()>(cg::this_thread_block());
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    uint32_t key = 0;
    bool seen = false;
    if (i < n) {
        key = keys[i];
        seen = f.insert_and_query(key, fg);
    }
    unsigned todo = tg.ballot(seen);
    while (todo) {
        const int src = __ffs(todo) - 1;
        c.insert(tg.shfl(key, src), tg);
        todo &= todo - 1;
    }
}

static void test_filtered_histogram()
{
    using Filter = wc::BloomFilter<uint32_t, wc::hashers::MuellerHash, uint32_t>;
    using Counter = wc::CountingHashTable<uint32_t, uint64_t>;
    const uint64_t n = 1 << 20, mult = 4;
    std::vector<uint32_t> keys(n);
    for (uint64_t i = 0; i < n / 2; ++i) keys[i] = uint32_t(i + 1); /* seen once */
    for (uint64_t i = n / 2; i < n; i += mult)                      /* seen 4 times */
        for (uint64_t j = 0; j < mult; ++j) keys[i + j] = uint32_t(i + 1);
    std::shuffle(keys.begin(), keys.end(), std::mt19937(77));
    Filter f(n * 16, 6, 420);
    Counter c(n);
    uint32_t *dk = dcopy(keys);
    filtered_histogram<<<unsigned(n / 256), 256>>>(dk, n, f, c);
    /* ask for every distinct key */
    std::vector<uint32_t> q;
    for (uint64_t i = 0; i < n / 2; ++i) q.push_back(uint32_t(i + 1));
    for (uint64_t i = n / 2; i < n; i += mult) q.push_back(uint32_t(i + 1));
    uint32_t *dq = dcopy(q);
    uint64_t *dcnt;
    cudaMalloc(&dcnt, sizeof(uint64_t) * q.size());
    cudaMemset(dcnt, 0, sizeof(uint64_t) * q.size());
    c.retrieve(dq, q.size(), dcnt);
    auto cnt = hcopy(dcnt, q.size());
    /* a repeated key is counted 3 times (its first occurrence is new to the
     * filter), 4 if that first occurrence was a false positive; a unique key
     * 0 times, or once after a false positive */
    uint64_t odd_unique = 0, odd_repeat = 0, bad = 0;
    for (uint64_t i = 0; i < n / 2; ++i) {
        odd_unique += cnt[i] == 1;
        bad += cnt[i] > 1;
    }
    for (uint64_t i = n / 2; i < q.size(); ++i) {
        odd_repeat += cnt[i] == mult;
        bad += cnt[i] != mult - 1 && cnt[i] != mult;
    }
    CHECK(bad == 0);
    CHECK(odd_unique < n / 2 / 100);
    CHECK(odd_repeat < (n / 2 / mult) / 100);
    /* the table holds exactly the repeated keys and the false positives */
    CHECK(c.size() == (n / 2) / mult + odd_unique);
    cudaFree(dk); cudaFree(dq); cudaFree(dcnt);
}

/* values of other widths than the key, and non-integral values */
static void test_mixed_widths()
{
    {
        using Table = wc::SingleValueHashTable<uint32_t, uint64_t>;
        const uint64_t n = 20000;
        auto keys = distinct_keys<uint32_t>(2 * n, 8);
        std::vector<uint64_t> vals(n);
        for (uint64_t i = 0; i < n; ++i) vals[i] = (uint64_t(keys[i]) << 32) | (i * 7 + 1);
        Table t(2 * n);
        uint32_t *dk = dcopy(keys);
        uint64_t *dv = dcopy(vals), *dout;
        cudaMalloc(&dout, sizeof(uint64_t) * 2 * n);
        cudaMemset(dout, 0xff, sizeof(uint64_t) * 2 * n);
        t.insert(dk, dv, n);
        CHECK(t.size() == n);
        t.retrieve(dk, 2 * n, dout);
        auto out = hcopy(dout, 2 * n);
        for (uint64_t i = 0; i < n; ++i) CHECK(out[i] == vals[i]);
        for (uint64_t i = n; i < 2 * n; ++i) CHECK(out[i] == ~0ull); /* misses untouched */
        /* device retrieve through the tile API */
        wc::Status *dst;
        cudaMalloc(&dst, sizeof(wc::Status) * n);
        cudaMemset(dout, 0, sizeof(uint64_t) * n);
        device_retrieve<<<blocks_for(n, Table::cg_size()), 256>>>(t, dk, n, dout, dst);
        out = hcopy(dout, n);
        for (uint64_t i = 0; i < n; ++i) CHECK(out[i] == vals[i]);
        /* for_each sees every pair */
        unsigned long long *dsum;
        cudaMalloc(&dsum, sizeof(unsigned long long));
        cudaMemset(dsum, 0, sizeof(unsigned long long));
        t.for_each([=] __device__(uint32_t k, uint64_t v) {
            if ((v >> 32) == k) atomicAdd(dsum, 1ull);
        });
        CHECK(hcopy(dsum, 1)[0] == n);
        cudaFree(dk); cudaFree(dv); cudaFree(dout); cudaFree(dst); cudaFree(dsum);
    }
    {
        using Table = wc::SingleValueHashTable<uint64_t, float>;
        const uint64_t n = 10000;
        auto keys = distinct_keys<uint64_t>(n, 9);
        std::vector<float> vals(n);
        for (uint64_t i = 0; i < n; ++i) vals[i] = 0.5f * float(i) - 17.25f;
        Table t(2 * n);
        uint64_t *dk = dcopy(keys);
        float *dv = dcopy(vals), *dout;
        cudaMalloc(&dout, sizeof(float) * n);
        t.insert(dk, dv, n);
        t.retrieve(dk, n, dout);
        auto out = hcopy(dout, n);
        CHECK(out == vals);
        uint64_t *dak;
        float *dav;
        cudaMalloc(&dak, sizeof(uint64_t) * n);
        cudaMalloc(&dav, sizeof(float) * n);
        wc::index_t num = 0;
        t.retrieve_all(dak, dav, num);
        CHECK(num == n);
        auto ak = hcopy(dak, n);
        auto av = hcopy(dav, n);
        std::unordered_map<uint64_t, float> m;
        for (uint64_t i = 0; i < n; ++i) m[keys[i]] = vals[i];
        for (uint64_t i = 0; i < n; ++i) CHECK(m.count(ak[i]) && m[ak[i]] == av[i]);
        cudaFree(dk); cudaFree(dv); cudaFree(dout); cudaFree(dak); cudaFree(dav);
    }
}

/* device per-key MultiValueHashTable methods: each group inserts one pair,
 * then counts a key's values and reads them */
template <class Table>
__global__ void device_mv_insert(Table t, const typename Table::key_type *k,
                                 const typename Table::value_type *v, uint64_t n, uint32_t *st)
{
    const auto g = cg::tiled_partition<Table::cg_size()>(cg::this_thread_block());
    const uint64_t gid = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / Table::cg_size();
    if (gid >= n) return;
    const auto s = t.insert(k[gid], v[gid], g);
    if (g.thread_rank() == 0) st[gid] = s.base();
}

template <class Table>
__global__ void device_mv_read(Table t, const typename Table::key_type *k, uint64_t n,
                               typename Table::value_type *vals, uint64_t per_key, uint64_t *nums)
{
    const auto g = cg::tiled_partition<Table::cg_size()>(cg::this_thread_block());
    const uint64_t gid = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / Table::cg_size();
    if (gid >= n) return;
    typename Table::index_type num = 0, num2 = 0;
    t.num_values(k[gid], num, g);
    t.retrieve(k[gid], vals + gid * per_key, num2, g);
    if (g.thread_rank() == 0) nums[gid] = num == num2 ? num : ~0ull;
}

static void test_multi_value()
{
    using T = wc::MultiValueHashTable<uint64_t, uint64_t>;
    const uint64_t n = 3000;
    T t(4 * n, wc::defaults::seed<uint64_t>(), 3);
    auto keys = distinct_keys<uint64_t>(n + 100, 91);
    std::vector<uint64_t> k(keys.begin(), keys.begin() + n);
    uint64_t *dk = dcopy(k);
    /* host bulk: two rounds with values r * 10^6 + i */
    for (uint64_t r = 0; r < 2; r++) {
        std::vector<uint64_t> v(n);
        for (uint64_t i = 0; i < n; i++) v[i] = r * 1000000 + i;
        uint64_t *dv = dcopy(v);
        t.insert(dk, dv, n);
        cudaFree(dv);
    }
    /* device per-key: a third round, then a fourth that hits max 3 */
    uint32_t *dst;
    cudaMalloc(&dst, sizeof(uint32_t) * n);
    for (uint64_t r = 2; r < 4; r++) {
        std::vector<uint64_t> v(n);
        for (uint64_t i = 0; i < n; i++) v[i] = r * 1000000 + i;
        uint64_t *dv = dcopy(v);
        device_mv_insert<<<blocks_for(n, T::cg_size()), 256>>>(t, dk, dv, n, dst);
        auto st = hcopy(dst, n);
        const uint32_t want = r == 2 ? wc::Status::duplicate_key().base()
                                     : (wc::Status::duplicate_key() + wc::Status::max_values_for_key_reached()).base();
        CHECK(std::all_of(st.begin(), st.end(), [&](uint32_t s) { return s == want; }));
        cudaFree(dv);
    }
    CHECK(t.size() == 3 * n);
    CHECK(t.num_keys() == n);
    /* host bulk retrieve: begin/end offsets and values in insertion order */
    std::vector<uint64_t> q(keys.begin(), keys.end());
    uint64_t *dq = dcopy(q), *db, *de, *dvals;
    cudaMalloc(&db, sizeof(uint64_t) * q.size());
    cudaMalloc(&de, sizeof(uint64_t) * q.size());
    T::index_type num_out = 0;
    t.retrieve(dq, q.size(), db, de, nullptr, num_out);
    CHECK(num_out == 3 * n);
    cudaMalloc(&dvals, sizeof(uint64_t) * num_out);
    t.retrieve(dq, q.size(), db, de, dvals, num_out);
    auto b = hcopy(db, q.size()), e = hcopy(de, q.size()), vals = hcopy(dvals, num_out);
    bool ok = true;
    for (uint64_t i = 0; i < n; i++) {
        ok &= b[i] == 3 * i && e[i] == 3 * i + 3;
        for (uint64_t r = 0; r < 3; r++) ok &= vals[3 * i + r] == r * 1000000 + i;
    }
    for (uint64_t i = n; i < q.size(); i++) ok &= e[i] == b[i];
    CHECK(ok);
    /* device per-key read */
    uint64_t *dvv, *dnums;
    cudaMalloc(&dvv, sizeof(uint64_t) * 3 * n);
    cudaMalloc(&dnums, sizeof(uint64_t) * n);
    device_mv_read<<<blocks_for(n, T::cg_size()), 256>>>(t, dk, n, dvv, 3, dnums);
    auto nums = hcopy(dnums, n);
    auto vv = hcopy(dvv, 3 * n);
    ok = true;
    for (uint64_t i = 0; i < n; i++) {
        ok &= nums[i] == 3;
        for (uint64_t r = 0; r < 3; r++) ok &= vv[3 * i + r] == r * 1000000 + i;
    }
    CHECK(ok);
    /* unique keys */
    T::index_type nk = 0;
    uint64_t *duk;
    cudaMalloc(&duk, sizeof(uint64_t) * n);
    t.retrieve_all_keys(duk, nk);
    auto uk = hcopy(duk, nk);
    std::sort(uk.begin(), uk.end());
    std::sort(k.begin(), k.end());
    CHECK(nk == n && uk == k);
    cudaFree(dk); cudaFree(dst); cudaFree(dq); cudaFree(db); cudaFree(de); cudaFree(dvals);
    cudaFree(dvv); cudaFree(dnums); cudaFree(duk);
}

/* MultiBucketHashTable<u32, u64> with buckets of 2 (the reference example's
 * types): host and device inserts, max_values_per_key, offsets and values
 * in insertion order, device reads, for_each_value / for_each_bucket with
 * device lambdas, unique keys */
static void test_multi_bucket()
{
    using T = wc::MultiBucketHashTable<uint32_t, uint64_t>;
    static_assert(T::bucket_size() == 2, "default bucket of two values");
    const uint64_t n = 3000;
    T t(4 * n, wc::defaults::seed<uint32_t>(), 5);
    auto keys = distinct_keys<uint32_t>(n + 100, 93);
    std::vector<uint32_t> k(keys.begin(), keys.begin() + n);
    uint32_t *dk = dcopy(k);
    auto value = [](uint64_t r, uint64_t i) { return r * 1000000 + i + 1; };
    for (uint64_t r = 0; r < 2; r++) {
        std::vector<uint64_t> v(n);
        for (uint64_t i = 0; i < n; i++) v[i] = value(r, i);
        uint64_t *dv = dcopy(v);
        t.insert(dk, dv, n);
        cudaFree(dv);
    }
    uint32_t *dst;
    cudaMalloc(&dst, sizeof(uint32_t) * n);
    for (uint64_t r = 2; r < 6; r++) {
        std::vector<uint64_t> v(n);
        for (uint64_t i = 0; i < n; i++) v[i] = value(r, i);
        uint64_t *dv = dcopy(v);
        device_mv_insert<<<blocks_for(n, T::cg_size()), 256>>>(t, dk, dv, n, dst);
        auto st = hcopy(dst, n);
        const uint32_t want = r < 5 ? wc::Status::duplicate_key().base()
                                    : (wc::Status::duplicate_key() + wc::Status::max_values_for_key_reached()).base();
        CHECK(std::all_of(st.begin(), st.end(), [&](uint32_t s) { return s == want; }));
        cudaFree(dv);
    }
    CHECK(t.size() == 5 * n);
    CHECK(t.num_keys() == n);
    CHECK(t.num_occupied() == 3 * n);
    CHECK(t.value_capacity() == 2 * t.capacity());
    std::vector<uint32_t> q(keys.begin(), keys.end());
    uint32_t *dq = dcopy(q);
    uint64_t *db, *de, *dvals;
    cudaMalloc(&db, sizeof(uint64_t) * q.size());
    cudaMalloc(&de, sizeof(uint64_t) * q.size());
    T::index_type num_out = 0;
    t.retrieve(dq, q.size(), db, de, nullptr, num_out);
    CHECK(num_out == 5 * n);
    cudaMalloc(&dvals, sizeof(uint64_t) * num_out);
    t.retrieve(dq, q.size(), db, de, dvals, num_out);
    auto b = hcopy(db, q.size()), e = hcopy(de, q.size()), vals = hcopy(dvals, num_out);
    bool ok = true;
    for (uint64_t i = 0; i < n; i++) {
        ok &= b[i] == 5 * i && e[i] == 5 * i + 5;
        for (uint64_t r = 0; r < 5; r++) ok &= vals[5 * i + r] == value(r, i);
    }
    for (uint64_t i = n; i < q.size(); i++) ok &= e[i] == b[i];
    CHECK(ok);
    uint64_t *dvv, *dnums;
    cudaMalloc(&dvv, sizeof(uint64_t) * 5 * n);
    cudaMalloc(&dnums, sizeof(uint64_t) * n);
    device_mv_read<<<blocks_for(n, T::cg_size()), 256>>>(t, dk, n, dvv, 5, dnums);
    auto nums = hcopy(dnums, n);
    auto vv = hcopy(dvv, 5 * n);
    ok = true;
    for (uint64_t i = 0; i < n; i++) {
        ok &= nums[i] == 5;
        for (uint64_t r = 0; r < 5; r++) ok &= vv[5 * i + r] == value(r, i);
    }
    CHECK(ok);
    /* for_each_value: every stored value once; for_each_bucket: every slot */
    unsigned long long *dsum;
    cudaMalloc(&dsum, 2 * sizeof(unsigned long long));
    cudaMemset(dsum, 0, 2 * sizeof(unsigned long long));
    t.for_each_value([=] __device__(uint32_t, uint64_t v) { atomicAdd(dsum, (unsigned long long)v); });
    t.for_each_bucket([=] __device__(uint32_t, const T::bucket_type &) { atomicAdd(dsum + 1, 1ull); });
    auto sums = hcopy(dsum, 2);
    unsigned long long want_sum = 0;
    for (uint64_t i = 0; i < n; i++)
        for (uint64_t r = 0; r < 5; r++) want_sum += value(r, i);
    CHECK(sums[0] == want_sum);
    CHECK(sums[1] == 3 * n);
    T::index_type nk = 0;
    uint32_t *duk;
    cudaMalloc(&duk, sizeof(uint32_t) * n);
    t.retrieve_all_keys(duk, nk);
    auto uk = hcopy(duk, nk);
    std::sort(uk.begin(), uk.end());
    std::sort(k.begin(), k.end());
    CHECK(nk == n && uk == k);
    cudaFree(dk); cudaFree(dst); cudaFree(dq); cudaFree(db); cudaFree(de); cudaFree(dvals);
    cudaFree(dvv); cudaFree(dnums); cudaFree(dsum); cudaFree(duk);
}

template <class Table>
__global__ void device_bl_insert(Table t, const typename Table::key_type *k,
                                 const typename Table::value_type *v, uint64_t n, uint32_t *st)
{
    const auto g = cg::tiled_partition<Table::cg_size()>(cg::this_thread_block());
    const uint64_t gid = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / Table::cg_size();
    if (gid >= n) return;
    const auto s = t.insert(k[gid], v[gid], g);
    if (g.thread_rank() == 0) st[gid] = s.base();
}

template <class Table>
__global__ void device_bl_read(Table t, const typename Table::key_type *k, uint64_t n,
                               typename Table::value_type *vals, uint64_t per_key, uint64_t *nums,
                               unsigned long long *sums)
{
    const auto g = cg::tiled_partition<Table::cg_size()>(cg::this_thread_block());
    const uint64_t gid = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / Table::cg_size();
    if (gid >= n) return;
    typename Table::index_type num = 0, num2 = 0;
    t.num_values(k[gid], num, g);
    t.retrieve(k[gid], vals + gid * per_key, num2, g);
    t.for_each([=](const typename Table::value_type &v, typename Table::index_type) {
        atomicAdd(sums, (unsigned long long)v);
    }, k[gid], g);
    if (g.thread_rank() == 0) nums[gid] = num == num2 ? num : ~0ull;
}

/* list order of values appended 0 .. c-1 (storage.cuh:1292-1343): buckets of
 * min, then ceil(previous * grow) up to max; newest bucket first */
static std::vector<uint64_t> list_order(uint64_t c, uint64_t min_b, float grow, uint64_t max_b)
{
    std::vector<std::pair<uint64_t, uint64_t>> buckets; /* [first, size) */
    uint64_t first = 0, size = min_b;
    while (first < c) {
        buckets.push_back({first, size});
        first += size;
        const float g = std::ceil(float(size) * grow);
        size = uint64_t(float(max_b) < g ? float(max_b) : g);
    }
    std::vector<uint64_t> out;
    for (auto it = buckets.rbegin(); it != buckets.rend(); ++it)
        for (uint64_t j = it->first; j < it->first + it->second && j < c; ++j) out.push_back(j);
    return out;
}

/* BucketListHashTable<u32, u32> (the reference example's types): host and
 * device inserts, lists in bucket order, device reads and for_each,
 * max_values_per_key, unique keys, load factors */
static void test_bucket_list()
{
    using T = wc::BucketListHashTable<uint32_t, uint32_t>;
    const uint64_t n = 3000, rounds = 7;
    T t(2 * n, 40 * n, wc::defaults::seed<uint32_t>(), 1.1f, 1, T::max_bucket_size(), 6);
    auto keys = distinct_keys<uint32_t>(n + 100, 97);
    std::vector<uint32_t> k(keys.begin(), keys.begin() + n);
    uint32_t *dk = dcopy(k);
    auto value = [](uint64_t r, uint64_t i) { return uint32_t(r * 100000 + i + 1); };
    uint32_t *dst;
    cudaMalloc(&dst, sizeof(uint32_t) * n);
    for (uint64_t r = 0; r < rounds; r++) {
        std::vector<uint32_t> v(n);
        for (uint64_t i = 0; i < n; i++) v[i] = value(r, i);
        uint32_t *dv = dcopy(v);
        if (r < 3) {
            t.insert<wc::status_handlers::ReturnStatus>(dk, dv, n, 0, wc::defaults::probing_length(),
                                                        reinterpret_cast<wc::Status *>(dst));
        } else {
            device_bl_insert<<<blocks_for(n, T::cg_size()), 256>>>(t, dk, dv, n, dst);
        }
        auto st = hcopy(dst, n);
        const uint32_t want = r == 0 ? 0u
                              : r < 6 ? wc::Status::duplicate_key().base()
                                      : (wc::Status::duplicate_key() + wc::Status::max_values_for_key_reached()).base();
        CHECK(std::all_of(st.begin(), st.end(), [&](uint32_t s) { return s == want; }));
        cudaFree(dv);
    }
    CHECK(t.num_keys() == n);
    CHECK(t.num_values() == 6 * n);
    std::vector<uint32_t> q(keys.begin(), keys.end());
    uint32_t *dq = dcopy(q), *dvals;
    uint64_t *db, *de;
    cudaMalloc(&db, sizeof(uint64_t) * q.size());
    cudaMalloc(&de, sizeof(uint64_t) * q.size());
    T::index_type num_out = 0;
    t.retrieve(dq, q.size(), db, de, nullptr, num_out);
    CHECK(num_out == 6 * n);
    cudaMalloc(&dvals, sizeof(uint32_t) * num_out);
    t.retrieve(dq, q.size(), db, de, dvals, num_out);
    auto b = hcopy(db, q.size()), e = hcopy(de, q.size());
    auto vals = hcopy(dvals, num_out);
    const auto order = list_order(6, 1, 1.1f, T::max_bucket_size());
    bool ok = true;
    for (uint64_t i = 0; i < n; i++) {
        ok &= b[i] == 6 * i && e[i] == 6 * i + 6;
        for (uint64_t j = 0; j < 6; j++) ok &= vals[6 * i + j] == value(order[j], i);
    }
    for (uint64_t i = n; i < q.size(); i++) ok &= e[i] == b[i];
    CHECK(ok);
    uint32_t *dvv;
    uint64_t *dnums;
    unsigned long long *dsum;
    cudaMalloc(&dvv, sizeof(uint32_t) * 6 * n);
    cudaMalloc(&dnums, sizeof(uint64_t) * n);
    cudaMalloc(&dsum, sizeof(unsigned long long));
    cudaMemset(dsum, 0, sizeof(unsigned long long));
    device_bl_read<<<blocks_for(n, T::cg_size()), 256>>>(t, dk, n, dvv, 6, dnums, dsum);
    auto nums = hcopy(dnums, n);
    auto vv = hcopy(dvv, 6 * n);
    auto sum = hcopy(dsum, 1);
    unsigned long long want_sum = 0;
    ok = true;
    for (uint64_t i = 0; i < n; i++) {
        ok &= nums[i] == 6;
        for (uint64_t j = 0; j < 6; j++) {
            ok &= vv[6 * i + j] == value(order[j], i);
            want_sum += value(j, i);
        }
    }
    CHECK(ok);
    CHECK(sum[0] == want_sum);
    T::index_type nk = 0;
    uint32_t *duk;
    cudaMalloc(&duk, sizeof(uint32_t) * n);
    t.retrieve_all_keys(duk, nk);
    auto uk = hcopy(duk, nk);
    std::sort(uk.begin(), uk.end());
    std::sort(k.begin(), k.end());
    CHECK(nk == n && uk == k);
    CHECK(t.key_load_factor() > 0.f && t.value_load_factor() > 0.f && t.storage_density() > 0.f);
    cudaFree(dk); cudaFree(dst); cudaFree(dq); cudaFree(db); cudaFree(de); cudaFree(dvals);
    cudaFree(dvv); cudaFree(dnums); cudaFree(dsum); cudaFree(duk);
}

int main()
{
    test_svht_u32();
    test_svht_u64_device_api();
    test_svht_soa<uint64_t, uint64_t>(41);
    test_svht_soa<uint32_t, uint32_t>(42);
    test_svht_soa<uint32_t, uint64_t>(43);
    test_hash_set();
    test_counting();
    test_bloom();
    test_filtered_histogram();
    test_mixed_widths();
    test_multi_value();
    test_multi_bucket();
    test_bucket_list();
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e));
        return 2;
    }
    std::printf(g_fail ? "dropin FAILED\n" : "dropin ok\n");
    return g_fail;
}
