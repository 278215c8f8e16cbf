/*
 * Golden-vector generator: drives the REFERENCE warpcore headers (compiled
 * from the reference's own sources by oracle/ref/build_ref.sh) on seeded
 * inputs produced by the C oracle's generators, and dumps inputs' seeds and
 * the reference's outputs as small binary fixtures.
 *
 *   make_golden host <outdir>   hashers, capacity rule, prime table, Status
 *                               algebra, Bloom fpr (runs without a GPU)
 *   make_golden gpu  <outdir>   probe sequences, status handlers, bulk table
 *                               ops and Bloom filter words (needs a GPU)
 *
 * Every fixture is "<name>.bin" (raw little-endian) plus a line in
 * manifest.txt: "<name> <dtype> <count>".
 */
#include <warpcore/single_value_hash_table.cuh>
#include <warpcore/hash_set.cuh>
#include <warpcore/counting_hash_table.cuh>
#include <warpcore/bloom_filter.cuh>
#include <warpcore/multi_value_hash_table.cuh>
#include <warpcore/multi_bucket_hash_table.cuh>
#include <warpcore/bucket_list_hash_table.cuh>
#include <algorithm>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

extern "C" {
#include "wc_oracle.h"
}

namespace wc = warpcore;

static std::string g_out;
static FILE *g_manifest = nullptr;

template <class T>
static const char *dtype_name()
{
    if (sizeof(T) == 1) return "u1";
    if (sizeof(T) == 4) return "u4";
    return "u8";
}

template <class T>
static void dump(const std::string &name, const std::vector<T> &v)
{
    const std::string path = g_out + "/" + name + ".bin";
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) { std::perror(path.c_str()); std::exit(2); }
    if (!v.empty()) std::fwrite(v.data(), sizeof(T), v.size(), f);
    std::fclose(f);
    std::fprintf(g_manifest, "%s %s %zu\n", name.c_str(), dtype_name<T>(), v.size());
}

#define CK(x)                                                                  \
    do {                                                                       \
        cudaError_t e_ = (x);                                                  \
        if (e_ != cudaSuccess) {                                               \
            std::fprintf(stderr, "%s failed: %s (line %d)\n", #x,              \
                         cudaGetErrorString(e_), __LINE__);                    \
            std::exit(3);                                                      \
        }                                                                      \
    } while (0)

template <class T>
static T *to_dev(const std::vector<T> &h)
{
    T *d = nullptr;
    CK(cudaMalloc(&d, sizeof(T) * (h.size() ? h.size() : 1)));
    if (!h.empty()) CK(cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return d;
}

template <class T>
static std::vector<T> to_host(const T *d, size_t n)
{
    std::vector<T> h(n);
    CK(cudaGetLastError()); /* reference launches are unchecked */
    CK(cudaDeviceSynchronize());
    if (n) CK(cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost));
    return h;
}

template <class T>
static std::vector<T> unique_keys(size_t n, uint64_t seed)
{
    std::vector<T> v(n);
    wco_gen_unique_keys(sizeof(T), n, seed, v.data());
    return v;
}

template <class T>
static std::vector<T> uniform(size_t n, uint64_t seed)
{
    std::vector<T> v(n);
    wco_gen_uniform(sizeof(T), n, seed, v.data());
    return v;
}

/* ------------------------------------------------------------------ host */

static void run_host()
{
    /* hashers on seeded inputs plus edge values */
    std::vector<uint64_t> xs = uniform<uint64_t>(256, 7);
    const uint64_t edge[] = {0ull, 1ull, 2ull, 0xffffffffull, 0x100000000ull,
                             0x5ad0dedull, ~0ull, 1ull << 63};
    xs.insert(xs.end(), edge, edge + 8);
    std::vector<uint32_t> m32, nv32, mu32;
    std::vector<uint64_t> m64;
    for (uint64_t x : xs) {
        m32.push_back(wc::hashers::MurmurHash<uint32_t>::hash(uint32_t(x)));
        m64.push_back(wc::hashers::MurmurHash<uint64_t>::hash(uint64_t(x)));
        nv32.push_back(wc::hashers::NvidiaHash::hash(uint32_t(x)));
        mu32.push_back(wc::hashers::MuellerHash::hash(uint32_t(x)));
    }
    dump("hash_inputs", xs);
    dump("hash_murmur32", m32);
    dump("hash_murmur64", m64);
    dump("hash_nvidia32", nv32);
    dump("hash_mueller32", mu32);

    /* capacity rule */
    std::vector<uint64_t> caps_in, caps_out;
    const uint64_t mins[] = {0, 1, 100, 12345, 42424, 6969, 131101, 131102,
                             1048576, 1310720, 4242424, 696969, 19737418,
                             149130808, 2796202, 1073741824ull,
                             137438953472ull, 17177758133ull * 2};
    const uint64_t cgs[] = {1, 2, 4, 8, 16, 32};
    for (uint64_t m : mins)
        for (uint64_t cg : cgs) {
            caps_in.push_back(m);
            caps_in.push_back(cg);
            caps_out.push_back(wc::detail::get_valid_capacity(m, cg));
        }
    dump("capacity_in", caps_in);
    dump("capacity_out", caps_out);

    /* prime table digest */
    uint64_t sum = 0, x = 0;
    for (uint64_t p : wc::detail::primes) { sum += p; x ^= p * 0x9e3779b97f4a7c15ull; }
    std::vector<uint64_t> pd = {uint64_t(wc::detail::primes.size()),
                                wc::detail::primes.front(),
                                wc::detail::primes.back(), sum, x};
    dump("primes_digest", pd);

    /* Status algebra: operator~, masks */
    std::vector<uint32_t> st;
    st.push_back(wc::Status::error_mask().base());
    st.push_back(wc::Status::warning_mask().base());
    for (uint32_t b = 0; b <= 12; b++) {
        const uint32_t s = 1u << b;
        wc::Status cur = wc::Status::none();
        /* build the status through the public factory functions */
        switch (b) {
        case 0: cur = wc::Status::unknown_error(); break;
        case 1: cur = wc::Status::probing_length_exceeded(); break;
        case 2: cur = wc::Status::invalid_configuration(); break;
        case 3: cur = wc::Status::invalid_key(); break;
        case 4: cur = wc::Status::duplicate_key(); break;
        case 5: cur = wc::Status::key_not_found(); break;
        case 6: cur = wc::Status::index_overflow(); break;
        case 7: cur = wc::Status::out_of_memory(); break;
        case 8: cur = wc::Status::not_initialized(); break;
        case 9: cur = wc::Status::dry_run(); break;
        case 10: cur = wc::Status::invalid_phase_overlap(); break;
        case 11: cur = wc::Status::max_values_for_key_reached(); break;
        case 12: cur = wc::Status::invalid_value(); break;
        }
        st.push_back(cur.base());
        st.push_back((~cur).base());
        (void)s;
    }
    st.push_back((~wc::Status::none()).base());
    dump("status_algebra", st);

    /* Bloom fpr (host double) */
    std::vector<uint64_t> fpr_in;
    std::vector<double> fpr_out;
    {
        wc::BloomFilter<uint64_t, wc::hashers::MurmurHash<uint64_t>, uint64_t, 8>
            b(1ull << 32, 8);
        fpr_in.insert(fpr_in.end(), {1ull << 32, 8, 1ull << 28});
        fpr_out.push_back(b.fpr(1ull << 28));
    }
    {
        wc::BloomFilter<uint64_t, wc::hashers::MurmurHash<uint64_t>, uint64_t, 8>
            b(1ull << 20, 8);
        fpr_in.insert(fpr_in.end(), {1ull << 20, 8, 4000});
        fpr_out.push_back(b.fpr(4000));
    }
    {
        wc::BloomFilter<uint64_t> b(1ull << 24, 6);
        fpr_in.insert(fpr_in.end(), {1ull << 24, 6, 1ull << 20});
        fpr_out.push_back(b.fpr(1ull << 20));
    }
    dump("bloom_fpr_in", fpr_in);
    std::vector<uint64_t> bits(fpr_out.size());
    std::memcpy(bits.data(), fpr_out.data(), bits.size() * 8);
    dump("bloom_fpr_out_f64bits", bits);
}

/* ------------------------------------------------------------------- gpu */

template <class Probing>
__global__ void probe_kernel(uint64_t cap, typename Probing::key_type key,
                             typename Probing::key_type seed, uint64_t windows,
                             uint64_t *out)
{
    namespace cg = cooperative_groups;
    const auto group = cg::tiled_partition<Probing::cg_size()>(cg::this_thread_block());
    Probing iter(cap, windows * Probing::cg_size(), group);
    uint64_t o = group.thread_rank();
    for (uint64_t i = iter.begin(key, seed); i != iter.end(); i = iter.next()) {
        out[o] = i;
        o += group.size();
    }
}

template <class Probing>
static void probes(const char *tag, std::vector<uint64_t> &meta,
                   std::vector<uint64_t> &pos)
{
    using K = typename Probing::key_type;
    const uint64_t windows = 12;
    const uint64_t mins[] = {12345, 42424, 6969};
    const K keys[] = {1, 42, 69, 1337};
    const K seeds[] = {5, 42};
    uint64_t *d;
    CK(cudaMalloc(&d, sizeof(uint64_t) * windows * 32));
    for (uint64_t m : mins)
        for (K k : keys)
            for (K s : seeds) {
                const uint64_t cap = wc::detail::get_valid_capacity(m, Probing::cg_size());
                probe_kernel<Probing><<<1, Probing::cg_size()>>>(cap, k, s, windows, d);
                auto h = to_host(d, windows * Probing::cg_size());
                meta.insert(meta.end(), {uint64_t(sizeof(K)), Probing::cg_size(), cap,
                                         uint64_t(k), uint64_t(s), windows});
                pos.insert(pos.end(), h.begin(), h.end());
            }
    CK(cudaFree(d));
    (void)tag;
}

template <class Handler>
__global__ void handler_kernel(const uint32_t *st, uint64_t n,
                               typename Handler::base_type *out)
{
    const uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (i < n) {
        wc::Status s = wc::Status::none();
        /* rebuild the Status from its bits through the public algebra */
        const wc::Status all[] = {
            wc::Status::unknown_error(), wc::Status::probing_length_exceeded(),
            wc::Status::invalid_configuration(), wc::Status::invalid_key(),
            wc::Status::duplicate_key(), wc::Status::key_not_found(),
            wc::Status::index_overflow(), wc::Status::out_of_memory(),
            wc::Status::not_initialized(), wc::Status::dry_run(),
            wc::Status::invalid_phase_overlap(),
            wc::Status::max_values_for_key_reached(), wc::Status::invalid_value()};
        for (int b = 0; b < 13; b++)
            if (st[i] & (1u << b)) s += all[b];
        Handler::handle(s, out, i);
    }
}

template <class Set>
__global__ void set_contains_kernel(const typename Set::key_type *keys, uint64_t n,
                                    bool *flags, uint32_t *status, Set set)
{
    namespace cg = cooperative_groups;
    const uint64_t tid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    const uint64_t gid = tid / Set::cg_size();
    const auto group = cg::tiled_partition<Set::cg_size()>(cg::this_thread_block());
    if (gid < n) {
        bool flag = false;
        const wc::Status s = set.retrieve(keys[gid], flag, group);
        if (group.thread_rank() == 0) {
            if (!s.has_any()) flags[gid] = flag;
            status[gid] = s.base();
        }
    }
}

template <class K, class V>
static void svht_case(const char *tag, uint64_t n, uint64_t min_cap, uint64_t kseed)
{
    using Table = wc::SingleValueHashTable<K, V>;
    using SH = wc::status_handlers::ReturnStatus;
    const std::string p = tag;
    std::vector<K> all = unique_keys<K>(2 * n, kseed);
    std::vector<K> keys(all.begin(), all.begin() + n);
    std::vector<V> vals = uniform<V>(n, kseed + 1);
    /* second batch: the first n/8 keys again with new values, plus invalid keys */
    const uint64_t nd = n / 8;
    std::vector<K> keys2(keys.begin(), keys.begin() + nd);
    std::vector<V> vals2 = uniform<V>(nd, kseed + 2);
    keys2.push_back(K(0));
    vals2.push_back(V(1));
    keys2.push_back(K(~K(0)));
    vals2.push_back(V(2));
    /* queries: inserted and absent keys, interleaved */
    std::vector<K> q;
    for (uint64_t i = 0; i < n; i++) { q.push_back(all[i]); q.push_back(all[n + i]); }
    /* erase every 5th inserted key and a few absent ones */
    std::vector<K> er;
    for (uint64_t i = 0; i < n; i += 5) er.push_back(keys[i]);
    for (uint64_t i = 0; i < 16; i++) er.push_back(all[n + i]);

    Table t(min_cap);
    K *dk = to_dev(keys), *dk2 = to_dev(keys2), *dq = to_dev(q), *de = to_dev(er);
    V *dv = to_dev(vals), *dv2 = to_dev(vals2);
    std::vector<V> fill(q.size(), V(0xA5A5A5A5A5A5A5A5ull));
    V *dout = to_dev(fill);
    wc::Status *dst;
    CK(cudaMalloc(&dst, sizeof(wc::Status) * q.size()));

    t.template insert<SH>(dk, dv, keys.size(), 0, wc::defaults::probing_length(), dst);
    auto st_ins = to_host((uint32_t *)dst, keys.size());
    const uint64_t size1 = t.size();
    const uint32_t status1 = t.pop_status().base();
    t.template insert<SH>(dk2, dv2, keys2.size(), 0, wc::defaults::probing_length(), dst);
    auto st_ins2 = to_host((uint32_t *)dst, keys2.size());
    const uint64_t size2 = t.size();
    const uint32_t status2 = t.pop_status().base();
    t.template retrieve<SH>(dq, q.size(), dout, 0, wc::defaults::probing_length(), dst);
    auto out1 = to_host(dout, q.size());
    auto st_r1 = to_host((uint32_t *)dst, q.size());
    const uint32_t status3 = t.pop_status().base();
    t.template erase<SH>(de, er.size(), 0, wc::defaults::probing_length(), dst);
    auto st_er = to_host((uint32_t *)dst, er.size());
    const uint64_t size3 = t.size();
    const uint32_t status4 = t.pop_status().base();
    CK(cudaMemcpy(dout, fill.data(), sizeof(V) * fill.size(), cudaMemcpyHostToDevice));
    t.template retrieve<SH>(dq, q.size(), dout, 0, wc::defaults::probing_length(), dst);
    auto out2 = to_host(dout, q.size());
    auto st_r2 = to_host((uint32_t *)dst, q.size());
    const uint32_t status5 = t.pop_status().base();

    dump(p + "_meta", std::vector<uint64_t>{n, min_cap, kseed, t.capacity(), size1,
                                            size2, size3, status1, status2, status3,
                                            status4, status5});
    dump(p + "_insert_status", st_ins);
    dump(p + "_insert2_status", st_ins2);
    dump(p + "_retrieve1_values", out1);
    dump(p + "_retrieve1_status", st_r1);
    dump(p + "_erase_status", st_er);
    dump(p + "_retrieve2_values", out2);
    dump(p + "_retrieve2_status", st_r2);
    cudaFree(dk); cudaFree(dk2); cudaFree(dq); cudaFree(de);
    cudaFree(dv); cudaFree(dv2); cudaFree(dout); cudaFree(dst);
}

template <class K>
static void set_case(const char *tag, uint64_t n, uint64_t min_cap, uint64_t kseed)
{
    using Set = wc::HashSet<K>;
    using SH = wc::status_handlers::ReturnStatus;
    const std::string p = tag;
    std::vector<K> all = unique_keys<K>(2 * n, kseed);
    std::vector<K> keys(all.begin(), all.begin() + n);
    std::vector<K> keys2(keys.begin(), keys.begin() + n / 8);
    keys2.push_back(K(0));
    std::vector<K> q;
    for (uint64_t i = 0; i < n; i++) { q.push_back(all[i]); q.push_back(all[n + i]); }
    std::vector<K> er;
    for (uint64_t i = 0; i < n; i += 5) er.push_back(keys[i]);

    Set s(min_cap);
    K *dk = to_dev(keys), *dk2 = to_dev(keys2), *dq = to_dev(q), *de = to_dev(er);
    std::vector<uint8_t> fill(q.size(), 7);
    bool *dflags = (bool *)to_dev(fill);
    uint32_t *dst;
    CK(cudaMalloc(&dst, sizeof(uint32_t) * q.size()));
    s.template insert<SH>(dk, keys.size(), 0, wc::defaults::probing_length(), (wc::Status *)dst);
    auto st_ins = to_host(dst, keys.size());
    const uint64_t size1 = s.size();
    const uint32_t status1 = s.pop_status().base();
    s.template insert<SH>(dk2, keys2.size(), 0, wc::defaults::probing_length(), (wc::Status *)dst);
    auto st_ins2 = to_host(dst, keys2.size());
    const uint32_t status2 = s.pop_status().base();
    const uint64_t blocks = (q.size() * Set::cg_size() + 255) / 256;
    set_contains_kernel<Set><<<blocks, 256>>>(dq, q.size(), dflags, dst, s);
    auto f1 = to_host((uint8_t *)dflags, q.size());
    auto st_r1 = to_host(dst, q.size());
    s.template erase<SH>(de, er.size(), 0, wc::defaults::probing_length(), (wc::Status *)dst);
    auto st_er = to_host(dst, er.size());
    const uint64_t size3 = s.size();
    CK(cudaMemcpy(dflags, fill.data(), fill.size(), cudaMemcpyHostToDevice));
    set_contains_kernel<Set><<<blocks, 256>>>(dq, q.size(), dflags, dst, s);
    auto f2 = to_host((uint8_t *)dflags, q.size());
    auto st_r2 = to_host(dst, q.size());
    const uint32_t status3 = s.pop_status().base();
    dump(p + "_meta", std::vector<uint64_t>{n, min_cap, kseed, s.capacity(), size1,
                                            size3, status1, status2, status3});
    dump(p + "_insert_status", st_ins);
    dump(p + "_insert2_status", st_ins2);
    dump(p + "_contains1", f1);
    dump(p + "_contains1_status", st_r1);
    dump(p + "_erase_status", st_er);
    dump(p + "_contains2", f2);
    dump(p + "_contains2_status", st_r2);
    cudaFree(dk); cudaFree(dk2); cudaFree(dq); cudaFree(de); cudaFree(dflags); cudaFree(dst);
}

template <class V>
static void counting_case(const char *tag, uint64_t distinct, uint64_t occ,
                          uint64_t min_cap, V max_count, uint64_t kseed)
{
    using Table = wc::CountingHashTable<uint32_t, V>;
    using SH = wc::status_handlers::ReturnStatus;
    const std::string p = tag;
    std::vector<uint32_t> all = unique_keys<uint32_t>(distinct + distinct / 4, kseed);
    std::vector<uint64_t> ranks(occ);
    wco_gen_zipf_ranks(distinct, 1.1, occ, kseed + 3, ranks.data());
    std::vector<uint32_t> keys(occ);
    for (uint64_t i = 0; i < occ; i++) keys[i] = all[ranks[i] - 1];
    std::vector<uint32_t> q(all.begin(), all.end());

    Table t(min_cap, wc::defaults::seed<uint32_t>(), max_count);
    uint32_t *dk = to_dev(keys), *dq = to_dev(q);
    std::vector<V> fill(q.size(), V(0xA5A5A5A5A5A5A5A5ull));
    V *dout = to_dev(fill);
    uint32_t *dst;
    CK(cudaMalloc(&dst, sizeof(uint32_t) * q.size()));
    t.insert(dk, keys.size());
    const uint32_t status1 = t.pop_status().base();
    t.template retrieve<SH>(dq, q.size(), dout, 0, wc::defaults::probing_length(), (wc::Status *)dst);
    auto out = to_host(dout, q.size());
    auto st = to_host(dst, q.size());
    const uint64_t size1 = t.size();
    dump(p + "_meta", std::vector<uint64_t>{distinct, occ, min_cap, max_count, kseed,
                                            t.capacity(), size1, status1});
    dump(p + "_counts", out);
    dump(p + "_status", st);
    cudaFree(dk); cudaFree(dq); cudaFree(dout); cudaFree(dst);
}

template <class K, class Slot, uint64_t CG>
static void bloom_case(const char *tag, uint64_t num_bits, uint64_t k, uint64_t n,
                       uint64_t kseed)
{
    using Filter = wc::BloomFilter<K, wc::hashers::MurmurHash<K>, Slot, CG>;
    const std::string p = tag;
    std::vector<K> all = unique_keys<K>(2 * n, kseed);
    std::vector<K> keys(all.begin(), all.begin() + n);
    Filter f(num_bits, k);
    K *dk = to_dev(keys), *dq = to_dev(all);
    bool *dflags;
    CK(cudaMalloc(&dflags, all.size()));
    f.insert(dk, keys.size());
    f.retrieve(dq, all.size(), dflags);
    auto flags = to_host((uint8_t *)dflags, all.size());
    /* BloomFilter keeps its bit vector private and has no accessor; the
     * device pointer is its first data member, so read it from the object. */
    Slot *words_d = nullptr;
    std::vector<Slot> words(f.num_slots());
    std::memcpy(&words_d, &f, sizeof(words_d));
    CK(cudaMemcpy(words.data(), words_d, sizeof(Slot) * words.size(), cudaMemcpyDeviceToHost));
    dump(p + "_meta", std::vector<uint64_t>{sizeof(K), sizeof(Slot), CG, num_bits, k, n,
                                            kseed, f.num_slots(), f.num_blocks()});
    dump(p + "_flags", flags);
    dump(p + "_words", words);
    cudaFree(dk); cudaFree(dq); cudaFree(dflags);
}

/* MultiValueHashTable: five insert rounds of unique keys over shrinking
 * prefixes of one key set (round r stores value r of each key it covers),
 * then a dry-run retrieve, a full retrieve over the keys plus absent ones,
 * and the unique keys.  Keys are unique within a round, so every outcome is
 * deterministic. */
template <class K, class V>
static void mv_case(const char *tag, uint64_t n, uint64_t min_cap, uint64_t kseed,
                    uint64_t max_values)
{
    using Table = wc::MultiValueHashTable<K, V>;
    using SH = wc::status_handlers::ReturnStatus;
    using index_t = wc::index_t;
    const std::string p = tag;
    std::vector<K> all = unique_keys<K>(n + n / 4, kseed);
    std::vector<K> keys(all.begin(), all.begin() + n);
    Table t(min_cap, wc::defaults::seed<K>(), max_values);
    wc::Status *dst;
    CK(cudaMalloc(&dst, sizeof(wc::Status) * (n + n / 4)));
    std::vector<uint32_t> st_rounds;
    std::vector<V> vals_rounds;
    for (uint64_t r = 0; r < 5; r++) {
        const uint64_t m = n - r * (n / 5);
        std::vector<K> kr(keys.begin(), keys.begin() + m);
        std::vector<V> vr = uniform<V>(m, kseed + 10 + r);
        K *dk = to_dev(kr);
        V *dv = to_dev(vr);
        t.template insert<SH>(dk, dv, m, 0, wc::defaults::probing_length(), dst);
        auto st = to_host((uint32_t *)dst, m);
        st_rounds.insert(st_rounds.end(), st.begin(), st.end());
        vals_rounds.insert(vals_rounds.end(), vr.begin(), vr.end());
        cudaFree(dk);
        cudaFree(dv);
    }
    const uint64_t num_keys = t.num_keys();
    const uint64_t size = t.size();
    const uint32_t status1 = t.pop_status().base();
    const uint64_t nq = all.size();
    K *dq = to_dev(all);
    index_t *db, *de;
    CK(cudaMalloc(&db, sizeof(index_t) * nq));
    CK(cudaMalloc(&de, sizeof(index_t) * nq));
    index_t num_dry = 0;
    t.template retrieve<SH>(dq, nq, db, de, nullptr, num_dry, 0, wc::defaults::probing_length(), dst);
    auto counts_dry = to_host((uint64_t *)de, nq);
    auto st_dry = to_host((uint32_t *)dst, nq);
    const uint32_t status2 = t.pop_status().base();
    V *dvals;
    CK(cudaMalloc(&dvals, sizeof(V) * (num_dry ? num_dry : 1)));
    index_t num_out = 0;
    t.template retrieve<SH>(dq, nq, db, de, dvals, num_out, 0, wc::defaults::probing_length(), dst);
    auto begin = to_host((uint64_t *)db, nq);
    auto end = to_host((uint64_t *)de, nq);
    auto values = to_host(dvals, num_out);
    auto st_ret = to_host((uint32_t *)dst, nq);
    const uint32_t status3 = t.pop_status().base();
    K *dku;
    CK(cudaMalloc(&dku, sizeof(K) * (size ? size : 1)));
    index_t num_unique = 0;
    t.retrieve_all_keys(dku, num_unique, 0);
    auto uk = to_host(dku, num_unique);
    std::sort(uk.begin(), uk.end());

    dump(p + "_meta", std::vector<uint64_t>{n, min_cap, kseed, t.capacity(), max_values, num_keys,
                                            size, status1, num_dry, status2, num_out, status3,
                                            num_unique});
    dump(p + "_insert_status", st_rounds);
    dump(p + "_insert_values", vals_rounds);
    dump(p + "_dry_counts", counts_dry);
    dump(p + "_dry_status", st_dry);
    dump(p + "_begin", begin);
    dump(p + "_end", end);
    dump(p + "_values", values);
    dump(p + "_retrieve_status", st_ret);
    dump(p + "_unique_keys_sorted", uk);
    cudaFree(dq); cudaFree(db); cudaFree(de); cudaFree(dvals); cudaFree(dku); cudaFree(dst);
}

/* MultiBucketHashTable<K, V> with AoSStore<K, ArrayBucket<V, B>> (the
 * layout of the reference's multi_bucket benchmark): five insert rounds
 * over shrinking prefixes of the keys (each key's values arrive one per
 * round, so their order is fixed), round 0 with an invalid key and an
 * invalid (empty) value; then counts, a dry run, the two-phase retrieve,
 * num_keys / num_occupied / size and the unique keys. */
template <class K, class V, uint32_t B>
static void mb_case(const char *tag, uint64_t n, uint64_t min_cap, uint64_t kseed,
                    uint64_t max_values)
{
    using Table = wc::MultiBucketHashTable<
        K, V, wc::defaults::empty_key<K>(), wc::defaults::tombstone_key<K>(),
        wc::defaults::empty_key<V>(), wc::defaults::probing_scheme_t<K, 8>,
        wc::storage::key_value::AoSStore<K, wc::ArrayBucket<V, B>>>;
    using SH = wc::status_handlers::ReturnStatus;
    using index_t = wc::index_t;
    const std::string p = tag;
    std::vector<K> all = unique_keys<K>(n + n / 4, kseed);
    std::vector<K> keys(all.begin(), all.begin() + n);
    Table t(min_cap, wc::defaults::seed<K>(), max_values);
    wc::Status *dst;
    CK(cudaMalloc(&dst, sizeof(wc::Status) * (n + n / 4)));
    std::vector<uint32_t> st_rounds;
    std::vector<K> keys_rounds;
    std::vector<V> vals_rounds;
    for (uint64_t r = 0; r < 5; r++) {
        const uint64_t m = n - r * (n / 5);
        std::vector<K> kr(keys.begin(), keys.begin() + m);
        std::vector<V> vr = uniform<V>(m, kseed + 10 + r);
        for (auto &v : vr)
            if (v == V(0)) v = V(1);
        if (r == 0) {
            kr[11] = wc::defaults::tombstone_key<K>();
            vr[7] = V(0);
        }
        K *dk = to_dev(kr);
        V *dv = to_dev(vr);
        t.template insert<SH>(dk, dv, m, 0, wc::defaults::probing_length(), dst);
        auto st = to_host((uint32_t *)dst, m);
        st_rounds.insert(st_rounds.end(), st.begin(), st.end());
        keys_rounds.insert(keys_rounds.end(), kr.begin(), kr.end());
        vals_rounds.insert(vals_rounds.end(), vr.begin(), vr.end());
        cudaFree(dk);
        cudaFree(dv);
    }
    const uint64_t num_keys = t.num_keys();
    const uint64_t num_occupied = t.num_occupied();
    const uint64_t size = t.size();
    const uint32_t status1 = t.pop_status().base();
    const uint64_t nq = all.size();
    K *dq = to_dev(all);
    index_t *db, *de;
    CK(cudaMalloc(&db, sizeof(index_t) * nq));
    CK(cudaMalloc(&de, sizeof(index_t) * nq));
    index_t num_dry = 0;
    t.template retrieve<SH>(dq, nq, db, de, nullptr, num_dry, 0, wc::defaults::probing_length(), dst);
    auto counts_dry = to_host((uint64_t *)de, nq);
    auto st_dry = to_host((uint32_t *)dst, nq);
    const uint32_t status2 = t.pop_status().base();
    V *dvals;
    CK(cudaMalloc(&dvals, sizeof(V) * (num_dry ? num_dry : 1)));
    index_t num_out = 0;
    t.template retrieve<SH>(dq, nq, db, de, dvals, num_out, 0, wc::defaults::probing_length(), dst);
    auto begin = to_host((uint64_t *)db, nq);
    auto end = to_host((uint64_t *)de, nq);
    auto values = to_host(dvals, num_out);
    auto st_ret = to_host((uint32_t *)dst, nq);
    const uint32_t status3 = t.pop_status().base();
    K *dku;
    CK(cudaMalloc(&dku, sizeof(K) * (num_occupied ? num_occupied : 1)));
    index_t num_unique = 0;
    t.retrieve_all_keys(dku, num_unique, 0);
    auto uk = to_host(dku, num_unique);
    std::sort(uk.begin(), uk.end());

    dump(p + "_meta", std::vector<uint64_t>{n, min_cap, kseed, t.capacity(), B, max_values,
                                            num_keys, num_occupied, size, status1, num_dry,
                                            status2, num_out, status3, num_unique,
                                            t.value_capacity()});
    dump(p + "_insert_keys", keys_rounds);
    dump(p + "_insert_values", vals_rounds);
    dump(p + "_insert_status", st_rounds);
    dump(p + "_dry_counts", counts_dry);
    dump(p + "_dry_status", st_dry);
    dump(p + "_begin", begin);
    dump(p + "_end", end);
    dump(p + "_values", values);
    dump(p + "_retrieve_status", st_ret);
    dump(p + "_unique_keys_sorted", uk);
    cudaFree(dq); cudaFree(db); cudaFree(de); cudaFree(dvals); cudaFree(dku); cudaFree(dst);
}

/* BucketListHashTable<K, V> over BucketListStore<V, IB, CB, SB>: eight
 * insert rounds over shrinking prefixes of n keys (one value per key per
 * round, so each key's list is built in a fixed order; every batch a
 * multiple of 128 keys, the bulk insert's groups per block), round 0 with an
 * invalid key; then counts, a dry run, the two-phase retrieve, num_keys,
 * num_values, the value load factor and all keys.  exhaust_after >= 0 sizes
 * the value pool to what the oracle's rounds 0 .. exhaust_after use, so
 * every later bucket allocation fails (out_of_memory) whatever the order.
 * The status buffer starts at 0xffffffff: the reference writes no status
 * for a key that found no slot. */
template <class K, class V, uint64_t IB, uint64_t CB, uint64_t SB>
static void bl_case(const char *tag, uint64_t n, uint64_t key_cap, uint64_t value_cap,
                    float grow, uint64_t min_b, uint64_t max_b, uint64_t max_values,
                    uint64_t kseed, int exhaust_after)
{
    using Store = wc::storage::multi_value::BucketListStore<V, IB, CB, SB>;
    using Table = wc::BucketListHashTable<K, V, wc::defaults::empty_key<K>(),
                                          wc::defaults::tombstone_key<K>(), Store,
                                          wc::defaults::probing_scheme_t<K, 8>>;
    using SH = wc::status_handlers::ReturnStatus;
    using index_t = wc::index_t;
    const std::string p = tag;
    std::vector<K> all = unique_keys<K>(n + n / 4, kseed);
    std::vector<K> keys(all.begin(), all.begin() + n);
    std::vector<std::vector<K>> rk;
    std::vector<std::vector<V>> rv;
    for (uint64_t r = 0; r < 8; r++) {
        const uint64_t m = n - r * (n / 8);
        std::vector<K> kr(keys.begin(), keys.begin() + m);
        std::vector<V> vr = uniform<V>(m, kseed + 10 + r);
        if (r == 0) kr[11] = wc::defaults::tombstone_key<K>();
        rk.push_back(kr);
        rv.push_back(vr);
    }
    if (exhaust_after >= 0) {
        wco_bl *o = wco_bl_create(sizeof(K), sizeof(V), key_cap, uint64_t(1) << 22, 0x5ad0ded,
                                  grow, min_b, max_b, max_values, IB, CB, SB, 8);
        for (int r = 0; r <= exhaust_after; r++)
            wco_bl_insert(o, rk[r].data(), rv[r].data(), rk[r].size(), ~0ull - 1024, nullptr);
        value_cap = wco_bl_next_free(o);
        wco_bl_destroy(o);
    }
    Table t(key_cap, value_cap, wc::defaults::seed<K>(), grow, min_b, max_b, max_values);
    wc::Status *dst;
    CK(cudaMalloc(&dst, sizeof(wc::Status) * (n + n / 4)));
    std::vector<uint32_t> st_rounds;
    std::vector<K> keys_rounds;
    std::vector<V> vals_rounds;
    for (uint64_t r = 0; r < 8; r++) {
        const uint64_t m = rk[r].size();
        K *dk = to_dev(rk[r]);
        V *dv = to_dev(rv[r]);
        CK(cudaMemset(dst, 0xff, sizeof(wc::Status) * m));
        t.template insert<SH>(dk, dv, m, 0, wc::defaults::probing_length(), dst);
        auto st = to_host((uint32_t *)dst, m);
        st_rounds.insert(st_rounds.end(), st.begin(), st.end());
        keys_rounds.insert(keys_rounds.end(), rk[r].begin(), rk[r].end());
        vals_rounds.insert(vals_rounds.end(), rv[r].begin(), rv[r].end());
        cudaFree(dk);
        cudaFree(dv);
    }
    const uint64_t num_keys = t.num_keys();
    const uint64_t num_values = t.num_values();
    const float vlf = t.value_load_factor();
    uint32_t vlf_bits;
    std::memcpy(&vlf_bits, &vlf, 4);
    const uint32_t status1 = t.pop_status().base();
    const uint64_t nq = all.size();
    K *dq = to_dev(all);
    index_t *db, *de;
    CK(cudaMalloc(&db, sizeof(index_t) * nq));
    CK(cudaMalloc(&de, sizeof(index_t) * nq));
    index_t num_dry = 0;
    t.template retrieve<SH>(dq, nq, db, de, nullptr, num_dry, 0, wc::defaults::probing_length(), dst);
    auto counts_dry = to_host((uint64_t *)de, nq);
    auto st_dry = to_host((uint32_t *)dst, nq);
    const uint32_t status2 = t.pop_status().base();
    V *dvals;
    CK(cudaMalloc(&dvals, sizeof(V) * (num_dry ? num_dry : 1)));
    /* a list whose pool ran out is not read (storage.cuh:1304): its part of
     * the output keeps this fill */
    CK(cudaMemset(dvals, 0xff, sizeof(V) * (num_dry ? num_dry : 1)));
    index_t num_out = 0;
    t.template retrieve<SH>(dq, nq, db, de, dvals, num_out, 0, wc::defaults::probing_length(), dst);
    auto begin = to_host((uint64_t *)db, nq);
    auto end = to_host((uint64_t *)de, nq);
    auto values = to_host(dvals, num_out);
    auto st_ret = to_host((uint32_t *)dst, nq);
    const uint32_t status3 = t.pop_status().base();
    K *dku;
    CK(cudaMalloc(&dku, sizeof(K) * (num_keys ? num_keys : 1)));
    index_t num_all = 0;
    t.retrieve_all_keys(dku, num_all, 0);
    auto ak = to_host(dku, num_all);
    std::sort(ak.begin(), ak.end());

    dump(p + "_meta", std::vector<uint64_t>{n, key_cap, value_cap, t.key_capacity(),
                                            t.value_capacity(), uint64_t(grow * 1000.0f + 0.5f),
                                            min_b, max_b, max_values, IB, CB, SB, num_keys,
                                            num_values, vlf_bits, status1, num_dry, status2,
                                            num_out, status3, num_all, kseed});
    dump(p + "_insert_keys", keys_rounds);
    dump(p + "_insert_values", vals_rounds);
    dump(p + "_insert_status", st_rounds);
    dump(p + "_dry_counts", counts_dry);
    dump(p + "_dry_status", st_dry);
    dump(p + "_begin", begin);
    dump(p + "_end", end);
    dump(p + "_values", values);
    dump(p + "_retrieve_status", st_ret);
    dump(p + "_all_keys_sorted", ak);
    cudaFree(dq); cudaFree(db); cudaFree(de); cudaFree(dvals); cudaFree(dku); cudaFree(dst);
}

static void run_gpu()
{
    namespace ps = wc::probing_schemes;
    namespace hs = wc::hashers;
    {
        std::vector<uint64_t> meta, pos;
        probes<ps::DoubleHashing<hs::MurmurHash<uint32_t>, hs::MurmurHash<uint32_t>, 1>>("d", meta, pos);
        probes<ps::DoubleHashing<hs::MurmurHash<uint32_t>, hs::MurmurHash<uint32_t>, 2>>("d", meta, pos);
        probes<ps::DoubleHashing<hs::MurmurHash<uint32_t>, hs::MurmurHash<uint32_t>, 4>>("d", meta, pos);
        probes<ps::DoubleHashing<hs::MurmurHash<uint32_t>, hs::MurmurHash<uint32_t>, 8>>("d", meta, pos);
        probes<ps::DoubleHashing<hs::MurmurHash<uint32_t>, hs::MurmurHash<uint32_t>, 16>>("d", meta, pos);
        probes<ps::DoubleHashing<hs::MurmurHash<uint32_t>, hs::MurmurHash<uint32_t>, 32>>("d", meta, pos);
        probes<ps::DoubleHashing<hs::MurmurHash<uint64_t>, hs::MurmurHash<uint64_t>, 8>>("d", meta, pos);
        probes<ps::DoubleHashing<hs::MurmurHash<uint64_t>, hs::MurmurHash<uint64_t>, 16>>("d", meta, pos);
        dump("probe_double_meta", meta);
        dump("probe_double_pos", pos);
    }
    {
        std::vector<uint64_t> meta, pos;
        probes<ps::LinearProbing<hs::MurmurHash<uint32_t>, 1>>("l", meta, pos);
        probes<ps::LinearProbing<hs::MurmurHash<uint32_t>, 8>>("l", meta, pos);
        probes<ps::LinearProbing<hs::MurmurHash<uint32_t>, 32>>("l", meta, pos);
        dump("probe_linear_meta", meta);
        dump("probe_linear_pos", pos);
    }
    {
        std::vector<uint64_t> meta, pos;
        probes<ps::QuadraticProbing<hs::MurmurHash<uint32_t>, 4>>("q", meta, pos);
        probes<ps::QuadraticProbing<hs::MurmurHash<uint32_t>, 8>>("q", meta, pos);
        dump("probe_quadratic_meta", meta);
        dump("probe_quadratic_pos", pos);
    }
    {
        /* every subset of the 13 status bits that matters: singles and pairs */
        std::vector<uint32_t> st;
        for (uint32_t a = 0; a <= 12; a++) {
            st.push_back(1u << a);
            for (uint32_t b = a + 1; b <= 12; b++) st.push_back((1u << a) | (1u << b));
        }
        st.push_back(0);
        uint32_t *dst = to_dev(st);
        bool *dout;
        CK(cudaMalloc(&dout, st.size()));
        const uint64_t blocks = (st.size() + 127) / 128;
        handler_kernel<wc::status_handlers::ReturnBoolean<0>><<<blocks, 128>>>(dst, st.size(), dout);
        auto b0 = to_host((uint8_t *)dout, st.size());
        handler_kernel<wc::status_handlers::ReturnBoolean<(1u << 5)>><<<blocks, 128>>>(dst, st.size(), dout);
        auto b1 = to_host((uint8_t *)dout, st.size());
        handler_kernel<wc::status_handlers::ReturnBoolean<(1u << 4) | (1u << 5)>><<<blocks, 128>>>(dst, st.size(), dout);
        auto b2 = to_host((uint8_t *)dout, st.size());
        dump("handler_status_in", st);
        dump("handler_bool_ignore_none", b0);
        dump("handler_bool_ignore_notfound", b1);
        dump("handler_bool_ignore_dup_notfound", b2);
        cudaFree(dst); cudaFree(dout);
    }
    svht_case<uint32_t, uint32_t>("svht_u32u32", 20000, 25000, 11);
    svht_case<uint64_t, uint64_t>("svht_u64u64", 20000, 25000, 21);
    set_case<uint64_t>("set_u64", 20000, 25000, 31);
    set_case<uint32_t>("set_u32", 20000, 25000, 41);
    counting_case<uint32_t>("count_u32", 5000, 200000, 6000, 0xffffffffu, 51);
    counting_case<uint32_t>("count_u32_max10", 5000, 200000, 6000, 10u, 52);
    counting_case<uint64_t>("count_u32u64", 5000, 200000, 6000, ~uint64_t(0), 53);
    counting_case<uint64_t>("count_u32u64_max10", 5000, 200000, 6000, uint64_t(10), 54);
    svht_case<uint32_t, uint64_t>("svht_u32u64", 20000, 25000, 12);
    svht_case<uint64_t, uint32_t>("svht_u64u32", 20000, 25000, 22);
    bloom_case<uint64_t, uint64_t, 8>("bloom_u64_s64_cg8", 1ull << 16, 8, 4000, 61);
    bloom_case<uint64_t, uint64_t, 1>("bloom_u64_s64_cg1", (1ull << 16) + 100, 6, 3000, 62);
    bloom_case<uint32_t, uint32_t, 4>("bloom_u32_s32_cg4", 3000, 5, 300, 63);
    bloom_case<uint32_t, uint64_t, 2>("bloom_u32_s64_cg2", 5000, 3, 400, 64);
    mv_case<uint32_t, uint32_t>("mv_u32u32_max3", 4000, 16000, 71, 3);
    mv_case<uint64_t, uint64_t>("mv_u64u64", 4000, 16000, 72, ~uint64_t(0));
    mv_case<uint32_t, uint64_t>("mv_u32u64_max3", 4000, 16000, 73, 3);
    mv_case<uint64_t, uint32_t>("mv_u64u32", 4000, 16000, 74, ~uint64_t(0));
    mb_case<uint32_t, uint32_t, 1>("mb_u32u32_b1", 4000, 16000, 81, ~uint64_t(0));
    mb_case<uint32_t, uint32_t, 2>("mb_u32u32_b2", 4000, 16000, 82, ~uint64_t(0));
    mb_case<uint32_t, uint32_t, 2>("mb_u32u32_b2_max3", 4000, 16000, 83, 3);
    mb_case<uint32_t, uint32_t, 4>("mb_u32u32_b4_max6", 4000, 8000, 84, 6);
    mb_case<uint32_t, uint32_t, 8>("mb_u32u32_b8", 4000, 8000, 85, ~uint64_t(0));
    mb_case<uint32_t, uint64_t, 2>("mb_u32u64_b2", 4000, 16000, 86, ~uint64_t(0));
    mb_case<uint64_t, uint64_t, 4>("mb_u64u64_b4_max2", 4000, 16000, 87, 2);
    bl_case<uint32_t, uint32_t, 32, 20, 10>("bl_u32u32", 4096, 5120, 65536, 1.1f, 1, 1023,
                                            (1u << 20) - 1, 91, -1);
    bl_case<uint32_t, uint32_t, 29, 18, 15>("bl_u32u32_bench_bits_max6", 4096, 5120, 65536, 1.1f, 1,
                                            (1u << 15) - 1, 6, 92, -1);
    bl_case<uint32_t, uint32_t, 32, 20, 10>("bl_u32u32_min2_grow15_max4", 4096, 5120, 65536, 1.5f,
                                            2, 4, (1u << 20) - 1, 93, -1);
    bl_case<uint64_t, uint64_t, 32, 20, 10>("bl_u64u64", 4096, 5120, 65536, 1.1f, 1, 1023,
                                            (1u << 20) - 1, 94, -1);
    bl_case<uint32_t, uint32_t, 32, 20, 10>("bl_u32u32_oom", 4096, 5120, 0, 1.1f, 1, 1023,
                                            (1u << 20) - 1, 95, 2);
}

int main(int argc, char **argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s host|gpu <outdir>\n", argv[0]);
        return 1;
    }
    g_out = argv[2];
    const std::string mpath = g_out + "/manifest_" + argv[1] + ".txt";
    g_manifest = std::fopen(mpath.c_str(), "w");
    if (!g_manifest) { std::perror(mpath.c_str()); return 2; }
    if (std::strcmp(argv[1], "host") == 0) run_host();
    else run_gpu();
    std::fclose(g_manifest);
    std::printf("fixtures written to %s\n", g_out.c_str());
    return 0;
}
