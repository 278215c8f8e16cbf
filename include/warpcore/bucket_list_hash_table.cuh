/*
 * warpcore::BucketListHashTable -- drop-in for the reference class
 * (bucket_list_hash_table.cuh:17-893) over the B200-native library.  Host
 * bulk methods call the C ABI (wc_blht_*).  The device per-key methods
 * (insert / retrieve / num_values / for_each with a cooperative group of
 * cg_size() threads) run the bulk kernels' per-key code
 * (detail/bl_ops.cuh) on the group's first thread and hand the result to
 * every thread of the group.  The value store parameter names the handle
 * bit widths (storage::multi_value::BucketListStore).  Objects are passed to
 * user kernels by value; copies are shallow, as in the reference.
 */
#ifndef WARPCORE_B200_CXX_BLHT_CUH
#define WARPCORE_B200_CXX_BLHT_CUH

#include "base.cuh"
#include "detail/bl_ops.cuh"

namespace warpcore {

template <class Key, class Value, Key EmptyKey = defaults::empty_key<Key>(),
          Key TombstoneKey = defaults::tombstone_key<Key>(),
          class ValueStore = defaults::value_storage_t<Value>,
          class ProbingScheme = defaults::probing_scheme_t<Key, 8>>
class BucketListHashTable {
    static_assert(checks::is_valid_key_type<Key>(), "invalid key type");
    static_assert(EmptyKey != TombstoneKey, "empty key and tombstone key must not be identical");
    static_assert(checks::is_probing_scheme<ProbingScheme>(), "not a valid probing scheme type");
    static_assert(std::is_same<typename ProbingScheme::key_type, Key>::value,
                  "probing key type differs from table's key type");
    static_assert(std::is_same<typename ValueStore::tag, tags::dynamic_value_storage>::value,
                  "not a valid storage type");
    static_assert((sizeof(Value) == 4 || sizeof(Value) == 8) && std::is_integral<Value>::value,
                  "this build stores 4- or 8-byte integral values");

    using K = typename std::make_unsigned<Key>::type;
    using V = typename std::make_unsigned<Value>::type;
    static constexpr int kW = int(ProbingScheme::cg_size());

  public:
    using handle_type = typename ValueStore::handle_type;
    using key_type = Key;
    using value_type = Value;
    using index_type = index_t;
    using status_type = Status;

    __host__ __device__ static constexpr key_type empty_key() noexcept { return EmptyKey; }
    __host__ __device__ static constexpr key_type tombstone_key() noexcept { return TombstoneKey; }
    __host__ __device__ static constexpr bool is_valid_key(const key_type key) noexcept
    {
        return key != empty_key() && key != tombstone_key();
    }
    __host__ __device__ static constexpr index_type cg_size() noexcept { return ProbingScheme::cg_size(); }
    __host__ __device__ static constexpr index_type max_bucket_size() noexcept
    {
        return handle_type::max_bucket_size();
    }

    /* bucket_list_hash_table.cuh:106-121 */
    explicit BucketListHashTable(const index_type key_capacity, const index_type value_capacity,
                                 const key_type seed = defaults::seed<key_type>(),
                                 const float grow_factor = 1.1,
                                 const index_type min_bucket_size = 1,
                                 const index_type max_bucket_size = BucketListHashTable::max_bucket_size(),
                                 const index_type max_values_per_key = handle_type::max_value_count(),
                                 const bool no_init = false) noexcept
    {
        wc_table_config cfg =
            detail::make_config<ProbingScheme, Key>(sizeof(Value), EmptyKey, TombstoneKey);
        if (wc_blht_create(&cfg, key_capacity, value_capacity, std::uint64_t(seed), grow_factor,
                           min_bucket_size, max_bucket_size, max_values_per_key,
                           std::uint32_t(ValueStore::bucket_index_bits()),
                           std::uint32_t(ValueStore::value_counter_bits()),
                           std::uint32_t(ValueStore::bucket_size_bits()), no_init ? 1 : 0,
                           &handle_) == WC_OK)
            refresh();
    }

    __host__ __device__ BucketListHashTable(const BucketListHashTable &o) noexcept
        : handle_(o.handle_), view_(o.view_), is_initialized_(o.is_initialized_), is_copy_(true)
    {}

    BucketListHashTable(BucketListHashTable &&o) noexcept
        : handle_(o.handle_), view_(o.view_), is_initialized_(o.is_initialized_),
          is_copy_(o.is_copy_)
    {
        o.is_copy_ = true;
    }

#ifndef __CUDA_ARCH__
    ~BucketListHashTable() noexcept
    {
        if (!is_copy_ && handle_) wc_blht_destroy(handle_);
    }
#endif

    /* init (:160-186) */
    void init(const key_type seed, const cudaStream_t stream = 0) noexcept
    {
        if (handle_ && wc_blht_init(handle_, std::uint64_t(seed), stream_of(stream)) == WC_OK)
            refresh();
    }
    void init(const cudaStream_t stream = 0) noexcept { init(key_type(view_.t.seed), stream); }

    /* device insert (:187-222) */
    __device__ status_type insert(const key_type key_in, const value_type &value_in,
                                  const cg::thread_block_tile<cg_size()> &group,
                                  const index_type probing_length = defaults::probing_length()) noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        std::uint32_t st = 0;
        if (group.thread_rank() == 0) {
            std::uint32_t join = 0;
            st = b200::bl_insert_one<K, V, kW>(
                view_, K(key_in), V(value_in),
                b200::max_windows(probing_length, cg_size(), view_.t.num_buckets), join);
            b200::join_status(view_.t.status, join);
        }
        return status_type(group.shfl(st, 0));
    }

    /* host insert (:235-326); every key gets its status */
    template <class StatusHandler = defaults::status_handler_t>
    void insert(const key_type *const keys_in, const value_type *const values_in,
                const index_type num_in, const cudaStream_t stream = 0,
                const index_type probing_length = defaults::probing_length(),
                typename StatusHandler::base_type *const status_out = nullptr) noexcept
    {
        static_assert(checks::is_status_handler<StatusHandler>(), "not a valid status handler type");
        if (!is_initialized_) return;
        wc_blht_insert(handle_, keys_in, values_in, num_in, stream_of(stream), probing_length,
                       (void *)status_out, StatusHandler::kId, StatusHandler::kIgnore);
    }

    /* device for_each over one key's list (:507-521): f(value, index) */
    template <class Func>
    __device__ status_type for_each(Func f, const key_type key_in,
                                    const cg::thread_block_tile<cg_size()> &group,
                                    const index_type probing_length = defaults::probing_length()) const noexcept
    {
        index_type num = 0;
        return walk(f, key_in, num, group, probing_length);
    }

    /* device retrieve (:337-371): values in list order, num_out its length */
    __device__ status_type retrieve(const key_type key_in, value_type *const values_out,
                                    index_type &num_out,
                                    const cg::thread_block_tile<cg_size()> &group,
                                    const index_type probing_length = defaults::probing_length()) const noexcept
    {
        return walk([=](const value_type &v, index_type j) { values_out[j] = v; }, key_in,
                    num_out, group, probing_length);
    }

    /* device num_values (:740-757) */
    __device__ status_type num_values(const key_type key_in, index_type &num_out,
                                      const cg::thread_block_tile<cg_size()> &group,
                                      const index_type probing_length = defaults::probing_length()) const noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        std::uint32_t st = 0;
        std::uint64_t num = 0;
        if (group.thread_rank() == 0) {
            st = b200::bl_for_each_one<K, V, kW, false>(
                view_, K(key_in), b200::max_windows(probing_length, cg_size(), view_.t.num_buckets),
                num, [](V, std::uint64_t) {});
            if (st) b200::join_status(view_.t.status, st);
        }
        num_out = group.shfl(num, 0);
        return status_type(group.shfl(st, 0));
    }

    /* host retrieve (:375-466): offsets are index_type (uint64); values_out
     * NULL is a dry run leaving the per-key counts in end_offsets_out */
    template <class StatusHandler = defaults::status_handler_t>
    void retrieve(const key_type *const keys_in, const index_type num_in,
                  index_type *const begin_offsets_out, index_type *const end_offsets_out,
                  value_type *const values_out, index_type &num_out,
                  const cudaStream_t stream = 0,
                  const index_type probing_length = defaults::probing_length(),
                  typename StatusHandler::base_type *const status_out = nullptr) const noexcept
    {
        static_assert(checks::is_status_handler<StatusHandler>(), "not a valid status handler type");
        num_out = 0;
        if (!is_initialized_) return;
        std::uint64_t n = 0;
        if (wc_blht_retrieve(handle_, keys_in, num_in, (std::uint64_t *)begin_offsets_out,
                             (std::uint64_t *)end_offsets_out, values_out, &n, stream_of(stream),
                             probing_length, (void *)status_out, StatusHandler::kId,
                             StatusHandler::kIgnore) == WC_OK)
            num_out = n;
    }

    /* retrieve_all (:537-565) */
    void retrieve_all(key_type *const keys_out, index_type &num_keys_out,
                      index_type *const begin_offsets_out, index_type *const end_offsets_out,
                      value_type *const values_out, value_type &num_values_out,
                      const cudaStream_t stream = 0) const noexcept
    {
        num_values_out = 0;
        retrieve_all_keys(keys_out, num_keys_out, stream);
        if (keys_out != nullptr) {
            index_type n = 0;
            retrieve(keys_out, num_keys_out, begin_offsets_out, end_offsets_out, values_out, n,
                     stream);
            num_values_out = value_type(n);
        }
    }

    /* retrieve_all_keys (:574-605); keys_out NULL gives num_keys() */
    void retrieve_all_keys(key_type *const keys_out, index_type &num_out,
                           const cudaStream_t stream = 0) const noexcept
    {
        num_out = 0;
        if (!is_initialized_) return;
        std::uint64_t n = 0;
        if (wc_blht_retrieve_all_keys(handle_, keys_out, &n, stream_of(stream)) == WC_OK)
            num_out = n;
    }

    /* host num_values (:776-800) and the table total (:797-818) */
    template <class StatusHandler = defaults::status_handler_t>
    void num_values(const key_type *const keys_in, const index_type num_in, index_type &num_out,
                    index_type *const num_per_key_out = nullptr, const cudaStream_t stream = 0,
                    const index_type probing_length = defaults::probing_length(),
                    typename StatusHandler::base_type *const status_out = nullptr) const noexcept
    {
        num_out = 0;
        if (!is_initialized_) return;
        std::uint64_t n = 0;
        if (wc_blht_num_values(handle_, keys_in, num_in, &n, (std::uint64_t *)num_per_key_out,
                               stream_of(stream), probing_length, (void *)status_out,
                               StatusHandler::kId, StatusHandler::kIgnore) == WC_OK)
            num_out = n;
    }
    index_type num_values(const cudaStream_t stream = 0) const noexcept
    {
        std::uint64_t n = 0;
        if (is_initialized_) wc_blht_total_values(handle_, stream_of(stream), &n);
        return n;
    }
    index_type num_keys(const cudaStream_t stream = 0) const noexcept
    {
        std::uint64_t n = 0;
        if (is_initialized_) wc_blht_num_keys(handle_, stream_of(stream), &n);
        return n;
    }

    /* load factors, byte counts and densities (:611-700) */
    float key_load_factor(const cudaStream_t stream = 0) const noexcept
    {
        return float(num_keys(stream)) / float(key_capacity());
    }
    float value_load_factor(const cudaStream_t stream = 0) const noexcept
    {
        std::uint64_t used = 0;
        if (is_initialized_) wc_blht_pool_used(handle_, stream_of(stream), &used);
        return float(used) / float(value_capacity());
    }
    index_type bytes_total() const noexcept { return info().bytes_total; }
    index_type bytes_keys(const cudaStream_t stream = 0) const noexcept
    {
        return num_keys(stream) * sizeof(key_type);
    }
    index_type bytes_values(const cudaStream_t stream = 0) const noexcept
    {
        return num_values(stream) * sizeof(value_type);
    }
    index_type bytes_payload(const cudaStream_t stream = 0) const noexcept
    {
        return bytes_keys(stream) + bytes_values(stream);
    }
    float storage_density(const cudaStream_t stream = 0) const noexcept
    {
        return float(bytes_payload(stream)) / float(bytes_total());
    }
    float relative_storage_density(const cudaStream_t stream = 0) const noexcept
    {
        std::uint64_t used = 0;
        if (is_initialized_) wc_blht_pool_used(handle_, stream_of(stream), &used);
        const float table = float(key_capacity()) * float(sizeof(key_type) + 8);
        return float(bytes_payload(stream)) / (float(used) * 8.0f + table);
    }

    __host__ __device__ bool is_initialized() const noexcept { return is_initialized_; }
    status_type peek_status(const cudaStream_t stream = 0) const noexcept
    {
        std::uint32_t s = WC_STATUS_NOT_INITIALIZED;
        if (handle_) wc_blht_peek_status(handle_, stream_of(stream), &s);
        return status_type(s);
    }
    status_type pop_status(const cudaStream_t stream = 0) noexcept
    {
        std::uint32_t s = WC_STATUS_NOT_INITIALIZED;
        if (handle_) wc_blht_pop_status(handle_, stream_of(stream), &s);
        return status_type(s);
    }
    index_type key_capacity() const noexcept { return info().key_capacity; }
    index_type value_capacity() const noexcept { return info().value_capacity; }
    __host__ __device__ bool is_copy() const noexcept { return is_copy_; }
    __host__ __device__ const b200::BlView &device_view() const noexcept { return view_; }
    wc_blht *handle() const noexcept { return handle_; }

  private:
    template <class Func>
    __device__ status_type walk(Func f, const key_type key_in, index_type &num_out,
                                const cg::thread_block_tile<cg_size()> &group,
                                const index_type probing_length) const noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        std::uint32_t st = 0;
        std::uint64_t num = 0;
        if (group.thread_rank() == 0) {
            st = b200::bl_for_each_one<K, V, kW, true>(
                view_, K(key_in), b200::max_windows(probing_length, cg_size(), view_.t.num_buckets),
                num, [&](V v, std::uint64_t j) { f(value_type(v), j); });
            if (st) b200::join_status(view_.t.status, st);
        }
        num_out = group.shfl(num, 0);
        return status_type(group.shfl(st, 0));
    }

    static wc_stream_t stream_of(cudaStream_t s) { return reinterpret_cast<wc_stream_t>(s); }
    wc_blht_info info() const noexcept
    {
        wc_blht_info inf{};
        if (handle_) wc_blht_get_info(handle_, &inf);
        return inf;
    }
    void refresh() noexcept
    {
        wc_blht_info inf;
        if (wc_blht_get_info(handle_, &inf) != WC_OK) return;
        b200::TableView t{};
        t.slots = inf.keys;
        t.status = inf.status;
        t.fps = nullptr;
        t.num_buckets = inf.num_buckets;
        t.seed = inf.seed;
        t.empty_key = inf.empty_key;
        t.tombstone_key = inf.tombstone_key;
        t.max_count = ~0ull;
        t.magic_nb = b200::barrett_magic(inf.num_buckets);
        t.magic_nb1 = b200::barrett_magic(inf.num_buckets > 1 ? inf.num_buckets - 1 : 1);
        t.probing = inf.probing;
        t.hasher1 = inf.hasher1;
        t.hasher2 = inf.hasher2;
        t.cg_size = inf.cg_size;
        view_.t = t;
        view_.handles = inf.handles;
        view_.pool = inf.pool;
        view_.next_free = inf.next_free;
        view_.capacity = inf.value_capacity;
        view_.min_bucket = inf.min_bucket_size;
        view_.max_bucket = inf.max_bucket_size;
        view_.max_values = inf.max_values_per_key;
        view_.grow = inf.grow_factor;
        view_.ib = inf.index_bits;
        view_.cb = inf.counter_bits;
        view_.sb = inf.size_bits;
        is_initialized_ = inf.is_initialized != 0;
    }

    wc_blht *handle_ = nullptr;
    b200::BlView view_{};
    bool is_initialized_ = false;
    bool is_copy_ = false;
};

} // namespace warpcore

#endif /* WARPCORE_B200_CXX_BLHT_CUH */
