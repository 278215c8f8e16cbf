/*
 * warpcore::MultiBucketHashTable -- drop-in for the reference class
 * (multi_bucket_hash_table.cuh:88-1371) over the B200-native library.
 * Host bulk methods call the C ABI (wc_mbht_*).  The device per-key methods
 * (insert / retrieve / num_values / for_each with a cooperative group of
 * cg_size() threads) run the bulk kernels' per-key code (detail/mb_ops.cuh)
 * on the group's first thread and hand the result to every thread of the
 * group.  The table storage parameter only names the bucket size: keys and
 * buckets are kept as two arrays.  Objects are passed to user kernels by
 * value; copies are shallow, as in the reference.
 */
#ifndef WARPCORE_B200_CXX_MBHT_CUH
#define WARPCORE_B200_CXX_MBHT_CUH

#include "base.cuh"
#include "detail/mb_ops.cuh"

namespace warpcore {

/* ArrayBucket<Value, BucketSize> (multi_bucket_hash_table.cuh:9-81): the
 * bucket type handed to for_each_bucket */
template <class Value, std::uint32_t BucketSize = 1>
struct ArrayBucket {
    using value_type = Value;
    using index_type = std::uint32_t;
    static_assert(BucketSize > 0, "invalid bucket size of 0");

    __host__ __device__ explicit ArrayBucket(value_type value) noexcept
    {
        for (index_type i = 0; i < bucket_size(); ++i) values_[i] = value;
    }
    __host__ __device__ ArrayBucket(const ArrayBucket &o) noexcept
    {
        for (index_type i = 0; i < bucket_size(); ++i) values_[i] = o.values_[i];
    }
    __host__ __device__ ArrayBucket &operator=(const ArrayBucket &o) noexcept
    {
        for (index_type i = 0; i < bucket_size(); ++i) values_[i] = o.values_[i];
        return *this;
    }
    __host__ __device__ static constexpr index_type bucket_size() noexcept { return BucketSize; }
    __device__ value_type &operator[](const index_type i) noexcept { return values_[i]; }
    __device__ const value_type &operator[](const index_type i) const noexcept { return values_[i]; }

    value_type values_[BucketSize];
};

namespace detail {
template <class Func, class K, class V, std::uint32_t B>
__global__ void mb_for_each_bucket_kernel(Func f, b200::MbView m, std::uint64_t capacity)
{
    const K empty = K(m.t.empty_key), tomb = K(m.t.tombstone_key);
    const std::uint64_t i = std::uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= capacity) return;
    const K k = reinterpret_cast<const K *>(m.t.slots)[i];
    if (k == empty || k == tomb) return;
    ArrayBucket<V, B> b(V(m.empty_value));
    for (std::uint32_t r = 0; r < B; ++r) b[r] = reinterpret_cast<const V *>(m.vals)[i * B + r];
    f(k, b);
}

template <class Func, class K, class V, int kW, int kB>
__global__ void mb_for_each_keys_kernel(Func f, b200::MbView m, const K *keys, std::uint64_t n,
                                        std::uint64_t max_windows, void *status_out, int handler,
                                        std::uint32_t bool_mask)
{
    const std::uint64_t i = std::uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const K key = keys[i];
    std::uint64_t num = 0;
    const std::uint32_t st = b200::mb_for_each_one<K, V, kW, kB>(
        m, key, max_windows, num, [&](V v, std::uint64_t j) { f(key, v, j); });
    if (st) b200::join_status(m.t.status, st);
    if (status_out && handler == b200::kHandlerStatus)
        reinterpret_cast<std::uint32_t *>(status_out)[i] = st;
    else if (status_out && handler == b200::kHandlerBoolean)
        reinterpret_cast<unsigned char *>(status_out)[i] = (st & bool_mask) != 0;
}
} // namespace detail

template <class Key, class Value, Key EmptyKey = defaults::empty_key<Key>(),
          Key TombstoneKey = defaults::tombstone_key<Key>(),
          Value EmptyValue = defaults::empty_key<Value>(),
          class ProbingScheme = defaults::probing_scheme_t<Key, 8>,
          class TableStorage = defaults::table_storage_t<Key, ArrayBucket<Value, 2>>,
          index_t TempMemoryBytes = defaults::temp_memory_bytes()>
class MultiBucketHashTable {
    static_assert(checks::is_valid_key_type<Key>(), "invalid key type");
    static_assert(EmptyKey != TombstoneKey, "empty key and tombstone key must not be identical");
    static_assert(checks::is_probing_scheme<ProbingScheme>(), "not a valid probing scheme type");
    static_assert(std::is_same<typename ProbingScheme::key_type, Key>::value,
                  "probing key type differs from table's key type");
    static_assert(std::is_same<typename TableStorage::key_type, Key>::value,
                  "storage's key type differs from table's key type");
    static_assert(std::is_same<typename TableStorage::value_type::value_type, Value>::value,
                  "storage's value type differs from table's value type");
    static_assert((sizeof(Value) == 4 || sizeof(Value) == 8) && std::is_integral<Value>::value,
                  "this build stores 4- or 8-byte integral values");
    static_assert(TableStorage::value_type::bucket_size() <= ProbingScheme::cg_size(),
                  "this build keeps buckets no larger than the cooperative group");

    using K = typename std::make_unsigned<Key>::type;
    using V = typename std::make_unsigned<Value>::type;

  public:
    using key_type = Key;
    using value_type = Value;
    using bucket_type = typename TableStorage::value_type;
    using index_type = index_t;
    using status_type = Status;
    using probing_scheme_type = ProbingScheme;

    __host__ __device__ static constexpr key_type empty_key() noexcept { return EmptyKey; }
    __host__ __device__ static constexpr key_type tombstone_key() noexcept { return TombstoneKey; }
    __host__ __device__ static constexpr value_type empty_value() noexcept { return EmptyValue; }
    __host__ __device__ static constexpr index_type cg_size() noexcept { return ProbingScheme::cg_size(); }
    __host__ __device__ static constexpr index_type bucket_size() noexcept
    {
        return bucket_type::bucket_size();
    }

    /* multi_bucket_hash_table.cuh:195-217 */
    explicit MultiBucketHashTable(const index_type min_capacity,
                                  const key_type seed = defaults::seed<key_type>(),
                                  const index_type max_values_per_key =
                                      std::numeric_limits<index_type>::max(),
                                  const bool no_init = false) noexcept
    {
        wc_table_config cfg =
            detail::make_config<ProbingScheme, Key>(sizeof(Value), EmptyKey, TombstoneKey);
        if (wc_mbht_create(&cfg, std::uint32_t(bucket_size()), std::uint64_t(V(EmptyValue)),
                           min_capacity, std::uint64_t(seed), max_values_per_key, no_init ? 1 : 0,
                           &handle_) == WC_OK)
            refresh();
    }

    __host__ __device__ MultiBucketHashTable(const MultiBucketHashTable &o) noexcept
        : handle_(o.handle_), view_(o.view_), capacity_(o.capacity_),
          is_initialized_(o.is_initialized_), is_copy_(true)
    {}

    MultiBucketHashTable(MultiBucketHashTable &&o) noexcept
        : handle_(o.handle_), view_(o.view_), capacity_(o.capacity_),
          is_initialized_(o.is_initialized_), is_copy_(o.is_copy_)
    {
        o.is_copy_ = true;
    }

#ifndef __CUDA_ARCH__
    ~MultiBucketHashTable() noexcept
    {
        if (!is_copy_ && handle_) wc_mbht_destroy(handle_);
    }
#endif

    /* init (:253-271) */
    void init(const cudaStream_t stream = 0) noexcept
    {
        if (handle_ && wc_mbht_init(handle_, stream_of(stream)) == WC_OK) refresh();
    }

    /* device insert (:343-517) */
    __device__ status_type insert(const key_type key_in, const value_type value_in,
                                  const cg::thread_block_tile<cg_size()> &group,
                                  const index_type probing_length = defaults::probing_length()) noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        std::uint32_t st = 0;
        if (group.thread_rank() == 0) {
            bool claimed = false, fresh = false;
            st = b200::mb_insert_one<K, V, int(cg_size()), int(bucket_size())>(
                view_, K(key_in), V(value_in),
                b200::max_windows(probing_length, cg_size(), view_.t.num_buckets), claimed, fresh);
            if (claimed) atomicAdd(view_.num_occupied, 1ull);
            if (fresh) atomicAdd(view_.num_keys, 1ull);
            if (st != 0 && st != b200::kStDuplicateKey) b200::join_status(view_.t.status, st);
        }
        return status_type(group.shfl(st, 0));
    }

    /* host insert (:528-542) */
    template <class StatusHandler = defaults::status_handler_t>
    void insert(const key_type *const keys_in, const value_type *const values_in,
                const index_type num_in, const cudaStream_t stream = 0,
                const index_type probing_length = defaults::probing_length(),
                typename StatusHandler::base_type *const status_out = nullptr) noexcept
    {
        static_assert(checks::is_status_handler<StatusHandler>(), "not a valid status handler type");
        if (!is_initialized_) return;
        wc_mbht_insert(handle_, keys_in, values_in, num_in, stream_of(stream), probing_length,
                       (void *)status_out, StatusHandler::kId, StatusHandler::kIgnore);
    }

    /* device for_each over one key's values (:786-846): f(key, value, index) */
    template <class Func>
    __device__ status_type for_each(Func f, const key_type key_in, index_type &num_values_out,
                                    const cg::thread_block_tile<cg_size()> &group,
                                    const index_type probing_length = defaults::probing_length()) const noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        std::uint32_t st = 0;
        std::uint64_t num = 0;
        if (group.thread_rank() == 0) {
            const std::uint64_t pl = probing_length < capacity_ ? probing_length : capacity_;
            st = b200::mb_for_each_one<K, V, int(cg_size()), int(bucket_size())>(
                view_, K(key_in), b200::max_windows(pl, cg_size(), view_.t.num_buckets), num,
                [&](V v, std::uint64_t j) { f(key_in, value_type(v), j); });
            if (st) b200::join_status(view_.t.status, st);
        }
        num_values_out = group.shfl(num, 0);
        return status_type(group.shfl(st, 0));
    }

    /* device retrieve (:553-572): values_out NULL is a dry run (num_values) */
    __device__ status_type retrieve(const key_type key_in, value_type *const values_out,
                                    index_type &num_out,
                                    const cg::thread_block_tile<cg_size()> &group,
                                    const index_type probing_length = defaults::probing_length()) const noexcept
    {
        if (values_out == nullptr) {
            const status_type s = num_values(key_in, num_out, group, probing_length);
            if (group.thread_rank() == 0) b200::join_status(view_.t.status, b200::kStDryRun);
            return status_type::dry_run() + s;
        }
        return for_each([=](key_type, const value_type &v, index_type j) { values_out[j] = v; },
                        key_in, num_out, group, probing_length);
    }

    /* device num_values (:993-1004) */
    __device__ status_type num_values(const key_type key_in, index_type &num_out,
                                      const cg::thread_block_tile<cg_size()> &group,
                                      const index_type probing_length = defaults::probing_length()) const noexcept
    {
        return for_each([](key_type, const value_type &, index_type) {}, key_in, num_out, group,
                        probing_length);
    }

    /* host retrieve (:574-680): offsets are index_type (uint64); values_out
     * NULL is a dry run leaving the per-key counts in end_offsets_out;
     * synchronises */
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
        if (wc_mbht_retrieve(handle_, keys_in, num_in, (std::uint64_t *)begin_offsets_out,
                             (std::uint64_t *)end_offsets_out, values_out, &n, stream_of(stream),
                             probing_length, (void *)status_out, StatusHandler::kId,
                             StatusHandler::kIgnore) == WC_OK)
            num_out = n;
    }

    /* retrieve_all (:692-722): unique keys, then their values */
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

    /* retrieve_all_keys (:730-777); keys_out NULL gives num_keys() */
    void retrieve_all_keys(key_type *const keys_out, index_type &num_out,
                           const cudaStream_t stream = 0) const noexcept
    {
        num_out = 0;
        if (!is_initialized_) return;
        std::uint64_t n = 0;
        if (wc_mbht_retrieve_all_keys(handle_, keys_out, &n, stream_of(stream)) == WC_OK)
            num_out = n;
    }

    /* for_each_bucket (:855-869): f(key, bucket) for every occupied slot */
    template <class Func>
    void for_each_bucket(Func f, const cudaStream_t stream = 0,
                         const index_type smem_bytes = 0) const noexcept
    {
        if (!is_initialized_) return;
        const unsigned grid = unsigned((capacity_ + 255) / 256);
        detail::mb_for_each_bucket_kernel<Func, K, V, std::uint32_t(bucket_size())>
            <<<grid, 256, smem_bytes, stream>>>(f, view_, capacity_);
    }

    /* for_each_value (:877-903): f(key, value) for every stored value */
    template <class Func>
    void for_each_value(Func f, const cudaStream_t stream = 0,
                        const index_type smem_bytes = 0) const noexcept
    {
        const value_type ev = empty_value();
        for_each_bucket(
            [=] __device__(const key_type key, const bucket_type &b) mutable {
                for (index_type r = 0; r < bucket_size(); ++r)
                    if (b[r] != ev) f(key, b[r]);
            },
            stream, smem_bytes);
    }

    /* for_each over given keys (:915-937): f(key, value, index) */
    template <class Func, class StatusHandler = defaults::status_handler_t>
    void for_each(Func f, const key_type *const keys_in, const index_type num_in,
                  const cudaStream_t stream = 0,
                  const index_type probing_length = defaults::probing_length(),
                  typename StatusHandler::base_type *const status_out = nullptr,
                  const index_type smem_bytes = 0) const noexcept
    {
        if (!is_initialized_ || num_in == 0) return;
        const std::uint64_t pl = probing_length < capacity_ ? probing_length : capacity_;
        const unsigned grid = unsigned((num_in + 255) / 256);
        detail::mb_for_each_keys_kernel<Func, K, V, int(cg_size()), int(bucket_size())>
            <<<grid, 256, smem_bytes, stream>>>(
            f, view_, reinterpret_cast<const K *>(keys_in), num_in,
            b200::max_windows(pl, cg_size(), view_.t.num_buckets), (void *)status_out,
            StatusHandler::kId, (~std::uint32_t(StatusHandler::kIgnore)) ^ 0xFFFu);
    }

    /* host num_values (:1013-1039) */
    template <class StatusHandler = defaults::status_handler_t>
    void num_values(const key_type *const keys_in, const index_type num_in, index_type &num_out,
                    index_type *const num_per_key_out = nullptr, const cudaStream_t stream = 0,
                    const index_type probing_length = defaults::probing_length(),
                    typename StatusHandler::base_type *const status_out = nullptr) const noexcept
    {
        num_out = 0;
        if (!is_initialized_) return;
        std::uint64_t n = 0;
        if (wc_mbht_num_values(handle_, keys_in, num_in, &n, (std::uint64_t *)num_per_key_out,
                               stream_of(stream), probing_length, (void *)status_out,
                               StatusHandler::kId, StatusHandler::kIgnore) == WC_OK)
            num_out = n;
    }
    index_type num_values(const cudaStream_t stream = 0) const noexcept { return size(stream); }

    /* num_keys (:945-956), num_occupied (:958-969), size (:1060-1082) */
    index_type num_keys(const cudaStream_t stream = 0) const noexcept
    {
        std::uint64_t n = 0;
        if (is_initialized_) wc_mbht_num_keys(handle_, stream_of(stream), &n);
        return n;
    }
    index_type num_occupied(const cudaStream_t stream = 0) const noexcept
    {
        std::uint64_t n = 0;
        if (is_initialized_) wc_mbht_num_occupied(handle_, stream_of(stream), &n);
        return n;
    }
    index_type size(const cudaStream_t stream = 0) const noexcept
    {
        std::uint64_t n = 0;
        if (is_initialized_) wc_mbht_size(handle_, stream_of(stream), &n);
        return n;
    }

    /* load factors and densities (:1084-1127) */
    float key_load_factor(const cudaStream_t stream = 0) const noexcept
    {
        return float(num_occupied(stream)) / float(capacity());
    }
    float value_load_factor(const cudaStream_t stream = 0) const noexcept
    {
        return float(num_values(stream)) / float(capacity() * bucket_size());
    }
    float storage_density(const cudaStream_t stream = 0) const noexcept
    {
        const index_type key_bytes = num_keys(stream) * sizeof(key_type);
        const index_type value_bytes = num_values(stream) * sizeof(value_type);
        return float(key_bytes + value_bytes) / float(bytes_total());
    }
    float relative_storage_density(const cudaStream_t stream = 0) const noexcept
    {
        const index_type key_bytes = num_keys(stream) * sizeof(key_type);
        const index_type value_bytes = num_values(stream) * sizeof(value_type);
        const index_type occupied_bytes = num_occupied(stream) * sizeof(key_type) + value_bytes;
        return float(key_bytes + value_bytes) / float(occupied_bytes);
    }

    __host__ __device__ index_type capacity() const noexcept { return capacity_; }
    __host__ __device__ index_type value_capacity() const noexcept
    {
        return capacity_ * bucket_size();
    }
    index_type bytes_total() const noexcept
    {
        wc_mbht_info inf;
        return (handle_ && wc_mbht_get_info(handle_, &inf) == WC_OK) ? inf.bytes_total : 0;
    }
    __host__ __device__ bool is_initialized() const noexcept { return is_initialized_; }

    status_type peek_status(const cudaStream_t stream = 0) const noexcept
    {
        std::uint32_t s = WC_STATUS_NOT_INITIALIZED;
        if (handle_) wc_mbht_peek_status(handle_, stream_of(stream), &s);
        return status_type(s);
    }
    status_type pop_status(const cudaStream_t stream = 0) noexcept
    {
        std::uint32_t s = WC_STATUS_NOT_INITIALIZED;
        if (handle_) wc_mbht_pop_status(handle_, stream_of(stream), &s);
        return status_type(s);
    }

    __host__ __device__ static constexpr bool is_empty_key(const key_type key) noexcept
    {
        return key == empty_key();
    }
    __host__ __device__ static constexpr bool is_tombstone_key(const key_type key) noexcept
    {
        return key == tombstone_key();
    }
    __host__ __device__ static constexpr bool is_valid_key(const key_type key) noexcept
    {
        return key != empty_key() && key != tombstone_key();
    }
    __host__ __device__ static constexpr bool is_empty_value(const value_type value) noexcept
    {
        return value == empty_value();
    }
    __host__ __device__ static constexpr bool is_valid_value(const value_type value) noexcept
    {
        return value != empty_value();
    }
    __host__ __device__ key_type seed() const noexcept { return key_type(view_.t.seed); }
    __host__ __device__ bool is_copy() const noexcept { return is_copy_; }
    __host__ __device__ const b200::MbView &device_view() const noexcept { return view_; }
    wc_mbht *handle() const noexcept { return handle_; }

  private:
    static wc_stream_t stream_of(cudaStream_t s) { return reinterpret_cast<wc_stream_t>(s); }
    void refresh() noexcept
    {
        wc_mbht_info inf;
        if (wc_mbht_get_info(handle_, &inf) != WC_OK) return;
        b200::TableView v{};
        v.slots = inf.keys;
        v.status = inf.status;
        v.fps = nullptr;
        v.num_buckets = inf.num_buckets;
        v.seed = inf.seed;
        v.empty_key = inf.empty_key;
        v.tombstone_key = inf.tombstone_key;
        v.max_count = ~0ull;
        v.magic_nb = b200::barrett_magic(inf.num_buckets);
        v.magic_nb1 = b200::barrett_magic(inf.num_buckets > 1 ? inf.num_buckets - 1 : 1);
        v.probing = inf.probing;
        v.hasher1 = inf.hasher1;
        v.hasher2 = inf.hasher2;
        v.cg_size = inf.cg_size;
        view_.t = v;
        view_.vals = inf.values;
        view_.empty_value = inf.empty_value;
        view_.max_values = inf.max_values_per_key;
        view_.bucket = inf.bucket_size;
        view_.num_keys = inf.num_keys;
        view_.num_occupied = inf.num_occupied;
        capacity_ = inf.capacity;
        is_initialized_ = inf.is_initialized != 0;
    }

    wc_mbht *handle_ = nullptr;
    b200::MbView view_{};
    index_type capacity_ = 0;
    bool is_initialized_ = false;
    bool is_copy_ = false;
};

} // namespace warpcore

#endif /* WARPCORE_B200_CXX_MBHT_CUH */
