/*
 * warpcore::MultiValueHashTable -- drop-in for the reference class
 * (multi_value_hash_table.cuh:18-1040) over the B200-native library.
 * Host bulk methods call the C ABI (wc_mvht_*).  The device per-key methods
 * (insert / retrieve / num_values / for_each with a cooperative group of
 * cg_size() threads) run the bulk kernels' per-key code
 * (detail/mv_ops.cuh) on the group's first thread and hand the result to
 * every thread of the group.  Objects are passed to user kernels by value;
 * copies are shallow, as in the reference.
 */
#ifndef WARPCORE_B200_CXX_MVHT_CUH
#define WARPCORE_B200_CXX_MVHT_CUH

#include "base.cuh"
#include "detail/mv_ops.cuh"

namespace warpcore {

template <class Key, class Value, Key EmptyKey = defaults::empty_key<Key>(),
          Key TombstoneKey = defaults::tombstone_key<Key>(),
          class ProbingScheme = defaults::probing_scheme_t<Key, 8>,
          class TableStorage = defaults::table_storage_t<Key, Value>,
          index_t TempMemoryBytes = defaults::temp_memory_bytes()>
class MultiValueHashTable {
    static_assert(checks::is_valid_key_type<Key>(), "invalid key type");
    static_assert(EmptyKey != TombstoneKey, "empty key and tombstone key must not be identical");
    static_assert(checks::is_probing_scheme<ProbingScheme>(), "not a valid probing scheme type");
    static_assert(std::is_same<typename ProbingScheme::key_type, Key>::value,
                  "probing key type differs from table's key type");
    static_assert((sizeof(Value) == 4 || sizeof(Value) == 8) && std::is_integral<Value>::value,
                  "this build stores integral values as wide as the key (u32/u32, u64/u64)");

    using layout = typename detail::layout_of<Key, typename std::make_unsigned<Value>::type>::type;
    static constexpr int kW = int(ProbingScheme::cg_size());

  public:
    using key_type = Key;
    using value_type = Value;
    using index_type = index_t;
    using status_type = Status;

    __host__ __device__ static constexpr key_type empty_key() noexcept { return EmptyKey; }
    __host__ __device__ static constexpr key_type tombstone_key() noexcept { return TombstoneKey; }
    __host__ __device__ static constexpr index_type cg_size() noexcept { return ProbingScheme::cg_size(); }

    /* multi_value_hash_table.cuh:101-125 */
    explicit MultiValueHashTable(const index_type min_capacity,
                                 const key_type seed = defaults::seed<key_type>(),
                                 const index_type max_values_per_key =
                                     std::numeric_limits<index_type>::max(),
                                 const bool no_init = false) noexcept
    {
        const wc_table_config cfg =
            detail::make_config<ProbingScheme, Key>(sizeof(Value), EmptyKey, TombstoneKey);
        if (wc_mvht_create(&cfg, min_capacity, std::uint64_t(seed), max_values_per_key,
                           no_init ? 1 : 0, &handle_) == WC_OK)
            refresh();
    }

    __host__ __device__ MultiValueHashTable(const MultiValueHashTable &o) noexcept
        : handle_(o.handle_), view_(o.view_), num_keys_(o.num_keys_), capacity_(o.capacity_),
          max_values_(o.max_values_), is_initialized_(o.is_initialized_), is_copy_(true)
    {}

    MultiValueHashTable(MultiValueHashTable &&o) noexcept
        : handle_(o.handle_), view_(o.view_), num_keys_(o.num_keys_), capacity_(o.capacity_),
          max_values_(o.max_values_), is_initialized_(o.is_initialized_), is_copy_(o.is_copy_)
    {
        o.is_copy_ = true;
    }

#ifndef __CUDA_ARCH__
    ~MultiValueHashTable() noexcept
    {
        if (!is_copy_ && handle_) wc_table_destroy(handle_);
    }
#endif

    /* multi_value_hash_table.cuh:170-191 */
    void init(const cudaStream_t stream = 0) noexcept
    {
        if (handle_ && wc_table_init(handle_, std::uint64_t(seed()), stream_of(stream)) == WC_OK)
            refresh();
    }

    /* device insert (:200-289) */
    __device__ status_type insert(const key_type key_in, const value_type &value_in,
                                  const cg::thread_block_tile<cg_size()> &group,
                                  const index_type probing_length = defaults::probing_length()) noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        std::uint32_t st = 0;
        if (group.thread_rank() == 0) {
            bool fresh = false;
            st = b200::mv_insert_one<layout, kW>(
                view_, key_in, typename layout::val_t(value_in),
                b200::max_windows(probing_length, cg_size(), view_.num_buckets), max_values_,
                fresh);
            if (fresh) atomicAdd(num_keys_, 1ull);
            if (st != 0 && st != b200::kStDuplicateKey) b200::join_status(view_.status, st);
        }
        return status_type(group.shfl(st, 0));
    }

    /* host insert (:301-326) */
    template <class StatusHandler = defaults::status_handler_t>
    void insert(const key_type *const keys_in, const value_type *const values_in,
                const index_type num_in, const cudaStream_t stream = 0,
                const index_type probing_length = defaults::probing_length(),
                typename StatusHandler::base_type *const status_out = nullptr) noexcept
    {
        static_assert(checks::is_status_handler<StatusHandler>(), "not a valid status handler type");
        if (!is_initialized_) return;
        wc_mvht_insert(handle_, keys_in, values_in, num_in, stream_of(stream), probing_length,
                       (void *)status_out, StatusHandler::kId, StatusHandler::kIgnore);
    }

    /* device for_each over one key's values (:607-663): f(key, value, index) */
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
            st = b200::mv_for_each_one<layout, kW>(
                view_, key_in, b200::max_windows(pl, cg_size(), view_.num_buckets), max_values_,
                num, [&](typename layout::val_t v, std::uint64_t j) { f(key_in, value_type(v), j); });
            if (st) b200::join_status(view_.status, st);
        }
        num_values_out = group.shfl(num, 0);
        return status_type(group.shfl(st, 0));
    }

    /* device retrieve (:329-363): values_out NULL is a dry run (num_values) */
    __device__ status_type retrieve(const key_type key_in, value_type *const values_out,
                                    index_type &num_out,
                                    const cg::thread_block_tile<cg_size()> &group,
                                    const index_type probing_length = defaults::probing_length()) const noexcept
    {
        if (values_out == nullptr) {
            const status_type s = num_values(key_in, num_out, group, probing_length);
            if (group.thread_rank() == 0) b200::join_status(view_.status, b200::kStDryRun);
            return status_type::dry_run() + s;
        }
        return for_each([=](key_type, const value_type &v, index_type j) { values_out[j] = v; },
                        key_in, num_out, group, probing_length);
    }

    /* device num_values (:739-757) */
    __device__ status_type num_values(const key_type key_in, index_type &num_out,
                                      const cg::thread_block_tile<cg_size()> &group,
                                      const index_type probing_length = defaults::probing_length()) const noexcept
    {
        return for_each([](key_type, const value_type &, index_type) {}, key_in, num_out, group,
                        probing_length);
    }

    /* host retrieve (:371-520): offsets are index_type (uint64); with
     * values_out NULL a dry run that leaves the per-key counts in
     * end_offsets_out; synchronises */
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
        if (wc_mvht_retrieve(handle_, keys_in, num_in, (std::uint64_t *)begin_offsets_out,
                             (std::uint64_t *)end_offsets_out, values_out, &n, stream_of(stream),
                             probing_length, (void *)status_out, StatusHandler::kId,
                             StatusHandler::kIgnore) == WC_OK)
            num_out = n;
    }

    /* retrieve_all (:523-553): unique keys, then their values */
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

    /* retrieve_all_keys (:561-598); keys_out NULL gives num_keys() */
    void retrieve_all_keys(key_type *const keys_out, index_type &num_out,
                           const cudaStream_t stream = 0) const noexcept
    {
        num_out = 0;
        if (!is_initialized_) return;
        std::uint64_t n = 0;
        if (wc_mvht_retrieve_all_keys(handle_, keys_out, &n, stream_of(stream)) == WC_OK)
            num_out = n;
    }

    /* host num_values (:769-800) */
    template <class StatusHandler = defaults::status_handler_t>
    void num_values(const key_type *const keys_in, const index_type num_in, index_type &num_out,
                    index_type *const num_per_key_out = nullptr, const cudaStream_t stream = 0,
                    const index_type probing_length = defaults::probing_length(),
                    typename StatusHandler::base_type *const status_out = nullptr) const noexcept
    {
        num_out = 0;
        if (!is_initialized_) return;
        std::uint64_t n = 0;
        if (wc_mvht_num_values(handle_, keys_in, num_in, &n, (std::uint64_t *)num_per_key_out,
                               stream_of(stream), probing_length, (void *)status_out,
                               StatusHandler::kId, StatusHandler::kIgnore) == WC_OK)
            num_out = n;
    }
    index_type num_values(const cudaStream_t stream = 0) const noexcept { return size(stream); }

    /* num_keys (:720-735) */
    index_type num_keys(const cudaStream_t stream = 0) const noexcept
    {
        std::uint64_t n = 0;
        if (is_initialized_) wc_mvht_num_keys(handle_, stream_of(stream), &n);
        return n;
    }

    /* size / load_factor / storage_density (:812-863) */
    index_type size(const cudaStream_t stream = 0) const noexcept
    {
        if (!is_initialized_) return 0;
        std::uint64_t n = 0;
        wc_table_size(handle_, stream_of(stream), &n);
        return n;
    }
    float load_factor(const cudaStream_t stream = 0) const noexcept
    {
        return float(size(stream)) / float(capacity());
    }
    float storage_density(const cudaStream_t stream = 0) const noexcept
    {
        const index_type key_bytes = num_keys(stream) * sizeof(key_type);
        const index_type value_bytes = num_values(stream) * sizeof(value_type);
        return float(key_bytes + value_bytes) / float(bytes_total());
    }

    __host__ __device__ index_type capacity() const noexcept { return capacity_; }
    index_type bytes_total() const noexcept
    {
        wc_table_info inf;
        return (handle_ && wc_table_get_info(handle_, &inf) == WC_OK) ? inf.bytes_total : 0;
    }
    __host__ __device__ bool is_initialized() const noexcept { return is_initialized_; }

    status_type peek_status(const cudaStream_t stream = 0) const noexcept
    {
        std::uint32_t s = WC_STATUS_NOT_INITIALIZED;
        if (handle_) wc_table_peek_status(handle_, stream_of(stream), &s);
        return status_type(s);
    }
    status_type pop_status(const cudaStream_t stream = 0) noexcept
    {
        std::uint32_t s = WC_STATUS_NOT_INITIALIZED;
        if (handle_) wc_table_pop_status(handle_, stream_of(stream), &s);
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
    __host__ __device__ key_type seed() const noexcept { return key_type(view_.seed); }
    __host__ __device__ index_type max_values_per_key() const noexcept { return max_values_; }
    __host__ __device__ bool is_copy() const noexcept { return is_copy_; }
    __host__ __device__ const b200::TableView &device_view() const noexcept { return view_; }
    wc_table *handle() const noexcept { return handle_; }

  private:
    static wc_stream_t stream_of(cudaStream_t s) { return reinterpret_cast<wc_stream_t>(s); }
    void refresh() noexcept
    {
        wc_table_info inf;
        if (wc_table_get_info(handle_, &inf) != WC_OK) return;
        view_ = detail::view_from(inf);
        num_keys_ = inf.num_keys;
        capacity_ = inf.capacity;
        max_values_ = inf.max_values_per_key;
        is_initialized_ = inf.is_initialized != 0;
    }

    wc_table *handle_ = nullptr;
    b200::TableView view_{};
    unsigned long long *num_keys_ = nullptr;
    index_type capacity_ = 0;
    index_type max_values_ = 0;
    bool is_initialized_ = false;
    bool is_copy_ = false;
};

} // namespace warpcore

#endif /* WARPCORE_B200_CXX_MVHT_CUH */
