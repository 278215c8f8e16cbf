/*
 * warpcore::SingleValueHashTable -- drop-in for the reference class
 * (single_value_hash_table.cuh:29-915) over the B200-native library.
 * Host bulk methods call the C ABI; device per-key methods
 * (insert/retrieve/erase with a cooperative group of cg_size() threads) run
 * the same bucket-aligned probing as the bulk kernels.  Objects are passed
 * to user kernels by value; copies are shallow, as in the reference.
 */
#ifndef WARPCORE_B200_CXX_SVHT_CUH
#define WARPCORE_B200_CXX_SVHT_CUH

#include "base.cuh"
#include "detail/tile_ops.cuh"

namespace warpcore {

namespace detail {
template <class F, class Table>
__global__ void svht_for_each_kernel(F f, const Table table);
}

template <class Key, class Value, Key EmptyKey = defaults::empty_key<Key>(),
          Key TombstoneKey = defaults::tombstone_key<Key>(),
          class ProbingScheme = defaults::probing_scheme_t<Key, 8>,
          class TableStorage = defaults::table_storage_t<Key, Value>,
          index_t TempMemoryBytes = defaults::temp_memory_bytes()>
class SingleValueHashTable {
    static_assert(checks::is_valid_key_type<Key>(), "invalid key type");
    static_assert(EmptyKey != TombstoneKey, "empty key and tombstone key must not be identical");
    static_assert(checks::is_probing_scheme<ProbingScheme>(), "not a valid probing scheme type");
    static_assert(std::is_same<typename ProbingScheme::key_type, Key>::value,
                  "probing key type differs from table's key type");
    static_assert((sizeof(Value) == 4 || sizeof(Value) == 8) &&
                      std::is_trivially_copyable<Value>::value,
                  "this build stores trivially copyable values of 4 or 8 bytes");

    /* the value's bits, held in the slot as an unsigned word of its width */
    using value_word = typename std::conditional<sizeof(Value) == 4, std::uint32_t, std::uint64_t>::type;
    using key_word = typename std::conditional<sizeof(Key) == 4, std::uint32_t, std::uint64_t>::type;
    static constexpr bool kSoA = detail::is_soa_store<TableStorage>::value;
    /* {key, value} slots, or a key array and a value array (SoAStore) */
    using layout = typename std::conditional<kSoA, b200::LayoutSoA<key_word, value_word>,
                                             typename detail::layout_of<Key, value_word>::type>::type;

  public:
    using key_type = Key;
    using value_type = Value;
    using index_type = index_t;
    using status_type = Status;

    __host__ __device__ static constexpr key_type empty_key() noexcept { return EmptyKey; }
    __host__ __device__ static constexpr key_type tombstone_key() noexcept { return TombstoneKey; }
    __host__ __device__ static constexpr index_type cg_size() noexcept { return ProbingScheme::cg_size(); }

    /* single_value_hash_table.cuh:112-128 */
    explicit SingleValueHashTable(const index_type min_capacity,
                                  const key_type seed = defaults::seed<key_type>(),
                                  const bool no_init = false) noexcept
    {
        const wc_table_config cfg =
            detail::make_config<ProbingScheme, Key>(sizeof(Value), EmptyKey, TombstoneKey);
        detail::load_tuning_once();
        const int rc = kSoA ? wc_svht_create_soa(&cfg, min_capacity, std::uint64_t(seed),
                                                 no_init ? 1 : 0, &handle_)
                            : wc_svht_create(&cfg, min_capacity, std::uint64_t(seed),
                                             no_init ? 1 : 0, &handle_);
        if (rc == WC_OK) refresh();
    }

    __host__ __device__ SingleValueHashTable(const SingleValueHashTable &o) noexcept
        : handle_(o.handle_), view_(o.view_), capacity_(o.capacity_),
          is_initialized_(o.is_initialized_), is_copy_(true)
    {}

    SingleValueHashTable(SingleValueHashTable &&o) noexcept
        : handle_(o.handle_), view_(o.view_), capacity_(o.capacity_),
          is_initialized_(o.is_initialized_), is_copy_(o.is_copy_)
    {
        o.is_copy_ = true;
    }

#ifndef __CUDA_ARCH__
    ~SingleValueHashTable() noexcept
    {
        if (!is_copy_ && handle_) wc_table_destroy(handle_);
    }
#endif

    /* single_value_hash_table.cuh:176-201 */
    void init(const key_type seed, const cudaStream_t stream = 0) noexcept
    {
        if (handle_ && wc_table_init(handle_, std::uint64_t(seed), stream_of(stream)) == WC_OK)
            refresh();
    }
    void init(const cudaStream_t stream = 0) noexcept { init(seed(), stream); }

    /* device insert (single_value_hash_table.cuh:211-228) */
    __device__ status_type insert(const key_type key_in, const value_type &value_in,
                                  const cg::thread_block_tile<cg_size()> &group,
                                  const index_type probing_length = defaults::probing_length()) noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        return status_type(b200::tile_modify<layout>(view_, group, key_in, value_bits(value_in), 0,
                                                     probing_length));
    }

    /* host insert (single_value_hash_table.cuh:241-258) */
    template <class StatusHandler = defaults::status_handler_t>
    void insert(const key_type *const keys_in, const value_type *const values_in,
                const index_type num_in, const cudaStream_t stream = 0,
                const index_type probing_length = defaults::probing_length(),
                typename StatusHandler::base_type *const status_out = nullptr) noexcept
    {
        static_assert(checks::is_status_handler<StatusHandler>(), "not a valid status handler type");
        if (!is_initialized_) return;
        wc_svht_insert(handle_, keys_in, values_in, num_in, stream_of(stream), probing_length,
                       (void *)status_out, StatusHandler::kId, StatusHandler::kIgnore);
    }

    /* device retrieve (single_value_hash_table.cuh:268-307) */
    __device__ status_type retrieve(const key_type key_in, value_type &value_out,
                                    const cg::thread_block_tile<cg_size()> &group,
                                    const index_type probing_length = defaults::probing_length()) const noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        typename layout::val_t v = 0;
        bool found = false;
        const status_type s(b200::tile_find<layout>(view_, group, key_in, v, found, false,
                                                    probing_length));
        if (found) value_out = value_of(v);
        return s;
    }

    /* host retrieve (single_value_hash_table.cuh:320-337) */
    template <class StatusHandler = defaults::status_handler_t>
    void retrieve(const key_type *const keys_in, const index_type num_in,
                  value_type *const values_out, const cudaStream_t stream = 0,
                  const index_type probing_length = defaults::probing_length(),
                  typename StatusHandler::base_type *const status_out = nullptr) const noexcept
    {
        static_assert(checks::is_status_handler<StatusHandler>(), "not a valid status handler type");
        if (!is_initialized_) return;
        wc_svht_retrieve(handle_, keys_in, num_in, values_out, stream_of(stream), probing_length,
                         (void *)status_out, StatusHandler::kId, StatusHandler::kIgnore);
    }

    /* retrieve_all (single_value_hash_table.cuh:391-417); synchronises */
    void retrieve_all(key_type *const keys_out, value_type *const values_out, index_type &num_out,
                      const cudaStream_t stream = 0) const noexcept
    {
        num_out = 0;
        if (!is_initialized_) return;
        std::uint64_t n = 0;
        if (wc_table_retrieve_all(handle_, keys_out, values_out, &n, stream_of(stream)) == WC_OK)
            num_out = n;
    }

    /* device erase (single_value_hash_table.cuh:426-468) */
    __device__ status_type erase(const key_type key_in, const cg::thread_block_tile<cg_size()> &group,
                                 const index_type probing_length = defaults::probing_length()) noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        return status_type(b200::tile_modify<layout>(view_, group, key_in, 0, 3, probing_length));
    }

    /* host erase (single_value_hash_table.cuh:480-496) */
    template <class StatusHandler = defaults::status_handler_t>
    void erase(const key_type *const keys_in, const index_type num_in, const cudaStream_t stream = 0,
               const index_type probing_length = defaults::probing_length(),
               typename StatusHandler::base_type *const status_out = nullptr) noexcept
    {
        static_assert(checks::is_status_handler<StatusHandler>(), "not a valid status handler type");
        if (!is_initialized_) return;
        wc_svht_erase(handle_, keys_in, num_in, stream_of(stream), probing_length,
                      (void *)status_out, StatusHandler::kId, StatusHandler::kIgnore);
    }

    /* for_each (single_value_hash_table.cuh:506-528): f(key, value) on every
     * occupied slot, in a kernel of the caller's translation unit */
    template <class Func>
    void for_each(Func f, const cudaStream_t stream = 0, const index_type smem_bytes = 0) const noexcept
    {
        if (!is_initialized_) return;
        const index_type blocks = (capacity_ + 255) / 256;
        detail::svht_for_each_kernel<<<unsigned(blocks), 256, smem_bytes, stream>>>(f, *this);
    }

    /* size / load_factor / storage_density (single_value_hash_table.cuh:535-611) */
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
    float storage_density(const cudaStream_t stream = 0) const noexcept { return load_factor(stream); }

    __host__ __device__ index_type capacity() const noexcept { return capacity_; }
    index_type bytes_total() const noexcept
    {
        wc_table_info inf;
        return (handle_ && wc_table_get_info(handle_, &inf) == WC_OK) ? inf.bytes_total : 0;
    }
    __host__ __device__ bool is_initialized() const noexcept { return is_initialized_; }

    /* peek_status / pop_status (single_value_hash_table.cuh:646-687) */
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
    __host__ __device__ bool is_copy() const noexcept { return is_copy_; }

    /* the device view of the slot array (for kernels of the caller) */
    __host__ __device__ const b200::TableView &device_view() const noexcept { return view_; }
    wc_table *handle() const noexcept { return handle_; }

  private:
    template <class F, class Table>
    friend __global__ void detail::svht_for_each_kernel(F, const Table);

    static wc_stream_t stream_of(cudaStream_t s) { return reinterpret_cast<wc_stream_t>(s); }
    __host__ __device__ static value_word value_bits(const value_type &v)
    {
        value_word w;
        memcpy(&w, &v, sizeof(w));
        return w;
    }
    __host__ __device__ static value_type value_of(const value_word w)
    {
        value_type v;
        memcpy(&v, &w, sizeof(v));
        return v;
    }
    void refresh() noexcept
    {
        wc_table_info inf;
        if (wc_table_get_info(handle_, &inf) != WC_OK) return;
        view_ = detail::view_from(inf);
        capacity_ = inf.capacity;
        is_initialized_ = inf.is_initialized != 0;
    }

    wc_table *handle_ = nullptr;
    b200::TableView view_{};
    index_type capacity_ = 0;
    bool is_initialized_ = false;
    bool is_copy_ = false;
};

namespace detail {
template <class F, class Table>
__global__ void svht_for_each_kernel(F f, const Table table)
{
    using K = typename Table::key_type;
    using L = typename Table::layout;
    const index_t tid = index_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (tid >= table.capacity()) return;
    const b200::TableView &t = table.device_view();
    unsigned char *const sp = reinterpret_cast<unsigned char *>(t.slots) + tid * L::kSlotBytes;
    const K key = *reinterpret_cast<const K *>(sp);
    if (!Table::is_valid_key(key)) return;
    if constexpr (b200::is_soa<L>::value)
        f(key, Table::value_of(b200::get_soa_value<L>(t, tid)));
    else
        f(key, Table::value_of(*b200::slot_value_ptr<L>(sp)));
}
} // namespace detail

} // namespace warpcore

#endif /* WARPCORE_B200_CXX_SVHT_CUH */
