/*
 * warpcore::CountingHashTable -- drop-in for the reference class
 * (counting_hash_table.cuh:18-431) over the B200-native library.  Counts are
 * values of the slot; bulk inserts merge equal keys of a warp into one
 * increment; retrieve clamps to max_count (counting_hash_table.cuh:215-222).
 */
#ifndef WARPCORE_B200_CXX_COUNTING_CUH
#define WARPCORE_B200_CXX_COUNTING_CUH

#include "single_value_hash_table.cuh"

namespace warpcore {

namespace detail {
/* f(key, count) on every occupied slot, one thread per slot */
template <class F, class L, class K, class V>
__global__ void counting_for_each_kernel(F f, const b200::TableView t, index_t capacity, K empty,
                                         K tomb)
{
    const index_t tid = index_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (tid >= capacity) return;
    unsigned char *const sp = reinterpret_cast<unsigned char *>(t.slots) + tid * L::kSlotBytes;
    const K key = *reinterpret_cast<const K *>(sp);
    if (key != empty && key != tomb) f(key, V(*b200::slot_value_ptr<L>(sp)));
}
} // namespace detail

template <class Key, class Value = index_t, Key EmptyKey = defaults::empty_key<Key>(),
          Key TombstoneKey = defaults::tombstone_key<Key>(),
          class ProbingScheme = defaults::probing_scheme_t<Key, 4>,
          class TableStorage = defaults::table_storage_t<Key, Value>,
          index_t TempMemoryBytes = defaults::temp_memory_bytes()>
class CountingHashTable {
    static_assert(checks::is_valid_key_type<Key>(), "invalid key type");
    static_assert(checks::is_valid_counter_type<Value>(),
                  "counts are int, std::uint32_t or std::uint64_t");
    using layout = typename detail::layout_of<Key, typename std::make_unsigned<Value>::type>::type;

  public:
    using key_type = Key;
    using value_type = Value;
    using index_type = index_t;
    using status_type = Status;

    __host__ __device__ static constexpr key_type empty_key() noexcept { return EmptyKey; }
    __host__ __device__ static constexpr key_type tombstone_key() noexcept { return TombstoneKey; }
    __host__ __device__ static constexpr index_type cg_size() noexcept { return ProbingScheme::cg_size(); }

    /* counting_hash_table.cuh:75-85 */
    explicit CountingHashTable(index_type min_capacity, key_type seed = defaults::seed<key_type>(),
                               value_type max_count = std::numeric_limits<value_type>::max(),
                               bool no_init = false) noexcept
    {
        const wc_table_config cfg =
            detail::make_config<ProbingScheme, Key>(sizeof(Value), EmptyKey, TombstoneKey);
        detail::load_tuning_once();
        if (wc_counting_create(&cfg, min_capacity, std::uint64_t(seed), std::uint64_t(max_count),
                               no_init ? 1 : 0, &handle_) == WC_OK)
            refresh();
        max_count_ = max_count;
    }
    __host__ __device__ CountingHashTable(const CountingHashTable &o) noexcept
        : handle_(o.handle_), view_(o.view_), capacity_(o.capacity_), max_count_(o.max_count_),
          is_initialized_(o.is_initialized_), is_copy_(true)
    {}
    CountingHashTable(CountingHashTable &&o) noexcept
        : handle_(o.handle_), view_(o.view_), capacity_(o.capacity_), max_count_(o.max_count_),
          is_initialized_(o.is_initialized_), is_copy_(o.is_copy_)
    {
        o.is_copy_ = true;
    }
#ifndef __CUDA_ARCH__
    ~CountingHashTable() noexcept
    {
        if (!is_copy_ && handle_) wc_table_destroy(handle_);
    }
#endif

    void init(const key_type seed, const cudaStream_t stream = 0) noexcept
    {
        if (handle_ && wc_table_init(handle_, std::uint64_t(seed), stream_of(stream)) == WC_OK)
            refresh();
    }
    void init(const cudaStream_t stream = 0) noexcept { init(seed(), stream); }

    /* device insert (counting_hash_table.cuh:142-172) */
    __device__ status_type insert(key_type key_in, const cg::thread_block_tile<cg_size()> &group,
                                  index_type probing_length = defaults::probing_length()) noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        return status_type(b200::tile_modify<layout>(view_, group, key_in, 0, 1, probing_length));
    }

    /* host insert (counting_hash_table.cuh:184-194) */
    template <class StatusHandler = defaults::status_handler_t>
    void insert(const key_type *keys_in, index_type num_in, cudaStream_t stream = 0,
                index_type probing_length = defaults::probing_length(),
                typename StatusHandler::base_type *status_out = nullptr) noexcept
    {
        if (!is_initialized_) return;
        wc_counting_insert(handle_, keys_in, num_in, stream_of(stream), probing_length,
                           (void *)status_out, StatusHandler::kId, StatusHandler::kIgnore);
    }

    /* device retrieve (counting_hash_table.cuh:204-225) */
    __device__ status_type retrieve(key_type key_in, value_type &value_out,
                                    const cg::thread_block_tile<cg_size()> &group,
                                    index_type probing_length = defaults::probing_length()) const noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        typename layout::val_t v = 0;
        bool found = false;
        const status_type s(b200::tile_find<layout>(view_, group, key_in, v, found, false,
                                                    probing_length));
        value_out = found ? value_type(v) : value_type(0);
        return s;
    }

    /* host retrieve (counting_hash_table.cuh:238-249) */
    template <class StatusHandler = defaults::status_handler_t>
    void retrieve(const key_type *keys_in, index_type num_in, value_type *values_out,
                  cudaStream_t stream = 0, index_type probing_length = defaults::probing_length(),
                  typename StatusHandler::base_type *status_out = nullptr) const noexcept
    {
        if (!is_initialized_) return;
        wc_counting_retrieve(handle_, keys_in, num_in, values_out, stream_of(stream),
                             probing_length, (void *)status_out, StatusHandler::kId,
                             StatusHandler::kIgnore);
    }

    void retrieve_all(key_type *keys_out, value_type *values_out, index_t &num_out,
                      cudaStream_t stream = 0) const noexcept
    {
        num_out = 0;
        if (!is_initialized_) return;
        std::uint64_t n = 0;
        if (wc_table_retrieve_all(handle_, keys_out, values_out, &n, stream_of(stream)) == WC_OK)
            num_out = n;
    }

    __device__ status_type erase(key_type key_in, const cg::thread_block_tile<cg_size()> &group,
                                 index_type probing_length = defaults::probing_length()) noexcept
    {
        if (!is_initialized_) return status_type::not_initialized();
        return status_type(b200::tile_modify<layout>(view_, group, key_in, 0, 3, probing_length));
    }

    /* host erase; the reference passes its arguments in the wrong order
     * (counting_hash_table.cuh:299-300), this one forwards the stream */
    template <class StatusHandler = defaults::status_handler_t>
    void erase(key_type *keys_in, index_type num_in, cudaStream_t stream = 0,
               index_type probing_length = defaults::probing_length(),
               typename StatusHandler::base_type *status_out = nullptr) noexcept
    {
        if (!is_initialized_) return;
        wc_counting_erase(handle_, keys_in, num_in, stream_of(stream), probing_length,
                          (void *)status_out, StatusHandler::kId, StatusHandler::kIgnore);
    }

    /* for_each (counting_hash_table.cuh:303-317): f(key, count) on every
     * key of the table, a device lambda, asynchronous on `stream` */
    template <class Func>
    void for_each(Func f, cudaStream_t stream = 0, index_type smem_bytes = 0) const noexcept
    {
        if (!is_initialized_ || capacity_ == 0) return;
        const index_type blocks = (capacity_ + 255) / 256;
        detail::counting_for_each_kernel<Func, layout, key_type, value_type>
            <<<unsigned(blocks), 256, smem_bytes, stream>>>(f, view_, capacity_, EmptyKey,
                                                            TombstoneKey);
    }

    index_type size(cudaStream_t stream = 0) const noexcept
    {
        if (!is_initialized_) return 0;
        std::uint64_t n = 0;
        wc_table_size(handle_, stream_of(stream), &n);
        return n;
    }
    float load_factor(cudaStream_t stream = 0) const noexcept { return float(size(stream)) / float(capacity()); }
    float storage_density(cudaStream_t stream = 0) const noexcept { return load_factor(stream); }
    __host__ __device__ index_type capacity() const noexcept { return capacity_; }
    __host__ __device__ value_type max_count() const noexcept { return max_count_; }
    index_type bytes_total() const noexcept
    {
        wc_table_info inf;
        return (handle_ && wc_table_get_info(handle_, &inf) == WC_OK) ? inf.bytes_total : 0;
    }
    __host__ __device__ bool is_initialized() const noexcept { return is_initialized_; }
    status_type peek_status(cudaStream_t stream = 0) const noexcept
    {
        std::uint32_t s = WC_STATUS_NOT_INITIALIZED;
        if (handle_) wc_table_peek_status(handle_, stream_of(stream), &s);
        return status_type(s);
    }
    status_type pop_status(cudaStream_t stream = 0) noexcept
    {
        std::uint32_t s = WC_STATUS_NOT_INITIALIZED;
        if (handle_) wc_table_pop_status(handle_, stream_of(stream), &s);
        return status_type(s);
    }
    __host__ __device__ static constexpr bool is_empty_key(key_type key) noexcept
    {
        return key == empty_key();
    }
    __host__ __device__ static constexpr bool is_tombstone_key(key_type key) noexcept
    {
        return key == tombstone_key();
    }
    __host__ __device__ static constexpr bool is_valid_key(key_type key) noexcept
    {
        return key != empty_key() && key != tombstone_key();
    }
    __host__ __device__ key_type seed() const noexcept { return key_type(view_.seed); }
    __host__ __device__ bool is_copy() const noexcept { return is_copy_; }
    __host__ __device__ const b200::TableView &device_view() const noexcept { return view_; }

  private:
    static wc_stream_t stream_of(cudaStream_t s) { return reinterpret_cast<wc_stream_t>(s); }
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
    value_type max_count_ = 0;
    bool is_initialized_ = false;
    bool is_copy_ = false;
};

} // namespace warpcore

#endif /* WARPCORE_B200_CXX_COUNTING_CUH */
