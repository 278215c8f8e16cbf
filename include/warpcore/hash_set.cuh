/*
 * warpcore::HashSet -- drop-in for the reference class (hash_set.cuh:16-739)
 * over the B200-native library.  Unlike the reference, the host bulk
 * retrieve compiles (the reference's launches kernels::retrieve, which needs
 * a value_type the set does not have, hash_set.cuh:356).
 */
#ifndef WARPCORE_B200_CXX_HASH_SET_CUH
#define WARPCORE_B200_CXX_HASH_SET_CUH

#include "base.cuh"
#include "detail/tile_ops.cuh"

namespace warpcore {

namespace detail {
template <class F, class Set>
__global__ void set_for_each_kernel(F f, const Set set);
}

template <class Key, Key EmptyKey = defaults::empty_key<Key>(),
          Key TombstoneKey = defaults::tombstone_key<Key>(),
          class ProbingScheme = defaults::probing_scheme_t<Key, 16>,
          index_t TempMemoryBytes = defaults::temp_memory_bytes()>
class HashSet {
    static_assert(checks::is_valid_key_type<Key>(), "invalid key type");
    static_assert(EmptyKey != TombstoneKey, "empty key and tombstone key must not be identical");
    static_assert(checks::is_probing_scheme<ProbingScheme>(), "not a valid probing scheme type");

    using layout = typename detail::layout_of<Key, void>::type;

  public:
    using key_type = Key;
    using index_type = index_t;
    using status_type = Status;

    __host__ __device__ static constexpr key_type empty_key() noexcept { return EmptyKey; }
    __host__ __device__ static constexpr key_type tombstone_key() noexcept { return TombstoneKey; }
    __host__ __device__ static constexpr index_type cg_size() noexcept { return ProbingScheme::cg_size(); }

    /* hash_set.cuh:81-110 */
    explicit HashSet(index_type min_capacity, key_type seed = defaults::seed<key_type>()) noexcept
    {
        const wc_table_config cfg = detail::make_config<ProbingScheme, Key>(0, EmptyKey, TombstoneKey);
        detail::load_tuning_once();
        if (wc_hashset_create(&cfg, min_capacity, std::uint64_t(seed), &handle_) == WC_OK) refresh();
    }
    __host__ __device__ HashSet(const HashSet &o) noexcept
        : handle_(o.handle_), view_(o.view_), capacity_(o.capacity_),
          is_initialized_(o.is_initialized_), is_copy_(true)
    {}
    HashSet(HashSet &&o) noexcept
        : handle_(o.handle_), view_(o.view_), capacity_(o.capacity_),
          is_initialized_(o.is_initialized_), is_copy_(o.is_copy_)
    {
        o.is_copy_ = true;
    }
#ifndef __CUDA_ARCH__
    ~HashSet() noexcept
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

    /* device insert (hash_set.cuh:193-254) */
    __device__ Status insert(key_type key_in, const cg::thread_block_tile<cg_size()> &group,
                             index_type probing_length = defaults::probing_length()) noexcept
    {
        if (!is_initialized_) return Status::not_initialized();
        return Status(b200::tile_modify<layout>(view_, group, key_in, 0, 0, probing_length));
    }

    /* host insert (hash_set.cuh:266-282) */
    template <class StatusHandler = defaults::status_handler_t>
    void insert(const key_type *keys_in, index_type num_in, cudaStream_t stream = 0,
                index_type probing_length = defaults::probing_length(),
                typename StatusHandler::base_type *status_out = nullptr) noexcept
    {
        if (!is_initialized_) return;
        wc_hashset_insert(handle_, keys_in, num_in, stream_of(stream), probing_length,
                          (void *)status_out, StatusHandler::kId, StatusHandler::kIgnore);
    }

    /* device retrieve (hash_set.cuh:292-329) */
    __device__ Status retrieve(Key key_in, bool &flag_out, const cg::thread_block_tile<cg_size()> &group,
                               index_type probing_length = defaults::probing_length()) const noexcept
    {
        if (!is_initialized_) return Status::not_initialized();
        typename layout::val_t v = 0;
        bool found = false;
        const Status s(b200::tile_find<layout>(view_, group, key_in, v, found, true, probing_length));
        if (!s.has_any()) flag_out = found;
        return s;
    }

    /* host retrieve (hash_set.cuh:342-359): one bool per key */
    template <class StatusHandler = defaults::status_handler_t>
    void retrieve(const key_type *keys_in, index_type num_in, bool *flags_out, cudaStream_t stream = 0,
                  index_type probing_length = defaults::probing_length(),
                  typename StatusHandler::base_type *status_out = nullptr) const noexcept
    {
        if (!is_initialized_) return;
        wc_hashset_retrieve(handle_, keys_in, num_in, reinterpret_cast<std::uint8_t *>(flags_out),
                            stream_of(stream), probing_length, (void *)status_out,
                            StatusHandler::kId, StatusHandler::kIgnore);
    }

    /* retrieve_all (hash_set.cuh:367-384) */
    void retrieve_all(key_type *keys_out, index_type &num_out, cudaStream_t stream = 0) const noexcept
    {
        num_out = 0;
        if (!is_initialized_) return;
        std::uint64_t n = 0;
        if (wc_table_retrieve_all(handle_, keys_out, nullptr, &n, stream_of(stream)) == WC_OK)
            num_out = n;
    }

    /* device erase (hash_set.cuh:396-438) */
    __device__ Status erase(key_type key_in, const cg::thread_block_tile<cg_size()> &group,
                            index_type probing_length = defaults::probing_length()) noexcept
    {
        if (!is_initialized_) return Status::not_initialized();
        const Status s(b200::tile_modify<layout>(view_, group, key_in, 0, 3, probing_length));
        return s.has_invalid_key() ? s : Status::none();
    }

    /* host erase (hash_set.cuh:450-462) */
    template <class StatusHandler = defaults::status_handler_t>
    void erase(key_type *keys_in, index_type num_in, cudaStream_t stream = 0,
               index_type probing_length = defaults::probing_length(),
               typename StatusHandler::base_type *status_out = nullptr) noexcept
    {
        if (!is_initialized_) return;
        wc_hashset_erase(handle_, keys_in, num_in, stream_of(stream), probing_length,
                         (void *)status_out, StatusHandler::kId, StatusHandler::kIgnore);
    }

    /* for_each (hash_set.cuh:470-494): f(key) on every occupied slot */
    template <class Func>
    void for_each(Func f, cudaStream_t stream = 0, index_type smem_bytes = 0) const noexcept
    {
        if (!is_initialized_) return;
        detail::set_for_each_kernel<<<unsigned((capacity_ + 255) / 256), 256, smem_bytes, stream>>>(f, *this);
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
    index_type bytes_total() const noexcept
    {
        wc_table_info inf;
        return (handle_ && wc_table_get_info(handle_, &inf) == WC_OK) ? inf.bytes_total : 0;
    }
    __host__ __device__ bool is_initialized() const noexcept { return is_initialized_; }
    Status peek_status(cudaStream_t stream = 0) const noexcept
    {
        std::uint32_t s = WC_STATUS_NOT_INITIALIZED;
        if (handle_) wc_table_peek_status(handle_, stream_of(stream), &s);
        return Status(s);
    }
    Status pop_status(cudaStream_t stream = 0) noexcept
    {
        std::uint32_t s = WC_STATUS_NOT_INITIALIZED;
        if (handle_) wc_table_pop_status(handle_, stream_of(stream), &s);
        return Status(s);
    }
    __host__ __device__ static constexpr bool is_empty_key(key_type key) noexcept { return key == empty_key(); }
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
    bool is_initialized_ = false;
    bool is_copy_ = false;
};

namespace detail {
template <class F, class Set>
__global__ void set_for_each_kernel(F f, const Set set)
{
    using K = typename Set::key_type;
    const index_t tid = index_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (tid >= set.capacity()) return;
    const K key = reinterpret_cast<const K *>(set.device_view().slots)[tid];
    if (Set::is_valid_key(key)) f(key);
}
} // namespace detail

} // namespace warpcore

#endif /* WARPCORE_B200_CXX_HASH_SET_CUH */
