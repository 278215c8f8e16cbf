/*
 * warpcore::BloomFilter -- drop-in for the reference class
 * (bloom_filter.cuh:15-421) over the B200-native library.  The bit pattern
 * of a key is the reference's (bloom_filter.cuh:168-237), so filters built
 * by the bulk kernels, by the device methods below and by the reference are
 * word-for-word identical.
 */
#ifndef WARPCORE_B200_CXX_BLOOM_CUH
#define WARPCORE_B200_CXX_BLOOM_CUH

#include <climits>

#include "base.cuh"

namespace warpcore {

template <class Key, class Hasher = defaults::hasher_t<Key>, class Slot = std::uint64_t,
          index_t CGSize = 1>
class BloomFilter {
    static_assert(checks::is_valid_key_type<Key>(), "invalid key type");
    static_assert(checks::is_hasher<Hasher>(), "not a valid hasher type");
    static_assert(std::is_same<Slot, std::uint32_t>::value || std::is_same<Slot, std::uint64_t>::value,
                  "invalid slot type");
    static_assert(checks::is_valid_cg_size(CGSize), "invalid cooperative group size");

  public:
    using key_type = Key;
    using value_type = bool;
    using index_type = index_t;
    using slot_type = Slot;
    using status_type = Status;

    __host__ __device__ static constexpr index_type cg_size() noexcept { return CGSize; }
    __host__ __device__ static constexpr index_type slot_bits() noexcept { return sizeof(slot_type) * CHAR_BIT; }
    __host__ __device__ static constexpr index_type block_bits() noexcept { return slot_bits() * cg_size(); }

    /* bloom_filter.cuh:78-93 */
    explicit BloomFilter(const index_type num_bits, const index_type k,
                         const key_type seed = defaults::seed<key_type>()) noexcept
    {
        wc_bloom_config cfg{std::uint32_t(sizeof(Key)), std::uint32_t(sizeof(Slot)),
                            std::uint32_t(CGSize), Hasher::kId};
        if (wc_bloom_create(&cfg, num_bits, k, std::uint64_t(seed), &handle_) == WC_OK) refresh();
    }
    __host__ __device__ BloomFilter(const BloomFilter &o) noexcept
        : handle_(o.handle_), words_(o.words_), num_bits_(o.num_bits_), num_slots_(o.num_slots_),
          num_blocks_(o.num_blocks_), k_(o.k_), seed_(o.seed_), is_copy_(true)
    {}
    BloomFilter(BloomFilter &&o) noexcept
        : handle_(o.handle_), words_(o.words_), num_bits_(o.num_bits_), num_slots_(o.num_slots_),
          num_blocks_(o.num_blocks_), k_(o.k_), seed_(o.seed_), is_copy_(o.is_copy_)
    {
        o.is_copy_ = true;
    }
#ifndef __CUDA_ARCH__
    ~BloomFilter() noexcept
    {
        if (!is_copy_ && handle_) wc_bloom_destroy(handle_);
    }
#endif

    void init(const key_type seed, const cudaStream_t stream = 0) noexcept
    {
        if (handle_ && wc_bloom_init(handle_, std::uint64_t(seed), reinterpret_cast<wc_stream_t>(stream)) == WC_OK)
            refresh();
    }
    void init(const cudaStream_t stream = 0) noexcept { init(seed_, stream); }

    /* device insert (bloom_filter.cuh:168-192) */
    __device__ void insert(const key_type key, const cg::thread_block_tile<cg_size()> &group) noexcept
    {
        const index_type idx = slot_index(key, group.thread_rank());
        const slot_type mask = lane_mask(key, group.thread_rank());
        if ((mask & words_[idx]) != mask) atomic_or(words_ + idx, mask);
    }

    /* host insert (bloom_filter.cuh:200-208) */
    void insert(const Key *const keys_in, const index_t num_in, const cudaStream_t stream = 0) noexcept
    {
        wc_bloom_insert(handle_, keys_in, num_in, reinterpret_cast<wc_stream_t>(stream));
    }

    /* device retrieve (bloom_filter.cuh:216-237) */
    __device__ bool retrieve(const key_type key, const cg::thread_block_tile<cg_size()> &group) const noexcept
    {
        const index_type idx = slot_index(key, group.thread_rank());
        const slot_type mask = lane_mask(key, group.thread_rank());
        return group.all((mask & words_[idx]) == mask);
    }

    /* host retrieve (bloom_filter.cuh:246-255) */
    void retrieve(const key_type *const keys_in, const index_type num_in, bool *const flags_out,
                  const cudaStream_t stream = 0) const noexcept
    {
        wc_bloom_retrieve(handle_, keys_in, num_in, reinterpret_cast<std::uint8_t *>(flags_out),
                          reinterpret_cast<wc_stream_t>(stream));
    }

    /* insert_and_query, CG 1 only (bloom_filter.cuh:263-297) */
    template <index_type CGSize_ = cg_size(), class = std::enable_if_t<CGSize_ == 1>>
    __device__ bool insert_and_query(const key_type key, const cg::thread_block_tile<cg_size()> &group) noexcept
    {
        const index_type idx = slot_index(key, 0);
        const slot_type mask = lane_mask(key, 0);
        if ((mask & words_[idx]) != mask) {
            const slot_type old = atomic_or(words_ + idx, mask);
            return (mask & old) == mask;
        }
        return true;
    }

    __host__ __device__ index_type num_bits() const noexcept { return num_bits_; }
    __host__ __device__ index_type num_slots() const noexcept { return num_slots_; }
    __host__ __device__ index_type num_blocks() const noexcept { return num_blocks_; }
    __host__ __device__ index_type k() const noexcept { return k_; }
    __host__ __device__ bool is_copy() const noexcept { return is_copy_; }
    __host__ __device__ const slot_type *words() const noexcept { return words_; }

    /* the reference's analytic estimate (bloom_filter.cuh:342-354) */
    double fpr(const index_type n) const noexcept
    {
        double r = 0;
        if (handle_) wc_bloom_fpr(handle_, n, &r);
        return r;
    }

  private:
    __host__ __device__ index_type slot_index(key_type key, index_type rank) const noexcept
    {
        return ((index_type(Hasher::hash(key_type(key + seed_))) % num_blocks_) * cg_size() + rank) %
               num_slots_;
    }
    __host__ __device__ slot_type lane_mask(key_type key, index_type rank) const noexcept
    {
        slot_type m = 0;
        for (index_type i = 0; i < k_; ++i) {
            const key_type seeded = key_type(key + seed_ + key_type(i));
            const index_type h = index_type(Hasher::hash(seeded)) % block_bits();
            if (h / slot_bits() == rank) m |= slot_type(1) << (h % slot_bits());
        }
        return m;
    }
    __device__ static slot_type atomic_or(slot_type *p, slot_type v)
    {
        if constexpr (sizeof(slot_type) == 8)
            return slot_type(atomicOr(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v));
        else
            return slot_type(atomicOr(reinterpret_cast<unsigned int *>(p), (unsigned int)v));
    }
    void refresh() noexcept
    {
        wc_bloom_info inf;
        if (wc_bloom_get_info(handle_, &inf) != WC_OK) return;
        words_ = reinterpret_cast<slot_type *>(inf.words);
        num_bits_ = inf.num_bits;
        num_slots_ = inf.num_slots;
        num_blocks_ = inf.num_blocks;
        k_ = inf.k;
        seed_ = key_type(inf.seed);
    }

    wc_bloom *handle_ = nullptr;
    slot_type *words_ = nullptr;
    index_type num_bits_ = 0, num_slots_ = 0, num_blocks_ = 0, k_ = 0;
    key_type seed_ = 0;
    bool is_copy_ = false;
};

} // namespace warpcore

#endif /* WARPCORE_B200_CXX_BLOOM_CUH */
