/*
 * warpcore/base.cuh -- C++ drop-in front end of the B200-native library.
 *
 * Same names and template knobs as the reference's headers
 * (include/warpcore/{base,tags,checks,status,hashers,probing_schemes,
 * defaults}.cuh).  Host bulk methods call the C ABI of libwarpcore_b200.so
 * (include/warpcore_b200.h); device per-key methods run the bucket-aligned
 * probing of warpcore/detail/b200_core.cuh, so both agree on where keys live.
 * Compile with nvcc (-std=c++17) and link -lwarpcore_b200.
 */
#ifndef WARPCORE_B200_CXX_BASE_CUH
#define WARPCORE_B200_CXX_BASE_CUH

#include <cstdint>
#include <cstring>
#include <limits>
#include <ostream>
#include <string>
#include <type_traits>
#include <vector>

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <warpcore_b200.h>
#include <warpcore/detail/b200_core.cuh>

namespace warpcore {

namespace cg = cooperative_groups;

using index_t = std::uint64_t;       /* base.cuh:21 */
using status_base_t = std::uint32_t; /* base.cuh:22 */

namespace detail {
/* base.cuh:27-34 */
inline index_t get_valid_capacity(index_t min_capacity, index_t cg_size) noexcept
{
    return wc_valid_capacity(min_capacity, cg_size);
}
} // namespace detail

/* ------------------------------------------------------------------ */
/* tags and checks (tags.cuh:9-21, checks.cuh:12-116)                  */
/* ------------------------------------------------------------------ */

namespace tags {
struct hasher {};
struct true_permutation_hasher {};
struct probing_scheme {};
struct cycle_free_probing_scheme {};
struct key_value_storage {};
struct dynamic_value_storage {};
struct status_handler {};
} // namespace tags

namespace checks {
__host__ __device__ constexpr bool is_valid_cg_size(index_t c) noexcept
{
    return c == 1 || c == 2 || c == 4 || c == 8 || c == 16 || c == 32;
}
template <class T>
__host__ __device__ constexpr bool is_valid_key_type() noexcept
{
    return std::is_same<T, std::uint32_t>::value || std::is_same<T, std::uint64_t>::value;
}
/* checks.cuh:46-61: values are any trivially copyable type (this build
 * stores 4- or 8-byte ones); counters are int, u32 or u64 */
template <class T>
__host__ __device__ constexpr bool is_valid_value_type() noexcept
{
    return std::is_trivially_copyable<T>::value;
}
template <class T>
__host__ __device__ constexpr bool is_valid_counter_type() noexcept
{
    return std::is_same<T, int>::value || std::is_same<T, std::uint32_t>::value ||
           std::is_same<T, std::uint64_t>::value;
}
template <class T>
__host__ __device__ constexpr bool is_hasher() noexcept
{
    return std::is_same<typename T::tag, tags::hasher>::value ||
           std::is_same<typename T::tag, tags::true_permutation_hasher>::value;
}
template <class T>
__host__ __device__ constexpr bool is_probing_scheme() noexcept
{
    return std::is_same<typename T::tag, tags::probing_scheme>::value ||
           std::is_same<typename T::tag, tags::cycle_free_probing_scheme>::value;
}
template <class T>
__host__ __device__ constexpr bool is_cycle_free_probing_scheme() noexcept
{
    return std::is_same<typename T::tag, tags::cycle_free_probing_scheme>::value;
}
template <class T>
__host__ __device__ constexpr bool is_status_handler() noexcept
{
    return std::is_same<typename T::tag, tags::status_handler>::value;
}
} // namespace checks

/* ------------------------------------------------------------------ */
/* Status (status.cuh:16-214); bit values are the reference's ABI       */
/* ------------------------------------------------------------------ */

class Status {
  public:
    using base_type = status_base_t;

    Status() noexcept = default;
    __host__ __device__ constexpr explicit Status(base_type s) noexcept : status_(s) {}

    __host__ __device__ constexpr base_type base() const noexcept { return status_; }
    __host__ __device__ constexpr operator base_type() const noexcept { return status_; }

    __host__ __device__ static constexpr Status none() noexcept { return Status(0u); }
    __host__ __device__ static constexpr Status all() noexcept { return Status(kMask); }
#define WC_STATUS_FLAG(name, bit)                                                           \
    __host__ __device__ static constexpr Status name() noexcept { return Status(1u << bit); } \
    __host__ __device__ constexpr bool has_##name() const noexcept { return status_ & (1u << bit); }
    WC_STATUS_FLAG(unknown_error, 0)
    WC_STATUS_FLAG(probing_length_exceeded, 1)
    WC_STATUS_FLAG(invalid_configuration, 2)
    WC_STATUS_FLAG(invalid_key, 3)
    WC_STATUS_FLAG(duplicate_key, 4)
    WC_STATUS_FLAG(key_not_found, 5)
    WC_STATUS_FLAG(index_overflow, 6)
    WC_STATUS_FLAG(out_of_memory, 7)
    WC_STATUS_FLAG(not_initialized, 8)
    WC_STATUS_FLAG(dry_run, 9)
    WC_STATUS_FLAG(invalid_phase_overlap, 10)
    WC_STATUS_FLAG(max_values_for_key_reached, 11)
    WC_STATUS_FLAG(invalid_value, 12)
#undef WC_STATUS_FLAG

    __host__ __device__ static constexpr Status error_mask() noexcept
    {
        return Status((1u << 0) | (1u << 2) | (1u << 6) | (1u << 7) | (1u << 8) | (1u << 10));
    }
    __host__ __device__ static constexpr Status warning_mask() noexcept
    {
        return Status(kMask & ~error_mask().status_);
    }
    __host__ __device__ constexpr Status get_errors() const noexcept
    {
        return Status(status_ & error_mask().status_);
    }
    __host__ __device__ constexpr Status get_warnings() const noexcept
    {
        return Status(status_ & warning_mask().status_);
    }
    __host__ __device__ constexpr bool has_any(const Status &s = all()) const noexcept
    {
        return status_ & s.status_;
    }
    __host__ __device__ constexpr bool has_any_errors() const noexcept { return has_any(error_mask()); }
    __host__ __device__ constexpr bool has_any_warnings() const noexcept { return has_any(warning_mask()); }
    __host__ __device__ constexpr bool has_all(const Status &s = all()) const noexcept
    {
        return (status_ & s.status_) == s.status_;
    }
    /* the reference's complement: (~s) ^ mask (status.cuh:142-146) */
    __host__ __device__ constexpr Status operator~() const noexcept { return Status((~status_) ^ kMask); }
    __host__ __device__ constexpr Status &operator+=(const Status &a) noexcept
    {
        status_ |= a.status_;
        return *this;
    }
    __host__ __device__ constexpr Status operator+(const Status &a) const noexcept
    {
        return Status(status_ | a.status_);
    }
    __host__ __device__ constexpr Status operator-(const Status &a) const noexcept
    {
        return Status(status_ - (status_ & a.status_));
    }
    __host__ __device__ constexpr Status &operator-=(const Status &a) noexcept
    {
        status_ -= status_ & a.status_;
        return *this;
    }
    __host__ __device__ constexpr bool operator==(const Status &a) const noexcept { return status_ == a.status_; }
    __host__ __device__ constexpr bool operator!=(const Status &a) const noexcept { return status_ != a.status_; }

    /* Status::atomic_join (status.cuh:187-193) */
    __device__ void atomic_join(Status s) noexcept
    {
        if (!has_all(s)) atomicOr(&status_, s.status_);
    }

  private:
    static constexpr base_type kMask = 0xFFFu;
    base_type status_ = 0;
};

inline std::ostream &operator<<(std::ostream &os, Status s)
{
    static const char *names[] = {"unknown error", "probing length exceeded", "invalid configuration",
                                  "invalid key", "duplicate key", "key not found", "index overflow",
                                  "out of memory", "not initialized", "dry run",
                                  "invalid phase overlap", "max values for key reached",
                                  "invalid value"};
    os << "[";
    bool first = true;
    for (int b = 0; b < 13; ++b)
        if (s.base() & (1u << b)) {
            os << (first ? "" : ", ") << names[b];
            first = false;
        }
    return os << "]";
}

/* per-key status handlers (status.cuh:278-333) */
namespace status_handlers {
struct ReturnNothing {
    using base_type = void;
    using tag = tags::status_handler;
    static constexpr int kId = WC_HANDLER_NOTHING;
    static constexpr status_base_t kIgnore = 0;
};
struct ReturnStatus {
    using base_type = Status;
    using tag = tags::status_handler;
    static constexpr int kId = WC_HANDLER_STATUS;
    static constexpr status_base_t kIgnore = 0;
};
template <status_base_t Ignore = 0>
struct ReturnBoolean {
    using base_type = bool;
    using tag = tags::status_handler;
    static constexpr int kId = WC_HANDLER_BOOLEAN;
    static constexpr status_base_t kIgnore = Ignore;
};
} // namespace status_handlers

/* ------------------------------------------------------------------ */
/* hashers (hashers.cuh:14-175)                                         */
/* ------------------------------------------------------------------ */

namespace hashers {
class NvidiaHash {
  public:
    using key_type = std::uint32_t;
    using hash_type = std::uint32_t;
    using tag = tags::hasher;
    static constexpr std::uint32_t kId = WC_HASH_NVIDIA;
    __host__ __device__ static hash_type hash(key_type x) noexcept { return b200::nvidia_hash32(x); }
};
class MuellerHash {
  public:
    using key_type = std::uint32_t;
    using hash_type = std::uint32_t;
    using tag = tags::true_permutation_hasher;
    static constexpr std::uint32_t kId = WC_HASH_MUELLER;
    __host__ __device__ static hash_type hash(key_type x) noexcept { return b200::mueller_hash32(x); }
};
template <class K>
class MurmurHash {
  public:
    using key_type = K;
    using hash_type = K;
    using tag = tags::true_permutation_hasher;
    static constexpr std::uint32_t kId = WC_HASH_MURMUR;
    __host__ __device__ static K hash(K x) noexcept
    {
        if constexpr (sizeof(K) == 4) return K(b200::fmix32(std::uint32_t(x)));
        else return K(b200::fmix64(std::uint64_t(x)));
    }
};
template <class K, class H = std::uint32_t>
class IdentityMap {
  public:
    using key_type = K;
    using hash_type = H;
    using tag = tags::true_permutation_hasher;
    static constexpr std::uint32_t kId = sizeof(H) == 4 ? WC_HASH_IDENTITY32 : WC_HASH_IDENTITY64;
    __host__ __device__ static hash_type hash(key_type x) noexcept { return hash_type(x); }
};
} // namespace hashers

/* ------------------------------------------------------------------ */
/* probing schemes (probing_schemes.cuh:22-305) as configuration tags   */
/* ------------------------------------------------------------------ */

namespace probing_schemes {
template <class Hasher1, class Hasher2, index_t CGSize = 1>
class DoubleHashing {
    static_assert(checks::is_valid_cg_size(CGSize), "invalid cooperative group size");
  public:
    using key_type = typename Hasher1::key_type;
    using tag = typename std::conditional<
        std::is_same<typename Hasher1::tag, tags::true_permutation_hasher>::value &&
            std::is_same<typename Hasher2::tag, tags::true_permutation_hasher>::value,
        tags::cycle_free_probing_scheme, tags::probing_scheme>::type;
    static constexpr std::uint32_t kId = WC_PROBING_DOUBLE;
    static constexpr std::uint32_t kHasher1 = Hasher1::kId;
    static constexpr std::uint32_t kHasher2 = Hasher2::kId;
    __host__ __device__ static constexpr index_t cg_size() noexcept { return CGSize; }
};
template <class Hasher, index_t CGSize = 1>
class LinearProbing {
    static_assert(checks::is_valid_cg_size(CGSize), "invalid cooperative group size");
  public:
    using key_type = typename Hasher::key_type;
    using tag = tags::cycle_free_probing_scheme;
    static constexpr std::uint32_t kId = WC_PROBING_LINEAR;
    static constexpr std::uint32_t kHasher1 = Hasher::kId;
    static constexpr std::uint32_t kHasher2 = Hasher::kId;
    __host__ __device__ static constexpr index_t cg_size() noexcept { return CGSize; }
};
template <class Hasher, index_t CGSize = 1>
class QuadraticProbing {
    static_assert(checks::is_valid_cg_size(CGSize), "invalid cooperative group size");
  public:
    using key_type = typename Hasher::key_type;
    using tag = tags::probing_scheme;
    static constexpr std::uint32_t kId = WC_PROBING_QUADRATIC;
    static constexpr std::uint32_t kHasher1 = Hasher::kId;
    static constexpr std::uint32_t kHasher2 = Hasher::kId;
    __host__ __device__ static constexpr index_t cg_size() noexcept { return CGSize; }
};
} // namespace probing_schemes

namespace storage {
namespace key_value {
/* the AoS slot store (storage.cuh:438-645): {key, value} slots */
template <class Key, class Value>
struct AoSStore {
    using key_type = Key;
    using value_type = Value;
    using tag = tags::key_value_storage;
};
/* SoAStore (storage.cuh:218-432): SingleValueHashTable<..., SoAStore<K, V>>
 * stores its keys and values as two arrays (wc_svht_create_soa): the key
 * array is probed like a hash set's slots, value i belongs to key slot i,
 * and an insert writes the value after the key's compare-and-swap, as the
 * reference's SoA store does.  The other tables accept the type and keep
 * their own layout (counting tables {key, count} slots, so that a claim
 * publishes both; multi-value tables their key and value arrays).  Answers
 * do not depend on the store. */
template <class Key, class Value>
struct SoAStore {
    using key_type = Key;
    using value_type = Value;
    using tag = tags::key_value_storage;
};
} // namespace key_value
namespace multi_value {
/* BucketListStore<Value, BucketIndexBits, ValueCounterBits, BucketSizeBits>
 * (storage.cuh:890-1454): names the value type and the bit widths of the
 * bucket-list handles; the store itself lives in the library */
template <class Value, index_t BucketIndexBits = 32, index_t ValueCounterBits = 20,
          index_t BucketSizeBits = 10>
struct BucketListStore {
    static_assert(BucketIndexBits + ValueCounterBits + BucketSizeBits + 2 <= 64,
                  "Too many bits for bucket index and value counter and bucket size.");
    using value_type = Value;
    using index_type = index_t;
    using tag = tags::dynamic_value_storage;
    struct handle_type {
        __host__ __device__ static constexpr index_t max_bucket_index() noexcept
        {
            return (index_t{1} << BucketIndexBits) - 1;
        }
        __host__ __device__ static constexpr index_t max_value_count() noexcept
        {
            return (index_t{1} << ValueCounterBits) - 1;
        }
        __host__ __device__ static constexpr index_t max_bucket_size() noexcept
        {
            return (index_t{1} << BucketSizeBits) - 1;
        }
    };
    __host__ __device__ static constexpr index_t bucket_index_bits() noexcept { return BucketIndexBits; }
    __host__ __device__ static constexpr index_t value_counter_bits() noexcept { return ValueCounterBits; }
    __host__ __device__ static constexpr index_t bucket_size_bits() noexcept { return BucketSizeBits; }
};
} // namespace multi_value
} // namespace storage

/* defaults.cuh:9-44 */
namespace defaults {
template <class Key>
__host__ __device__ constexpr Key empty_key() noexcept { return Key{0}; }
template <class Key>
__host__ __device__ constexpr Key tombstone_key() noexcept { return ~Key{0}; }
template <class Key>
__host__ __device__ constexpr Key seed() noexcept { return Key{0x5ad0ded}; }
__host__ __device__ constexpr index_t temp_memory_bytes() noexcept { return 2048; }
__host__ __device__ constexpr index_t probing_length() noexcept { return ~index_t(0) - 1024; }
template <class Key>
using hasher_t = hashers::MurmurHash<Key>;
template <class Key, index_t CGSize>
using probing_scheme_t = probing_schemes::DoubleHashing<hasher_t<Key>, hasher_t<Key>, CGSize>;
using status_handler_t = status_handlers::ReturnNothing;
template <class Key, class Value>
using table_storage_t = storage::key_value::AoSStore<Key, Value>;
template <class Value>
using value_storage_t = storage::multi_value::BucketListStore<Value>;
} // namespace defaults

namespace detail {

/* slot layout of a (key, value) pair of widths; 0 = hash set */
template <class Key, class Value>
struct layout_of;
template <>
struct layout_of<std::uint32_t, std::uint32_t> { using type = b200::LayoutKV32; };
template <>
struct layout_of<std::uint64_t, std::uint64_t> { using type = b200::LayoutKV64; };
template <>
struct layout_of<std::uint32_t, std::uint64_t> { using type = b200::LayoutK32V64; };
template <>
struct layout_of<std::uint64_t, std::uint32_t> { using type = b200::LayoutK64V32; };
template <>
struct layout_of<std::uint32_t, void> { using type = b200::LayoutSet32; };
template <>
struct layout_of<std::uint64_t, void> { using type = b200::LayoutSet64; };

/* storage::key_value::SoAStore selects the struct-of-arrays layout */
template <class Store>
struct is_soa_store : std::false_type {};
template <class K, class V>
struct is_soa_store<storage::key_value::SoAStore<K, V>> : std::true_type {};

/* device-usable description of a table handle, refreshed from the C ABI */
/* the launch geometry measured by the autotuner (tuning_b200.json next to
 * the library, or WARPCORE_B200_TUNING), loaded once per process */
inline void load_tuning_once()
{
    static const int loaded = [] {
        std::uint64_t n = 0;
        return wc_tune_load(nullptr, &n);
    }();
    (void)loaded;
}

inline b200::TableView view_from(const wc_table_info &inf)
{
    b200::TableView v{};
    v.slots = inf.slots;
    v.status = inf.status;
    v.fps = inf.fingerprints;
    v.live = inf.live;
    v.num_buckets = inf.num_buckets;
    v.seed = inf.seed;
    v.empty_key = inf.empty_key;
    v.tombstone_key = inf.tombstone_key;
    v.max_count = inf.max_count;
    v.magic_nb = b200::barrett_magic(inf.num_buckets);
    v.magic_nb1 = b200::barrett_magic(inf.num_buckets > 1 ? inf.num_buckets - 1 : 1);
    v.probing = inf.probing;
    v.hasher1 = inf.hasher1;
    v.hasher2 = inf.hasher2;
    v.cg_size = inf.cg_size;
    v.values = inf.values;
    return v;
}

template <class ProbingScheme, class Key>
inline wc_table_config make_config(std::uint32_t value_bytes, Key empty, Key tomb)
{
    wc_table_config c{};
    c.key_bytes = sizeof(Key);
    c.value_bytes = value_bytes;
    c.empty_key = std::uint64_t(empty);
    c.tombstone_key = std::uint64_t(tomb);
    c.probing = ProbingScheme::kId;
    c.hasher1 = ProbingScheme::kHasher1;
    c.hasher2 = ProbingScheme::kHasher2;
    c.cg_size = std::uint32_t(ProbingScheme::cg_size());
    return c;
}

} // namespace detail

} // namespace warpcore

#endif /* WARPCORE_B200_CXX_BASE_CUH */
