/* Stand-in for hpc_helpers' packed_types.cuh, which the reference headers
 * include but do not ship.  Written from the names the reference's
 * BucketListStore uses (storage.cuh:665-880): PackedPair<A, B> and
 * PackedQuadruple<A, B, C, D> hold unsigned fields of the given bit widths
 * in one word, with getters first() .. fourth(), setters of the same
 * names, first_as<T>(), equality, and atomicCAS / atomicExch on the word.
 * The field order inside the word is this stand-in's own; nothing in the
 * reference depends on it. */
#ifndef WC_REF_PACKED_TYPES_STANDIN
#define WC_REF_PACKED_TYPES_STANDIN
#include <cstdint>
#include <type_traits>

namespace packed_types {

namespace detail {
template <std::uint64_t Bits>
using word_t = typename std::conditional<(Bits <= 32), unsigned int, unsigned long long>::type;

template <std::uint64_t W>
__host__ __device__ constexpr std::uint64_t mask() { return W >= 64 ? ~0ull : ((1ull << W) - 1); }
} // namespace detail

template <std::uint64_t A, std::uint64_t B>
class PackedPair {
    static_assert(A + B <= 64, "fields wider than a word");
    using word = detail::word_t<A + B>;
    word w_;

    __host__ __device__ constexpr explicit PackedPair(word w, int) noexcept : w_(w) {}

  public:
    __host__ __device__ constexpr PackedPair() noexcept : w_(0) {}
    __host__ __device__ constexpr PackedPair(std::uint64_t a, std::uint64_t b) noexcept
        : w_(word((a & detail::mask<A>()) | ((b & detail::mask<B>()) << A)))
    {}
    __host__ __device__ constexpr std::uint64_t first() const noexcept { return w_ & detail::mask<A>(); }
    __host__ __device__ constexpr std::uint64_t second() const noexcept
    {
        return (std::uint64_t(w_) >> A) & detail::mask<B>();
    }
    __host__ __device__ void first(std::uint64_t a) noexcept
    {
        w_ = word((std::uint64_t(w_) & ~detail::mask<A>()) | (a & detail::mask<A>()));
    }
    __host__ __device__ void second(std::uint64_t b) noexcept
    {
        w_ = word((std::uint64_t(w_) & ~(detail::mask<B>() << A)) | ((b & detail::mask<B>()) << A));
    }
    __host__ __device__ constexpr bool operator==(const PackedPair &o) const noexcept { return w_ == o.w_; }
    __host__ __device__ constexpr bool operator!=(const PackedPair &o) const noexcept { return w_ != o.w_; }

    __device__ friend PackedPair atomicCAS(PackedPair *p, PackedPair cmp, PackedPair val) noexcept
    {
        return PackedPair(::atomicCAS(&p->w_, cmp.w_, val.w_), 0);
    }
    __device__ friend PackedPair atomicExch(PackedPair *p, PackedPair val) noexcept
    {
        return PackedPair(::atomicExch(&p->w_, val.w_), 0);
    }
};

template <std::uint64_t A, std::uint64_t B, std::uint64_t C, std::uint64_t D>
class PackedQuadruple {
    static_assert(A + B + C + D <= 64, "fields wider than a word");
    using word = detail::word_t<A + B + C + D>;
    word w_;

    __host__ __device__ constexpr explicit PackedQuadruple(word w, int) noexcept : w_(w) {}

    template <std::uint64_t Shift, std::uint64_t Width>
    __host__ __device__ constexpr std::uint64_t get() const noexcept
    {
        return (std::uint64_t(w_) >> Shift) & detail::mask<Width>();
    }
    template <std::uint64_t Shift, std::uint64_t Width>
    __host__ __device__ void set(std::uint64_t v) noexcept
    {
        w_ = word((std::uint64_t(w_) & ~(detail::mask<Width>() << Shift)) |
                  ((v & detail::mask<Width>()) << Shift));
    }

  public:
    __host__ __device__ constexpr PackedQuadruple() noexcept : w_(0) {}
    __host__ __device__ constexpr std::uint64_t first() const noexcept { return get<0, A>(); }
    __host__ __device__ constexpr std::uint64_t second() const noexcept { return get<A, B>(); }
    __host__ __device__ constexpr std::uint64_t third() const noexcept { return get<A + B, C>(); }
    __host__ __device__ constexpr std::uint64_t fourth() const noexcept { return get<A + B + C, D>(); }
    template <class T>
    __host__ __device__ constexpr T first_as() const noexcept { return T(first()); }
    template <class T>
    __host__ __device__ void first(T v) noexcept { set<0, A>(std::uint64_t(v)); }
    template <class T>
    __host__ __device__ void second(T v) noexcept { set<A, B>(std::uint64_t(v)); }
    template <class T>
    __host__ __device__ void third(T v) noexcept { set<A + B, C>(std::uint64_t(v)); }
    template <class T>
    __host__ __device__ void fourth(T v) noexcept { set<A + B + C, D>(std::uint64_t(v)); }
    __host__ __device__ constexpr bool operator==(const PackedQuadruple &o) const noexcept
    {
        return w_ == o.w_;
    }
    __host__ __device__ constexpr bool operator!=(const PackedQuadruple &o) const noexcept
    {
        return w_ != o.w_;
    }

    __device__ friend PackedQuadruple atomicCAS(PackedQuadruple *p, PackedQuadruple cmp,
                                                PackedQuadruple val) noexcept
    {
        return PackedQuadruple(::atomicCAS(&p->w_, cmp.w_, val.w_), 0);
    }
    __device__ friend PackedQuadruple atomicExch(PackedQuadruple *p, PackedQuadruple val) noexcept
    {
        return PackedQuadruple(::atomicExch(&p->w_, val.w_), 0);
    }
};

} // namespace packed_types
#endif
