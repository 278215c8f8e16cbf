/*
 * b200_core.cuh -- device-side core of the B200-native warpcore library.
 *
 * Shared by the bulk kernels compiled into libwarpcore_b200.so and by the
 * C++ drop-in headers' device-side per-key API, so that both agree on the
 * table layout and probe order.
 *
 * Layout in HBM
 *   The slot array is the reference's AoS store (storage.cuh:165-187,
 *   438-645): {Key key; Value value;} per slot, a bare Key for hash sets.
 *   u32/u32 slots are one 64-bit word (key in the low half), u64/u64 slots
 *   one 16-byte word, so a slot is claimed with ONE compare-and-swap that
 *   publishes key and value together (64-bit atomicCAS, 128-bit atom.cas).
 *
 * Probing
 *   The reference probes cg_size consecutive, unaligned slots per step
 *   (probing_schemes.cuh:79-100).  Here the table is split into buckets of
 *   cg_size slots that start on a bucket boundary, so a probe window is one
 *   aligned, sector-multiple block read with 16-byte vector loads.  The
 *   number of buckets is capacity / cg_size, which under the reference's
 *   capacity rule (base.cuh:27-34) is a prime, and the probing schemes are
 *   restated over buckets:
 *     double hashing  b0 = h1(key+seed) % nb,
 *                     step = h2(key+seed+1) % (nb-1) + 1, b = (b+step) % nb
 *     linear          b = (b+1) % nb
 *     quadratic       b = (b+1) % nb, (b+2) % nb, ... (step grows by one)
 *   With nb prime, double hashing and linear probing visit every bucket in
 *   nb windows (cycle-free like the reference's), so probing stops after at
 *   most nb windows and reports probing_length_exceeded instead of spinning.
 *   Slot placement therefore differs from the reference; results (values,
 *   flags, counts, statuses, table contents as a multiset) do not.
 */
#ifndef WARPCORE_B200_CORE_CUH
#define WARPCORE_B200_CORE_CUH

#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

namespace warpcore {
namespace b200 {

/* Status bits (status.cuh:44-68) */
enum : uint32_t {
    kStNone = 0u,
    kStUnknownError = 1u << 0,
    kStProbingLengthExceeded = 1u << 1,
    kStInvalidConfiguration = 1u << 2,
    kStInvalidKey = 1u << 3,
    kStDuplicateKey = 1u << 4,
    kStKeyNotFound = 1u << 5,
    kStIndexOverflow = 1u << 6,
    kStOutOfMemory = 1u << 7,
    kStNotInitialized = 1u << 8,
    kStDryRun = 1u << 9,
    kStInvalidPhaseOverlap = 1u << 10,
    kStMaxValuesReached = 1u << 11,
};

enum : uint32_t {
    kHashMurmur = 0,
    kHashNvidia = 1,
    kHashMueller = 2,
    kHashIdentity32 = 3,
    kHashIdentity64 = 4,
};

enum : uint32_t { kProbeDouble = 0, kProbeLinear = 1, kProbeQuadratic = 2 };

enum : int { kHandlerNothing = 0, kHandlerStatus = 1, kHandlerBoolean = 2 };

/* ------------------------------------------------------------------ */
/* hashers (hashers.cuh:34-44, 70-77, 116-139, 147-175)                */
/* ------------------------------------------------------------------ */

__host__ __device__ __forceinline__ uint32_t fmix32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

__host__ __device__ __forceinline__ uint64_t fmix64(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

__host__ __device__ __forceinline__ uint32_t nvidia_hash32(uint32_t x)
{
    x = (x + 0x7ed55d16u) + (x << 12);
    x = (x ^ 0xc761c23cu) ^ (x >> 19);
    x = (x + 0x165667b1u) + (x << 5);
    x = (x + 0xd3a2646cu) ^ (x << 9);
    x = (x + 0xfd7046c5u) + (x << 3);
    x = (x ^ 0xb55a4f09u) ^ (x >> 16);
    return x;
}

__host__ __device__ __forceinline__ uint32_t mueller_hash32(uint32_t x)
{
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = ((x >> 16) ^ x);
    return x;
}

template <class K>
__host__ __device__ __forceinline__ uint64_t hash_key(uint32_t hasher, K x)
{
    switch (hasher) {
    case kHashMurmur:
        return sizeof(K) == 4 ? uint64_t(fmix32(uint32_t(x)))
                              : fmix64(uint64_t(x));
    case kHashNvidia: return nvidia_hash32(uint32_t(x));
    case kHashMueller: return mueller_hash32(uint32_t(x));
    case kHashIdentity32: return uint32_t(x);
    default: return uint64_t(x);
    }
}

/* x % m, with the cheaper 32-bit path when both fit */
__host__ __device__ __forceinline__ uint64_t mod_u64(uint64_t x, uint64_t m)
{
    if (((x | m) >> 32) == 0) return uint32_t(x) % uint32_t(m);
    return x % m;
}

/* x % d by Barrett reduction with m = floor((2^64 - 1) / d): the estimate
 * q = mulhi(x, m) is floor(x / d) or one less for every 64-bit x, so one
 * conditional subtraction makes the remainder exact. */
__host__ __device__ __forceinline__ uint64_t barrett_magic(uint64_t d)
{
    return d ? ~0ull / d : 0;
}

__host__ __device__ __forceinline__ uint64_t mulhi64(uint64_t a, uint64_t b)
{
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return uint64_t((unsigned __int128)a * b >> 64);
#endif
}

__host__ __device__ __forceinline__ uint64_t fast_mod(uint64_t x, uint64_t d, uint64_t magic)
{
    uint64_t r = x - mulhi64(x, magic) * d;
    return r >= d ? r - d : r;
}

/* ------------------------------------------------------------------ */
/* table view and bucket probing                                        */
/* ------------------------------------------------------------------ */

/* A table's count of valid keys is kept in kLiveStripes counters,
 * kLiveStride words apart (one 32-byte sector each), so that writers spread
 * their atomics; size() is the sum of the stripes modulo 2^64.  Every claim
 * of an empty slot adds one, every erase that turns a key into a tombstone
 * subtracts one. */
constexpr int kLiveStripes = 32;
constexpr int kLiveStride = 4;

struct TableView {
    void *slots;
    uint32_t *status;
    unsigned char *fps;   /* one fingerprint byte per slot, or NULL */
    unsigned long long *live; /* kLiveStripes striped key counters, or NULL */
    uint64_t num_buckets; /* capacity / cg_size; prime under the capacity rule */
    uint64_t seed;
    uint64_t empty_key;
    uint64_t tombstone_key;
    uint64_t max_count;
    uint64_t magic_nb;   /* barrett_magic(num_buckets) */
    uint64_t magic_nb1;  /* barrett_magic(num_buckets - 1) */
    uint32_t probing, hasher1, hasher2, cg_size;
    void *values;        /* struct-of-arrays tables: the value array, one
                            value per slot index; NULL otherwise */
};

template <class K>
__host__ __device__ __forceinline__ uint64_t probe_begin(const TableView &t, K key)
{
    const K k = K(key + K(t.seed));
    return fast_mod(hash_key<K>(t.hasher1, k), t.num_buckets, t.magic_nb);
}

template <class K>
__host__ __device__ __forceinline__ uint64_t probe_step(const TableView &t, K key)
{
    if (t.probing != kProbeDouble || t.num_buckets < 2) return 1;
    const K k = K(key + K(t.seed) + K(1));
    return fast_mod(hash_key<K>(t.hasher2, k), t.num_buckets - 1, t.magic_nb1) + 1;
}

/* advance to the next bucket; `step` grows by one per window for
 * quadratic probing */
__host__ __device__ __forceinline__ uint64_t probe_next(const TableView &t,
                                                        uint64_t b,
                                                        uint64_t &step)
{
    uint64_t s = step;
    if (s >= t.num_buckets) s = fast_mod(s, t.num_buckets, t.magic_nb);
    b += s;
    if (b >= t.num_buckets) b -= t.num_buckets;
    if (t.probing == kProbeQuadratic) step++;
    return b;
}

/* ------------------------------------------------------------------ */
/* fingerprints                                                          */
/* ------------------------------------------------------------------ */

/* A table may keep one byte per slot beside the slot array: 0 for an empty
 * slot, 1 for a tombstone, 2..255 for a key (a multiplicative hash of the
 * key, independent of the probing hashers).  A bucket's fingerprints are
 * cg_size bytes, so probing can read them instead of the whole window and
 * read a slot only where the fingerprint matches.  Every write of a slot
 * key (claim, erase) writes its fingerprint after it, when the table has
 * them. */
enum : uint32_t { kFpEmpty = 0, kFpTomb = 1 };

template <class K>
__host__ __device__ __forceinline__ uint32_t fingerprint(K key)
{
    const uint64_t h = (uint64_t(key) * 0x9E3779B97F4A7C15ull) >> 56; /* 0..255 */
    return uint32_t((h * 254u) >> 8) + 2u;                             /* 2..255 */
}

__device__ __forceinline__ void fp_store(const TableView &t, uint64_t slot, uint32_t fp)
{
    if (t.fps) *reinterpret_cast<volatile unsigned char *>(t.fps + slot) = (unsigned char)fp;
}

/* windows the reference visits for a probing length: SDIV(pl, cg) windows
 * (probing_schemes.cuh:61, same unsigned wrap), at least one; capped at the
 * number of buckets */
__host__ __device__ __forceinline__ uint64_t max_windows(uint64_t probing_length,
                                                         uint64_t cg,
                                                         uint64_t num_buckets)
{
    uint64_t w = (probing_length + cg - 1) / cg;
    if (w == 0) w = 1;
    return w < num_buckets ? w : num_buckets;
}

/* ------------------------------------------------------------------ */
/* slot layouts                                                          */
/* ------------------------------------------------------------------ */

/* u32 key, u32 value: one 64-bit word, key in the low half */
struct LayoutKV32 {
    using key_t = uint32_t;
    using val_t = uint32_t;
    static constexpr int kSlotBytes = 8;
    static constexpr bool kHasValue = true;
};
/* u64 key, u64 value: one 16-byte word */
struct LayoutKV64 {
    using key_t = uint64_t;
    using val_t = uint64_t;
    static constexpr int kSlotBytes = 16;
    static constexpr bool kHasValue = true;
};
/* mixed widths, one 16-byte word each: the key in bytes 0..7 and the value
 * in bytes 8..15, the narrower field zero-extended (its upper half stays 0
 * in every state, so the 128-bit compare-and-swap sees whole words) */
struct LayoutK32V64 {
    using key_t = uint32_t;
    using val_t = uint64_t;
    static constexpr int kSlotBytes = 16;
    static constexpr bool kHasValue = true;
};
struct LayoutK64V32 {
    using key_t = uint64_t;
    using val_t = uint32_t;
    static constexpr int kSlotBytes = 16;
    static constexpr bool kHasValue = true;
};
/* hash set of u32 / u64 keys */
struct LayoutSet32 {
    using key_t = uint32_t;
    using val_t = uint32_t;
    static constexpr int kSlotBytes = 4;
    static constexpr bool kHasValue = false;
};
struct LayoutSet64 {
    using key_t = uint64_t;
    using val_t = uint64_t;
    static constexpr int kSlotBytes = 8;
    static constexpr bool kHasValue = false;
};
/* single-value table stored as a struct of arrays (SoAStore,
 * storage.cuh:218-432): the slot array holds the keys only and is probed
 * like a hash set's; the value of slot i is element i of a separate array
 * (TableView::values).  An insert writes the value after the key's
 * compare-and-swap, as the reference's SoA store does. */
template <class K, class V>
struct LayoutSoA {
    using key_t = K;
    using val_t = V;
    static constexpr int kSlotBytes = int(sizeof(K));
    static constexpr bool kHasValue = false; /* the slots carry no value */
    static constexpr bool kSoA = true;
};

template <class L, class = void>
struct is_soa : std::false_type {};
template <class L>
struct is_soa<L, std::void_t<decltype(L::kSoA)>> : std::integral_constant<bool, L::kSoA> {};

/* up to 16 bytes of a probe window held by one lane */
struct LaneWords {
    uint32_t w[4];
};

template <int kBytes>
__device__ __forceinline__ LaneWords load_lane(const void *p)
{
    LaneWords r;
    if constexpr (kBytes == 16) {
        const uint4 v = __ldcg(reinterpret_cast<const uint4 *>(p));
        r.w[0] = v.x; r.w[1] = v.y; r.w[2] = v.z; r.w[3] = v.w;
    } else if constexpr (kBytes == 8) {
        const uint2 v = __ldcg(reinterpret_cast<const uint2 *>(p));
        r.w[0] = v.x; r.w[1] = v.y; r.w[2] = 0; r.w[3] = 0;
    } else {
        r.w[0] = __ldcg(reinterpret_cast<const unsigned int *>(p));
        r.w[1] = 0; r.w[2] = 0; r.w[3] = 0;
    }
    return r;
}

template <class L>
__device__ __forceinline__ typename L::key_t slot_key(const LaneWords &lw, int s)
{
    if constexpr (L::kSlotBytes == 4) return lw.w[s];
    else if constexpr (L::kSlotBytes == 8 && !L::kHasValue)
        return uint64_t(lw.w[2 * s]) | (uint64_t(lw.w[2 * s + 1]) << 32);
    else if constexpr (L::kSlotBytes == 8) return lw.w[2 * s];
    else return uint64_t(lw.w[0]) | (uint64_t(lw.w[1]) << 32);
}

template <class L>
__device__ __forceinline__ typename L::val_t slot_val(const LaneWords &lw, int s)
{
    if constexpr (L::kSlotBytes == 8 && L::kHasValue) return lw.w[2 * s + 1];
    else if constexpr (L::kSlotBytes == 16)
        return uint64_t(lw.w[2]) | (uint64_t(lw.w[3]) << 32);
    else return 0;
}

/* 128-bit compare-and-swap (atom.cas.b128, sm_90 and newer) */
__device__ __forceinline__ void cas128(void *addr, uint64_t cmp_lo,
                                       uint64_t cmp_hi, uint64_t new_lo,
                                       uint64_t new_hi, uint64_t &old_lo,
                                       uint64_t &old_hi)
{
    asm volatile(
        "{\n\t"
        ".reg .b128 cmp, nv, old;\n\t"
        "mov.b128 cmp, {%2, %3};\n\t"
        "mov.b128 nv, {%4, %5};\n\t"
        "atom.global.cas.b128 old, [%6], cmp, nv;\n\t"
        "mov.b128 {%0, %1}, old;\n\t"
        "}"
        : "=l"(old_lo), "=l"(old_hi)
        : "l"(cmp_lo), "l"(cmp_hi), "l"(new_lo), "l"(new_hi), "l"(addr)
        : "memory");
}

/* Claim an empty slot for key with payload v (value or initial count).
 * Empty slots hold the empty key and a zero payload (the init kernels write
 * whole slots).  Returns true on success; otherwise old_key is the key now
 * in the slot. */
template <class L>
__device__ __forceinline__ bool claim_slot(void *sp, typename L::key_t empty,
                                           typename L::key_t key,
                                           typename L::val_t v,
                                           typename L::key_t &old_key)
{
    if constexpr (L::kSlotBytes == 4) {
        old_key = atomicCAS(reinterpret_cast<unsigned int *>(sp), empty, key);
        return old_key == empty;
    } else if constexpr (L::kSlotBytes == 8 && !L::kHasValue) {
        old_key = atomicCAS(reinterpret_cast<unsigned long long *>(sp),
                            (unsigned long long)empty, (unsigned long long)key);
        return old_key == empty;
    } else if constexpr (L::kSlotBytes == 8) {
        unsigned long long expect = (unsigned long long)empty;
        const unsigned long long nw =
            (unsigned long long)key | ((unsigned long long)v << 32);
        for (int tries = 0; tries < 4; ++tries) {
            const unsigned long long old =
                atomicCAS(reinterpret_cast<unsigned long long *>(sp), expect, nw);
            if (old == expect) return true;
            old_key = uint32_t(old);
            if (old_key != empty) return false;
            expect = old; /* empty key with a stale payload: retry on it */
        }
        return false;
    } else {
        uint64_t exp_lo = empty, exp_hi = 0;
        for (int tries = 0; tries < 4; ++tries) {
            uint64_t olo, ohi;
            cas128(sp, exp_lo, exp_hi, key, v, olo, ohi);
            if (olo == exp_lo && ohi == exp_hi) return true;
            old_key = olo;
            if (old_key != empty) return false;
            exp_hi = ohi;
        }
        return false;
    }
}

/* One compare-and-swap attempt on slot sp, expecting an empty slot with
 * payload `expect_payload` and installing key with payload v.  Returns the
 * key found in the slot before the attempt (the attempt succeeded iff that
 * key is `empty` and *old_payload == expect_payload). */
template <class L>
__device__ __forceinline__ typename L::key_t cas_slot(void *sp, typename L::key_t empty,
                                                      typename L::val_t expect_payload,
                                                      typename L::key_t key,
                                                      typename L::val_t v,
                                                      typename L::val_t *old_payload)
{
    if constexpr (L::kSlotBytes == 4) {
        *old_payload = expect_payload;
        return atomicCAS(reinterpret_cast<unsigned int *>(sp), empty, key);
    } else if constexpr (L::kSlotBytes == 8 && !L::kHasValue) {
        *old_payload = expect_payload;
        return atomicCAS(reinterpret_cast<unsigned long long *>(sp), (unsigned long long)empty,
                         (unsigned long long)key);
    } else if constexpr (L::kSlotBytes == 8) {
        const unsigned long long old = atomicCAS(
            reinterpret_cast<unsigned long long *>(sp),
            (unsigned long long)empty | ((unsigned long long)expect_payload << 32),
            (unsigned long long)key | ((unsigned long long)v << 32));
        *old_payload = uint32_t(old >> 32);
        return uint32_t(old);
    } else {
        uint64_t olo, ohi;
        cas128(sp, empty, expect_payload, key, v, olo, ohi);
        *old_payload = ohi;
        return olo;
    }
}

template <class L>
__device__ __forceinline__ typename L::val_t *slot_value_ptr(void *sp)
{
    if constexpr (L::kSlotBytes == 8 && L::kHasValue)
        return reinterpret_cast<uint32_t *>(sp) + 1;
    else
        return reinterpret_cast<typename L::val_t *>(reinterpret_cast<uint64_t *>(sp) + 1);
}

template <class L>
__device__ __forceinline__ void store_value(void *sp, typename L::val_t v)
{
    if constexpr (L::kHasValue) {
        volatile typename L::val_t *p = slot_value_ptr<L>(sp);
        *p = v;
    }
}

/* the value of slot index `slot` (address sp): in the slot, or in the
 * value array of a struct-of-arrays table */
template <class L>
__device__ __forceinline__ void put_value(const TableView &t, void *sp, uint64_t slot,
                                          typename L::val_t v)
{
    if constexpr (is_soa<L>::value) {
        volatile typename L::val_t *p = reinterpret_cast<typename L::val_t *>(t.values) + slot;
        *p = v;
    } else {
        store_value<L>(sp, v);
    }
}

template <class L>
__device__ __forceinline__ typename L::val_t get_soa_value(const TableView &t, uint64_t slot)
{
    using V = typename L::val_t;
    if constexpr (sizeof(V) == 8)
        return V(__ldcg(reinterpret_cast<const unsigned long long *>(t.values) + slot));
    else
        return V(__ldcg(reinterpret_cast<const unsigned int *>(t.values) + slot));
}

template <class L>
__device__ __forceinline__ void store_key(void *sp, typename L::key_t k)
{
    volatile typename L::key_t *p = reinterpret_cast<typename L::key_t *>(sp);
    *p = k;
}

/* add d to the table's count of valid keys (one stripe, chosen by block and
 * warp) */
__device__ __forceinline__ void live_add(const TableView &t, long long d)
{
    if (t.live && d) {
        const unsigned stripe = (blockIdx.x + (threadIdx.x >> 5)) & (kLiveStripes - 1);
        atomicAdd(t.live + kLiveStride * stripe, (unsigned long long)d);
    }
}

/* Turn the slot holding `key` into a tombstone with a compare-and-swap of
 * the whole slot (the width of the claims' compare-and-swap), keeping its
 * payload.  `seen` is the slot as this thread last read it from L2: the
 * first expected value of the compare-and-swap of a slot with a payload (a
 * key-only slot needs none).  Returns true if this call erased the key;
 * false if the slot no longer holds it (an equal key erased by another
 * thread). */
template <class L>
__device__ __forceinline__ bool erase_slot_seen(void *sp, typename L::key_t key,
                                                typename L::key_t tomb, const LaneWords &seen)
{
    if constexpr (L::kSlotBytes == 4) {
        return atomicCAS(reinterpret_cast<unsigned int *>(sp), key, tomb) == key;
    } else if constexpr (L::kSlotBytes == 8 && !L::kHasValue) {
        return atomicCAS(reinterpret_cast<unsigned long long *>(sp), (unsigned long long)key,
                         (unsigned long long)tomb) == (unsigned long long)key;
    } else if constexpr (L::kSlotBytes == 8) {
        unsigned long long *p = reinterpret_cast<unsigned long long *>(sp);
        unsigned long long cur = uint64_t(seen.w[0]) | (uint64_t(seen.w[1]) << 32);
        /* a retry only follows a concurrent value update of the same key */
        for (int tries = 0; tries < 1024; ++tries) {
            if (uint32_t(cur) != uint32_t(key)) return false;
            const unsigned long long old =
                atomicCAS(p, cur, (cur & 0xffffffff00000000ull) | uint32_t(tomb));
            if (old == cur) return true;
            cur = old;
        }
        store_key<L>(sp, tomb);
        return true;
    } else {
        uint64_t lo = uint64_t(seen.w[0]) | (uint64_t(seen.w[1]) << 32);
        uint64_t hi = uint64_t(seen.w[2]) | (uint64_t(seen.w[3]) << 32);
        for (int tries = 0; tries < 1024; ++tries) {
            if (lo != uint64_t(key)) return false;
            uint64_t olo, ohi;
            cas128(sp, lo, hi, uint64_t(tomb), hi, olo, ohi);
            if (olo == lo && ohi == hi) return true;
            lo = olo;
            hi = ohi;
        }
        store_key<L>(sp, tomb);
        return true;
    }
}

/* the same, reading the slot first (from L2) where it has a payload */
template <class L>
__device__ __forceinline__ bool erase_slot(void *sp, typename L::key_t key,
                                           typename L::key_t tomb)
{
    if constexpr (L::kSlotBytes == 4 || !L::kHasValue)
        return erase_slot_seen<L>(sp, key, tomb, LaneWords{{0u, 0u, 0u, 0u}});
    else
        return erase_slot_seen<L>(sp, key, tomb, load_lane<L::kSlotBytes>(sp));
}

/* width-generic wrappers: uint64_t is unsigned long on LP64, while the CUDA
 * intrinsics are declared for unsigned long long */
template <class T>
__device__ __forceinline__ T atomic_add_any(T *p, T v)
{
    if constexpr (sizeof(T) == 8)
        return T(atomicAdd(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v));
    else
        return T(atomicAdd(reinterpret_cast<unsigned int *>(p), (unsigned int)v));
}

template <class T>
__device__ __forceinline__ T atomic_exch_any(T *p, T v)
{
    if constexpr (sizeof(T) == 8)
        return T(atomicExch(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v));
    else
        return T(atomicExch(reinterpret_cast<unsigned int *>(p), (unsigned int)v));
}

template <class T>
__device__ __forceinline__ T ld_stream(const T *p)
{
    if constexpr (sizeof(T) == 8)
        return T(__ldcs(reinterpret_cast<const unsigned long long *>(p)));
    else if constexpr (sizeof(T) == 4)
        return T(__ldcs(reinterpret_cast<const unsigned int *>(p)));
    else
        return *p;
}

template <class T>
__device__ __forceinline__ void st_stream(T *p, T v)
{
    if constexpr (sizeof(T) == 8)
        __stcs(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v);
    else if constexpr (sizeof(T) == 4)
        __stcs(reinterpret_cast<unsigned int *>(p), (unsigned int)v);
    else
        *p = v;
}

/* counting increment with the reference's wrap guard
 * (counting_hash_table.cuh:152-169), c occurrences at once */
template <class L>
__device__ __forceinline__ void count_add(void *sp, uint32_t c, uint64_t max_count,
                                          uint32_t &st, uint32_t &join)
{
    using V = typename L::val_t;
    V *vp = slot_value_ptr<L>(sp);
    const V old = atomic_add_any(vp, V(c));
    if (V(old + V(c)) < old) {
        st |= kStIndexOverflow;
        join |= kStIndexOverflow;
        atomic_exch_any(vp, V(max_count));
    }
}

/* A window's hit / free masks are slot-major inside a lane group: lane qq
 * of the group holds slots qq * SPL .. qq * SPL + SPL - 1, and the ballot of
 * its slot s lands at bits s * TPK .. s * TPK + TPK - 1, so building a mask
 * is one shift per slot.  slot_of_bit maps a bit back to the slot index it
 * stands for (a key has at most one hit, so any bit order finds it).
 * Claims are different: every insert path (window and fingerprint kernels,
 * the count cache's flush, the device per-key API) must try a window's free
 * slots in the same order, lowest slot first, or two paths inserting one key
 * at the same time could each claim a different slot for it.  A free mask
 * is read lowest slot first (lowest_slot_bit). */
template <int TPK, int SPL>
__device__ __forceinline__ uint32_t window_bits(uint32_t group_bits, int s)
{
    return SPL == 1 ? group_bits : group_bits << (s * TPK);
}

template <int TPK, int SPL>
__device__ __forceinline__ int slot_of_bit(int p)
{
    return SPL == 1 ? p : (p % TPK) * SPL + p / TPK;
}

/* the bit, in a non-empty slot-major mask, of its lowest slot: the lowest
 * lane that has any bit set, then that lane's first slot */
template <int TPK, int SPL>
__device__ __forceinline__ int lowest_slot_bit(uint32_t m)
{
    if constexpr (SPL == 1) {
        return __ffs(m) - 1;
    } else {
        constexpr uint32_t kLane = TPK == 32 ? 0xffffffffu : ((1u << TPK) - 1u);
        uint32_t lanes = 0;
#pragma unroll
        for (int s = 0; s < SPL; ++s) lanes |= (m >> (s * TPK)) & kLane;
        const int qq = __ffs(lanes) - 1;
        int p = qq;
#pragma unroll
        for (int s = SPL - 1; s >= 0; --s)
            if ((m >> (s * TPK + qq)) & 1u) p = s * TPK + qq;
        return p;
    }
}

__device__ __forceinline__ int nth_set_bit(uint32_t mask, int n)
{
    return int(__fns(mask, 0, n + 1));
}

__device__ __forceinline__ void join_status(uint32_t *status, uint32_t bits)
{
    /* Status::atomic_join (status.cuh:187-193) */
    if (bits) {
        const uint32_t cur = *reinterpret_cast<volatile uint32_t *>(status);
        if ((cur & bits) != bits) atomicOr(status, bits);
    }
}

} // namespace b200
} // namespace warpcore

#endif /* WARPCORE_B200_CORE_CUH */
