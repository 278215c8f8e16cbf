/*
 * wc_fp_kernels.cuh -- fingerprint-first bulk kernel for tables that keep
 * one fingerprint byte per slot (b200_core.cuh, "fingerprints").
 *
 * The bucket sequence, the slot order of claims and every per-key status
 * are those of table_op_kernel (wc_kernels.cuh); only what is read per
 * bucket differs.  table_op_kernel reads each bucket's whole window of
 * slots (128 B for u64 pairs at CG 8).  This kernel reads the bucket's
 * cg_size fingerprint bytes and then only the slots whose fingerprint
 * equals the key's:
 *   - a miss at load 0.9 costs ~2.9 fingerprint words instead of ~2.9
 *     windows, and the fingerprint array (1 byte per slot, 1/16 of a u64
 *     pair table) mostly stays in L2;
 *   - a hit costs the fingerprint words plus one slot, read with an
 *     evict-first hint so that slot lines do not push fingerprints out
 *     (retrieve), or from L2 without an L1 copy (inserts: a claim's
 *     compare-and-swap lands in L2, and an equal key's lane must see it;
 *     erase: its compare-and-swap on the slot follows, with the words read
 *     as the expected value).
 *
 * Each lane owns one key and issues one memory operation per wave: a
 * fingerprint load, a candidate slot load, or a compare-and-swap claim.
 * The 32 lanes' operations are independent, so a warp keeps 32 requests in
 * flight.  Keys are refilled in input order from a double-buffered
 * prefetch, duplicates in one refill are merged with __match_any_sync, and
 * counting inserts go through the per-block count cache, as in
 * table_op_kernel.
 */
#ifndef WC_FP_KERNELS_CUH
#define WC_FP_KERNELS_CUH

#include "wc_kernels.cuh"

namespace warpcore {
namespace b200 {

/* resident 256-thread blocks per SM the fingerprint kernels are compiled
 * for: inserts (which hold a key, a value and a claim in flight) and the
 * read-only retrieve / erase, which gain from more warps in flight */
#ifndef WC_FP_MIN_BLOCKS
#define WC_FP_MIN_BLOCKS 4
#endif
#ifndef WC_FP_MIN_BLOCKS_READ
#define WC_FP_MIN_BLOCKS_READ 6
#endif

/* L2 eviction priorities: fingerprint lines are loaded and stored with
 * evict_last and slot lines read by retrieve with evict_first (ld.cs),
 * so that the
 * random slot traffic of a table larger than L2 evicts slot lines before
 * fingerprint lines (a fingerprint byte written into an evicted sector
 * costs a DRAM read to merge). */
#ifndef WC_FP_L2_HINTS
#define WC_FP_L2_HINTS 1
#endif

__device__ __forceinline__ uint64_t l2_policy_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint32_t ld_hint_u32(const void *p, uint64_t pol)
{
    uint32_t v;
    asm volatile("ld.global.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ uint2 ld_hint_v2(const void *p, uint64_t pol)
{
    uint2 v;
    asm volatile("ld.global.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
                 : "=r"(v.x), "=r"(v.y) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ uint4 ld_hint_v4(const void *p, uint64_t pol)
{
    uint4 v;
    asm volatile("ld.global.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ uint32_t ld_hint_u16(const void *p, uint64_t pol)
{
    uint16_t v;
    asm volatile("ld.global.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ uint32_t ld_hint_u8(const void *p, uint64_t pol)
{
    uint16_t v;
    asm volatile("ld.global.L2::cache_hint.u8 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ void st_hint_u8(void *p, uint32_t v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.u8 [%0], %1, %2;" ::"l"(p), "h"(uint16_t(v)), "l"(pol)
                 : "memory");
}

/* 4 bytes of 0x00 / 0xff (a __vcmpeq4 result) to 4 bits, byte k -> bit k:
 * the multiplier moves bit 7 + 8k to bit 28 + k with no two terms meeting */
__device__ __forceinline__ uint32_t pack_bytes4(uint32_t v)
{
    return ((v & 0x80808080u) * 0x00204081u) >> 28;
}

/* load the W fingerprint bytes of a bucket; bit s of `match` / `empty`
 * says whether slot s holds fingerprint fp / is empty */
template <int W>
__device__ __forceinline__ void fp_masks(const unsigned char *p, uint32_t fp, uint32_t &match,
                                         uint32_t &empty, uint64_t pol)
{
    const uint32_t pat = fp * 0x01010101u;
    if constexpr (W >= 4) {
        constexpr int NW = W / 4;
        uint32_t w[NW];
        if constexpr (W == 4) {
            w[0] = WC_FP_L2_HINTS ? ld_hint_u32(p, pol)
                                  : __ldcg(reinterpret_cast<const unsigned int *>(p));
        } else if constexpr (W == 8) {
            const uint2 v = WC_FP_L2_HINTS ? ld_hint_v2(p, pol)
                                           : __ldcg(reinterpret_cast<const uint2 *>(p));
            w[0] = v.x;
            w[1] = v.y;
        } else {
#pragma unroll
            for (int h = 0; h < W / 16; ++h) {
                const uint4 v = WC_FP_L2_HINTS ? ld_hint_v4(p + 16 * h, pol)
                                               : __ldcg(reinterpret_cast<const uint4 *>(p) + h);
                w[4 * h + 0] = v.x;
                w[4 * h + 1] = v.y;
                w[4 * h + 2] = v.z;
                w[4 * h + 3] = v.w;
            }
        }
        match = 0;
        empty = 0;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            match |= pack_bytes4(__vcmpeq4(w[k], pat)) << (4 * k);
            empty |= pack_bytes4(__vcmpeq4(w[k], 0u)) << (4 * k);
        }
    } else {
        const uint32_t x =
            WC_FP_L2_HINTS ? (W == 2 ? ld_hint_u16(p, pol) : ld_hint_u8(p, pol))
                           : (W == 2 ? uint32_t(__ldcg(reinterpret_cast<const unsigned short *>(p)))
                                     : uint32_t(__ldcg(p)));
        constexpr uint32_t lim = (1u << W) - 1u; /* the zero bytes above W are not slots */
        match = pack_bytes4(__vcmpeq4(x, pat)) & lim;
        empty = pack_bytes4(__vcmpeq4(x, 0u)) & lim;
    }
}

/* one slot, read once: evict-first, so that the fingerprints stay in L2 */
template <class L>
__device__ __forceinline__ LaneWords load_slot_once(const unsigned char *sp)
{
    LaneWords r{{0u, 0u, 0u, 0u}};
    if constexpr (L::kSlotBytes == 16) {
        const uint4 v = __ldcs(reinterpret_cast<const uint4 *>(sp));
        r.w[0] = v.x; r.w[1] = v.y; r.w[2] = v.z; r.w[3] = v.w;
    } else if constexpr (L::kSlotBytes == 8) {
        const uint2 v = __ldcs(reinterpret_cast<const uint2 *>(sp));
        r.w[0] = v.x; r.w[1] = v.y;
    } else {
        r.w[0] = __ldcs(reinterpret_cast<const unsigned int *>(sp));
    }
    return r;
}

template <class L, int W, int OP>
__global__ void __launch_bounds__(256, (OP == kOpRetrieve || OP == kOpErase) ? WC_FP_MIN_BLOCKS_READ
                                                                            : WC_FP_MIN_BLOCKS)
    fp_op_kernel(const TableOpArgs a)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    constexpr int SB = L::kSlotBytes;
    constexpr bool kValueIn = OP == kOpInsert && L::kHasValue;
    enum : int { kPhaseFps = 0, kPhaseCheck = 1, kPhaseClaim = 2, kPhasePreload = 3 };
    const bool preload = (a.flags & kFlagPreloadClaim) != 0;
    const uint64_t pol_keep = l2_policy_evict_last(); /* fingerprint lines */

    const TableView &t = a.t;
    const int lane = threadIdx.x & 31;
    const unsigned lanemask_lt = (1u << lane) - 1u;
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;

    /* this warp's contiguous range of keys */
    uint64_t per = (a.n + nwarps - 1) / nwarps;
    per = (per + 31) & ~uint64_t(31);
    const uint64_t wb = warp * per < a.n ? warp * per : a.n;
    const uint64_t we = wb + per < a.n ? wb + per : a.n;

    const K empty = K(t.empty_key);
    const K tomb = K(t.tombstone_key);
    unsigned char *const slots = reinterpret_cast<unsigned char *>(t.slots);
    const K *const keys = reinterpret_cast<const K *>(a.keys);
    const V *const vals_in = reinterpret_cast<const V *>(a.values);

    uint64_t pf_base = wb;
    K pfA = (wb + lane < we) ? ld_stream(keys + wb + lane) : empty;
    K pfB = (wb + 32 + lane < we) ? ld_stream(keys + wb + 32 + lane) : empty;
    V pvA = 0, pvB = 0;
    if constexpr (kValueIn) {
        if (wb + lane < we) pvA = ld_stream(vals_in + wb + lane);
        if (wb + 32 + lane < we) pvB = ld_stream(vals_in + wb + 32 + lane);
    }
    uint64_t cursor = wb;

    bool has = false, pending = false, flag = false;
    int phase = kPhaseFps;
    uint32_t cand = 0, emp = 0, fp = 0;
    V claim_expect = 0;
    uint64_t i = 0, bucket = 0, step = 0, wins = 0;
    K key = empty;
    V val = 0;
    uint32_t st = kStNone, join = 0, cnt_add = 1;
    int live_delta = 0; /* claims minus erases of this lane */

    constexpr int kCache = OP == kOpCount ? (1 << count_cache_bits<L>()) : 1;
    __shared__ K sc_key[kCache];
    __shared__ V sc_cnt[kCache];
    const bool use_cache = OP == kOpCount && a.handler == kHandlerNothing;
    if (use_cache) {
        for (int c = threadIdx.x; c < kCache; c += blockDim.x) {
            sc_key[c] = empty;
            sc_cnt[c] = 0;
        }
        __syncthreads();
    }

    for (;;) {
        /* ---- refill lanes whose key is done, in input order ---- */
        const unsigned need = __ballot_sync(kFull, !has);
        const uint64_t avail = we - cursor;
        const int take = int(uint64_t(__popc(need)) < avail ? uint64_t(__popc(need)) : avail);
        if (take == 0 && need == kFull) break;
        const int r = __popc(need & lanemask_lt);
        const bool refill = !has && r < take;
        const int off = int(cursor - pf_base) + r;
        const K ka = shfl_any(pfA, off & 31);
        const K kb = shfl_any(pfB, off & 31);
        V va = 0, vb = 0;
        if constexpr (kValueIn) {
            va = shfl_any(pvA, off & 31);
            vb = shfl_any(pvB, off & 31);
        }
        if (refill) {
            key = off < 32 ? ka : kb;
            if constexpr (kValueIn) val = off < 32 ? va : vb;
            i = cursor + r;
            has = true;
            pending = true;
            flag = false;
            st = kStNone;
            cnt_add = 1;
            wins = 0;
            step = 0;
            phase = kPhaseFps;
            cand = 0;
            emp = 0;
            claim_expect = 0;
            if (key == empty || key == tomb) {
                st = kStInvalidKey;
                join |= kStInvalidKey;
                pending = false;
            }
        }
        cursor += uint64_t(take);
        if (cursor - pf_base >= 32) {
            pf_base += 32;
            pfA = pfB;
            pvA = pvB;
            const uint64_t nx = pf_base + 32 + lane;
            pfB = nx < we ? ld_stream(keys + nx) : empty;
            if constexpr (kValueIn) pvB = nx < we ? ld_stream(vals_in + nx) : V(0);
        }

        if constexpr (OP == kOpInsert || OP == kOpCount) {
            const bool fresh = refill && pending;
            const unsigned fmask = __ballot_sync(kFull, fresh);
            const unsigned peers = __match_any_sync(kFull, fresh ? key : empty) & fmask;
            int last = lane;
            if (fresh) {
                const int leader = __ffs(peers) - 1;
                last = 31 - __clz(peers);
                cnt_add = __popc(peers);
                if (lane != leader) {
                    st = kStDuplicateKey;
                    join |= kStDuplicateKey;
                    pending = false;
                }
            }
            if constexpr (kValueIn) {
                const V lv = shfl_any(val, last);
                if (fresh) val = lv;
            }
        }
        if constexpr (OP == kOpCount) {
            if (use_cache && refill && pending) {
                using CW = typename std::conditional<sizeof(K) == 8, unsigned long long,
                                                     unsigned int>::type;
                const uint32_t h = uint32_t((uint64_t(key) * 0x9E3779B97F4A7C15ull) >> (64 - count_cache_bits<L>()));
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    const int c = int((h + p) & (kCache - 1));
                    K cur = *reinterpret_cast<volatile K *>(&sc_key[c]);
                    bool first = false;
                    if (cur == empty) {
                        cur = K(atomicCAS(reinterpret_cast<CW *>(&sc_key[c]), CW(empty), CW(key)));
                        first = cur == empty;
                        if (first) cur = key;
                    }
                    if (cur == key) {
                        atomic_add_any(&sc_cnt[c], V(cnt_add));
                        if (!first) join |= kStDuplicateKey;
                        st = kStNone;
                        pending = false;
                        break;
                    }
                }
            }
        }
        if (refill && pending) {
            bucket = probe_begin<K>(t, key);
            fp = fingerprint(key);
        }

        /* ---- one memory operation per pending lane ---- */
        if (pending) {
            const uint64_t base_slot = bucket * uint64_t(W);
            bool advance = false;
            if (phase == kPhaseFps) {
                uint32_t m = 0, e = 0;
                fp_masks<W>(t.fps + base_slot, fp, m, e, pol_keep);
                cand = m;
                emp = e;
            } else if (phase == kPhaseCheck) {
                const int s = __ffs(cand) - 1;
                unsigned char *const sp = slots + (base_slot + uint64_t(s)) * SB;
                /* inserts read the slot where the claims' atomics land (L2):
                 * an L1 copy may predate the claim of an equal key by
                 * another lane, which would then be inserted twice.  Erase
                 * reads it the same way, since its compare-and-swap follows
                 * on the same line: with the evict-first read and a second
                 * read before the compare-and-swap, erasing 2^27 keys of a
                 * 2.4 GB table ran at 7.0 G keys/s, against 9.2 now */
                const LaneWords sw = (OP != kOpRetrieve) ? load_lane<SB>(sp)
                                                         : load_slot_once<L>(sp);
                const K sk = slot_key<L>(sw, 0);
                if (sk == key) {
                    if constexpr (OP == kOpRetrieve) {
                        st = kStNone;
                        flag = true;
                        if constexpr (L::kHasValue) {
                            if (!a.is_set) {
                                V v = slot_val<L>(sw, 0);
                                if (uint64_t(v) > t.max_count) v = V(t.max_count);
                                st_stream(reinterpret_cast<V *>(a.out) + i, v);
                            }
                        }
                    } else if constexpr (OP == kOpInsert) {
                        st = kStDuplicateKey;
                        join |= kStDuplicateKey;
                        store_value<L>(sp, val);
                    } else if constexpr (OP == kOpCount) {
                        st = kStDuplicateKey;
                        join |= kStDuplicateKey;
                        count_add<L>(sp, cnt_add, t.max_count, st, join);
                    } else {
                        if (erase_slot_seen<L>(sp, key, tomb, sw)) {
                            fp_store(t, base_slot + uint64_t(s), kFpTomb);
                            --live_delta;
                        }
                        st = kStNone;
                    }
                    pending = false;
                } else {
                    /* a set fingerprint over a key that reads empty is
                     * left to the compare-and-swap, which sees the key */
                    if ((OP == kOpInsert || OP == kOpCount) && sk == empty) emp |= 1u << s;
                    cand &= cand - 1u;
                }
            } else if (phase == kPhasePreload) {
                /* bring the claim's slot line into L2 with a plain load; a
                 * slot that is no longer empty is skipped (its key is
                 * another one: equal keys show up as fingerprint matches,
                 * or as the CAS's old key) */
                if constexpr (OP == kOpInsert || OP == kOpCount) {
                    int s = __ffs(emp) - 1;
                    const LaneWords sw = load_lane<SB>(slots + (base_slot + uint64_t(s)) * SB);
                    const K sk = slot_key<L>(sw, 0);
                    if (sk == key) {
                        st = kStDuplicateKey;
                        join |= kStDuplicateKey;
                        unsigned char *const sp = slots + (base_slot + uint64_t(s)) * SB;
                        if constexpr (OP == kOpInsert) store_value<L>(sp, val);
                        else count_add<L>(sp, cnt_add, t.max_count, st, join);
                        pending = false;
                    } else if (sk != empty) {
                        emp &= emp - 1u;
                        if (!emp) advance = true;
                    } else {
                        phase = kPhaseClaim;
                        claim_expect = slot_val<L>(sw, 0);
                    }
                }
            } else {
                if constexpr (OP == kOpInsert || OP == kOpCount) {
                    const int s = __ffs(emp) - 1;
                    unsigned char *const sp = slots + (base_slot + uint64_t(s)) * SB;
                    const V payload = OP == kOpCount ? V(cnt_add) : val;
                    V old_payload = 0;
                    /* (atom.cas takes no L2 cache hint) */
                    const K old = cas_slot<L>(sp, empty, claim_expect, key, payload, &old_payload);
                    if (old == empty && old_payload == claim_expect) {
#if WC_FP_L2_HINTS
                        st_hint_u8(t.fps + base_slot + uint64_t(s), fp, pol_keep);
#else
                        fp_store(t, base_slot + uint64_t(s), fp);
#endif
                        ++live_delta;
                        st = kStNone;
                        pending = false;
                    } else if (old == key) {
                        st = kStDuplicateKey;
                        join |= kStDuplicateKey;
                        if constexpr (OP == kOpInsert) store_value<L>(sp, val);
                        else count_add<L>(sp, cnt_add, t.max_count, st, join);
                        pending = false;
                    } else if (old == empty) {
                        claim_expect = old_payload; /* free slot, stale payload: again */
                    } else {
                        emp &= emp - 1u;
                        if (!emp) advance = true;
                        else if (preload) phase = kPhasePreload;
                    }
                }
            }

            /* a bucket with no candidate left decides: absent if it had a
             * free slot (claim it for inserts), else the next bucket */
            if (pending && phase != kPhaseClaim && phase != kPhasePreload && !advance) {
                if (cand) {
                    phase = kPhaseCheck;
                } else if (emp) {
                    if constexpr (OP == kOpRetrieve) {
                        if (a.is_set) {
                            st = kStNone;
                            flag = false;
                        } else {
                            st = kStKeyNotFound;
                            join |= kStKeyNotFound;
                        }
                        pending = false;
                    } else if constexpr (OP == kOpErase) {
                        st = a.is_set ? kStNone : kStKeyNotFound;
                        pending = false;
                    } else {
                        phase = preload ? kPhasePreload : kPhaseClaim;
                        claim_expect = 0;
                    }
                } else {
                    advance = true;
                }
            }
            if (pending && advance) {
                phase = kPhaseFps;
                cand = 0;
                emp = 0;
                claim_expect = 0;
                if (++wins >= a.max_windows) {
                    pending = false;
                    if (OP == kOpErase) {
                        st = a.is_set ? kStNone : kStProbingLengthExceeded;
                    } else {
                        st = kStProbingLengthExceeded;
                        join |= kStProbingLengthExceeded;
                    }
                } else {
                    if (wins == 1) step = probe_step<K>(t, key);
                    bucket = probe_next(t, bucket, step);
                }
            }
        }

        /* ---- keys that finished this wave write their results ---- */
        if (has && !pending) {
            if constexpr (OP == kOpRetrieve) {
                if (a.is_set && st == kStNone)
                    reinterpret_cast<unsigned char *>(a.out)[i] = (unsigned char)flag;
            }
            if (a.status_out) {
                if (a.handler == kHandlerStatus)
                    st_stream(reinterpret_cast<uint32_t *>(a.status_out) + i, st);
                else if (a.handler == kHandlerBoolean)
                    reinterpret_cast<unsigned char *>(a.status_out)[i] =
                        (unsigned char)((st & a.bool_mask) != 0);
            }
            has = false;
        }
    }
    if constexpr (OP == kOpCount) {
        if (use_cache) {
            __syncthreads();
            for (int c = threadIdx.x; c < kCache; c += blockDim.x) {
                const K ck = sc_key[c];
                if (ck != empty)
                    count_one<L, W>(t, ck, uint32_t(sc_cnt[c]), a.max_windows, join, live_delta);
            }
        }
    }
    const uint32_t wjoin = __reduce_or_sync(kFull, join);
    const int wlive = int(__reduce_add_sync(kFull, unsigned(live_delta)));
    if (lane == 0) {
        join_status(t.status, wjoin);
        live_add(t, wlive);
    }
}

/* Recompute every fingerprint from the slot array in one streaming pass.
 * Lane l of a warp reads 16-byte vector v + l (coalesced) and writes the
 * fingerprints of its 1, 2 or 4 slots as one store, so a warp writes 32,
 * 64 or 128 consecutive bytes; four vectors per thread are in flight.  A
 * large insert runs the whole-window kernel without fingerprint writes and
 * then this pass: streaming the slot array costs less than one random byte
 * write per key once a batch covers more than about 1/8 of a table larger
 * than L2. */
template <class L>
__device__ __forceinline__ uint32_t fp_of_slot_key(typename L::key_t k, typename L::key_t e,
                                                   typename L::key_t tb)
{
    return k == e ? kFpEmpty : (k == tb ? kFpTomb : fingerprint(k));
}

template <class L>
__global__ void __launch_bounds__(256) fp_rebuild_kernel(const void *slots, uint64_t capacity,
                                                         uint64_t empty, uint64_t tomb,
                                                         unsigned char *fps)
{
    using K = typename L::key_t;
    constexpr int SB = L::kSlotBytes;
    constexpr int SPV = 16 / SB; /* slots per 16-byte vector: 1, 2 or 4 */
    constexpr int kUnroll = 4;
    const K e = K(empty), tb = K(tomb);
    const uint4 *const vec = reinterpret_cast<const uint4 *>(slots);
    const uint64_t nvec = capacity / SPV;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t v0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v0 < nvec;
         v0 += stride * kUnroll) {
        uint4 x[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t v = v0 + uint64_t(u) * stride;
            x[u] = v < nvec ? __ldcs(vec + v) : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t v = v0 + uint64_t(u) * stride;
            if (v >= nvec) break;
            const LaneWords lw{{x[u].x, x[u].y, x[u].z, x[u].w}};
            uint32_t f = 0;
#pragma unroll
            for (int s = 0; s < SPV; ++s) f |= fp_of_slot_key<L>(slot_key<L>(lw, s), e, tb) << (8 * s);
            if constexpr (SPV == 1) fps[v] = (unsigned char)f;
            else if constexpr (SPV == 2) reinterpret_cast<unsigned short *>(fps)[v] = (unsigned short)f;
            else reinterpret_cast<uint32_t *>(fps)[v] = f;
        }
    }
    /* ragged tail: capacity need not be a multiple of SPV */
    if (blockIdx.x == 0 && threadIdx.x < capacity % SPV) {
        const uint64_t si = nvec * SPV + threadIdx.x;
        const K k = *reinterpret_cast<const K *>(reinterpret_cast<const unsigned char *>(slots) + si * SB);
        fps[si] = (unsigned char)fp_of_slot_key<L>(k, e, tb);
    }
}

} // namespace b200
} // namespace warpcore

#endif /* WC_FP_KERNELS_CUH */
