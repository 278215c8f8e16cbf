/*
 * wc_kernels.cuh -- bulk kernels of the B200-native warpcore library.
 *
 * One kernel template serves insert / retrieve / erase of
 * SingleValueHashTable, HashSet and CountingHashTable (the reference's
 * kernels::insert / retrieve / erase, gpu_engine.cuh:177-262, 352-376, and
 * the per-key device methods they call).
 *
 * Warp-batched probing
 *   A warp takes 32 keys at a time; lane l OWNS key l (coalesced input and
 *   output, one status per lane).  The probe windows of the owned keys are
 *   fetched cooperatively: TPK lanes load one window with 16-byte vector
 *   loads (one request per window), and the windows of ALL pending keys of
 *   the warp are requested before any is inspected, so each warp keeps up to
 *   32 windows in flight.  Match and empty masks go back to the owner lane
 *   with ballots; the owner then issues its own compare-and-swap, so the
 *   claims of all 32 keys leave the SM in the same instruction.  Keys whose
 *   window had no match and no free slot advance to their next bucket and
 *   are fetched again in the next wave, packed densely onto the lanes.
 *   Before any atomic, equal keys inside a warp are merged with
 *   __match_any_sync: one leader inserts (with the count of its peers for
 *   counting, with the last peer's value for single-value tables) and the
 *   others report duplicate_key, as they would in the reference.
 */
#ifndef WC_KERNELS_CUH
#define WC_KERNELS_CUH

#include <warpcore/detail/b200_core.cuh>
#include "wc_compact.cuh"

namespace warpcore {
namespace b200 {

enum : int { kOpInsert = 0, kOpCount = 1, kOpRetrieve = 2, kOpErase = 3 };

struct TableOpArgs {
    TableView t;
    const void *keys;
    const void *values;   /* insert */
    void *out;            /* retrieve: values (tables) or uint8 flags (sets) */
    void *status_out;
    uint64_t n;
    uint64_t max_windows;
    uint32_t bool_mask;   /* ReturnBoolean: status & mask != 0 */
    int handler;
    int is_set;
    uint32_t flags;       /* kFlag* */
};

/* fingerprint kernel: before the compare-and-swap of a claim, read the
 * target slot with a plain load (into L2), then CAS on the resident line */
constexpr uint32_t kFlagPreloadClaim = 1u;

constexpr unsigned kFull = 0xffffffffu;

/* The per-block shared-memory count cache of counting inserts holds 32 KiB
 * of keys and counts: 4096 entries of u32 pairs, 2048 of wider ones.  A key
 * probes 4 entries from a multiplicative hash of count_cache_bits<L>()
 * bits.  On 2^28 Zipf(1.1) u32 keys over 2^24 (u32 counts) the insert ran
 * 34.9 / 36.3 / 37.6 G keys/s with 1024 / 2048 / 4096 entries; more does
 * not fit the 48 KiB of static shared memory. */
template <class L>
constexpr int count_cache_bits()
{
    return sizeof(typename L::key_t) + sizeof(typename L::val_t) <= 8 ? 12 : 11;
}

/* resident 256-thread blocks per SM the table kernels are compiled for:
 * 3 (at most 85 registers) keeps 24 warps x 32 probe windows in flight per
 * SM, measured 22%/19% faster (insert/retrieve, u64 keys at load 0.9) than
 * 2 blocks, and spill-free unlike 4 */
#ifndef WC_TABLE_MIN_BLOCKS
#define WC_TABLE_MIN_BLOCKS 3
#endif

template <class T>
__device__ __forceinline__ T shfl_any(T v, int src)
{
    if constexpr (sizeof(T) == 8) {
        const uint32_t lo = __shfl_sync(kFull, uint32_t(v), src);
        const uint32_t hi = __shfl_sync(kFull, uint32_t(uint64_t(v) >> 32), src);
        return T(uint64_t(lo) | (uint64_t(hi) << 32));
    } else {
        return T(__shfl_sync(kFull, uint32_t(v), src));
    }
}

/* one thread counts c occurrences of key into the table (claim an empty
 * slot in slot order or add to the key's slot), as the warp kernel does */
template <class L, int W>
__device__ void count_one(const TableView &t, typename L::key_t key, uint32_t c,
                          uint64_t max_windows, uint32_t &join, int &live_delta)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    constexpr int SB = L::kSlotBytes;
    const K empty = K(t.empty_key);
    unsigned char *const slots = reinterpret_cast<unsigned char *>(t.slots);
    uint64_t b = probe_begin<K>(t, key), step = 0, wins = 0;
    uint32_t st = kStNone;
    if (c > 1) join |= kStDuplicateKey;
    for (;;) {
        unsigned char *const bptr = slots + b * uint64_t(W) * SB;
        bool resolved = false;
        for (int s = 0; s < W && !resolved; ++s) {
            unsigned char *const sp = bptr + s * SB;
            const K sk = __ldcg(reinterpret_cast<const typename std::conditional<
                                    sizeof(K) == 8, unsigned long long, unsigned int>::type *>(sp));
            if (sk == key) {
                join |= kStDuplicateKey;
                count_add<L>(sp, c, t.max_count, st, join);
                resolved = true;
            } else if (sk == empty) {
                K old_key;
                if (claim_slot<L>(sp, empty, key, V(c), old_key)) {
                    fp_store(t, b * W + s, fingerprint(key));
                    ++live_delta;
                    resolved = true;
                } else if (old_key == key) {
                    join |= kStDuplicateKey;
                    count_add<L>(sp, c, t.max_count, st, join);
                    resolved = true;
                }
            }
        }
        if (resolved) return;
        if (++wins >= max_windows) {
            join |= kStProbingLengthExceeded;
            return;
        }
        if (wins == 1) step = probe_step<K>(t, key);
        b = probe_next(t, b, step);
    }
}

/* The warp-batched probing loop of table_op_kernel over the keys
 * [wb, we) of one warp: used by table_op_kernel for its warp's range and by
 * the persistent serving kernel for one chunk of a request.  sh_bucket,
 * sh_key and sh_off are this warp's 32-entry rows in shared memory; sc_key /
 * sc_cnt the block's count cache (counting inserts with use_cache).  Joins
 * the status bits of its keys into `join` and its claims minus erases into
 * `live_delta`. */
template <class L, int W, int OP>
__device__ __forceinline__ void group_range(const TableOpArgs &a, const uint64_t wb,
                                            const uint64_t we, uint64_t *sh_bucket,
                                            typename L::key_t *sh_key, uint32_t *sh_off,
                                            typename L::key_t *sc_key, typename L::val_t *sc_cnt,
                                            const bool use_cache, uint32_t &join,
                                            int &live_delta)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    constexpr int SB = L::kSlotBytes;
    constexpr int WB = W * SB;
    constexpr int LB = WB < 16 ? WB : 16; /* bytes per lane per window */
    constexpr int TPK = WB / LB;          /* lanes per window */
    constexpr int SPL = LB / SB;          /* slots per lane */
    constexpr int G = 32 / TPK;           /* windows per warp per round */
    constexpr uint32_t kGroupMask = TPK == 32 ? kFull : ((1u << TPK) - 1u);
    constexpr bool kSoA = is_soa<L>::value;
    constexpr bool kValueIn = OP == kOpInsert && (L::kHasValue || kSoA);
    constexpr int kCache = OP == kOpCount ? (1 << count_cache_bits<L>()) : 1;
    static_assert(TPK * LB == WB && SPL * SB == LB, "window split");

    const TableView &t = a.t;
    const int lane = threadIdx.x & 31;
    const int g = lane / TPK;
    const int q = lane % TPK;
    const unsigned lanemask_lt = (1u << lane) - 1u;

    const K empty = K(t.empty_key);
    const K tomb = K(t.tombstone_key);
    unsigned char *const slots = reinterpret_cast<unsigned char *>(t.slots);
    const K *const keys = reinterpret_cast<const K *>(a.keys);
    const V *const vals_in = reinterpret_cast<const V *>(a.values);

    /* two 32-key prefetch buffers: keys are read one buffer ahead of use */
    uint64_t pf_base = wb;
    K pfA = (wb + lane < we) ? ld_stream(keys + wb + lane) : empty;
    K pfB = (wb + 32 + lane < we) ? ld_stream(keys + wb + 32 + lane) : empty;
    V pvA = 0, pvB = 0;
    if constexpr (kValueIn) {
        if (wb + lane < we) pvA = ld_stream(vals_in + wb + lane);
        if (wb + 32 + lane < we) pvB = ld_stream(vals_in + wb + 32 + lane);
    }
    uint64_t cursor = wb;

    /* state of the key this lane owns; a pending key either waits for its
     * window (claiming == false) or for a compare-and-swap on the lowest
     * slot of claim_bits, the free slots its last window showed */
    bool has = false, pending = false, flag = false, claiming = false;
    uint32_t claim_bits = 0;
    V claim_expect = 0;
    uint64_t i = 0, bucket = 0, step = 0, wins = 0;
    K key = empty;
    V val = 0;
    uint32_t st = kStNone, cnt_add = 1;

    for (;;) {
        /* ---- refill lanes whose key is done, in input order ---- */
        const unsigned need = __ballot_sync(kFull, !has);
        const uint64_t avail = we - cursor;
        const int take = int(uint64_t(__popc(need)) < avail ? uint64_t(__popc(need)) : avail);
        if (take == 0 && need == kFull) break;
        const int r = __popc(need & lanemask_lt);
        const bool refill = !has && r < take;
        const int off = int(cursor - pf_base) + r; /* < 64 for refilling lanes */
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
            claiming = false;
            claim_bits = 0;
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
            /* merge equal keys among the newly taken ones before any atomic:
             * one leader claims, with the count of its peers (counting) or
             * the value of the last of them (single-value tables) */
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
                const uint32_t h = uint32_t((uint64_t(key) * 0x9E3779B97F4A7C15ull) >> (64 - count_cache_bits<L>()));
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    const int c = int((h + p) & (kCache - 1));
                    K cur = *reinterpret_cast<volatile K *>(&sc_key[c]);
                    bool first = false;
                    if (cur == empty) {
                        cur = K(atomicCAS(reinterpret_cast<typename std::conditional<sizeof(K) == 8,
                                          unsigned long long, unsigned int>::type *>(&sc_key[c]),
                                          (typename std::conditional<sizeof(K) == 8, unsigned long long,
                                                                     unsigned int>::type)empty,
                                          (typename std::conditional<sizeof(K) == 8, unsigned long long,
                                                                     unsigned int>::type)key));
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
        if (refill && pending) bucket = probe_begin<K>(t, key);

        /* ---- one probe wave: window loads for keys that need one, then the
         * compare-and-swaps of keys that are claiming a slot; both are in
         * flight together and only consumed afterwards ---- */
        const bool loading = pending && !claiming;
        const unsigned pmask = __ballot_sync(kFull, loading);
        bool did_cas = false;
        K cas_old = empty;
        V cas_old_payload = 0;
        if (__any_sync(kFull, pending)) {
            const int cnt = __popc(pmask);
            const int rounds = (cnt + G - 1) / G;
            const int my_rank = __popc(pmask & lanemask_lt);
            const int my_round = my_rank / G;
            const int my_g = my_rank % G;

            /* owners publish (bucket, key, index) in rank order; group g of
             * round rr then serves the owner of rank rr * G + g */
            __syncwarp();
            if (loading) {
                sh_bucket[my_rank] = bucket;
                sh_key[my_rank] = key;
                sh_off[my_rank] = uint32_t(i - wb);
            }
            __syncwarp();

            LaneWords win[TPK];
#pragma unroll
            for (int rr = 0; rr < TPK; ++rr) {
                if (rr < rounds) {
                    const int idx = rr * G + g;
                    if (idx < cnt) {
                        const uint64_t b = sh_bucket[idx];
                        win[rr] = load_lane<LB>(slots + (b * W + uint64_t(q) * SPL) * SB);
                    } else {
                        win[rr] = LaneWords{{0u, 0u, 0u, 0u}};
                    }
                }
            }

            if constexpr (OP == kOpInsert || OP == kOpCount) {
                if (pending && claiming) {
                    const int s = slot_of_bit<TPK, SPL>(lowest_slot_bit<TPK, SPL>(claim_bits));
                    unsigned char *const sp = slots + (bucket * W + uint64_t(s)) * SB;
                    const V payload = OP == kOpCount ? V(cnt_add) : val;
                    cas_old = cas_slot<L>(sp, empty, claim_expect, key, payload, &cas_old_payload);
                    did_cas = true;
                }
            }

            uint32_t hit_bits = 0, empty_bits = 0;
#pragma unroll
            for (int rr = 0; rr < TPK; ++rr) {
                if (rr < rounds) {
                    const int idx = rr * G + g;
                    const bool served = idx < cnt;
                    const K kr = served ? sh_key[idx] : empty;
#pragma unroll
                    for (int s = 0; s < SPL; ++s) {
                        const K sk = slot_key<L>(win[rr], s);
                        const bool h = served && sk == kr;
                        const unsigned hb = __ballot_sync(kFull, h);
                        const unsigned eb = __ballot_sync(kFull, served && sk == empty);
                        if (loading && my_round == rr) {
                            hit_bits |= window_bits<TPK, SPL>((hb >> (my_g * TPK)) & kGroupMask, s);
                            empty_bits |= window_bits<TPK, SPL>((eb >> (my_g * TPK)) & kGroupMask, s);
                        }
                        if constexpr (OP == kOpRetrieve && L::kHasValue) {
                            /* a key occupies at most one slot, so the lane
                             * that sees it writes the value itself */
                            if (h && !a.is_set) {
                                V v = slot_val<L>(win[rr], s);
                                if (uint64_t(v) > t.max_count) v = V(t.max_count);
                                st_stream(reinterpret_cast<V *>(a.out) + wb + sh_off[idx], v);
                            }
                        }
                    }
                }
            }

            bool advance = false;
            if (loading) {
                unsigned char *const bptr = slots + bucket * uint64_t(W) * SB;
                if (hit_bits) {
                    const int fh = slot_of_bit<TPK, SPL>(__ffs(hit_bits) - 1);
                    unsigned char *const sp = bptr + fh * SB;
                    if constexpr (OP == kOpRetrieve) {
                        st = kStNone;
                        flag = true;
                        if constexpr (kSoA)
                            st_stream(reinterpret_cast<V *>(a.out) + i,
                                      get_soa_value<L>(t, bucket * W + uint64_t(fh)));
                    } else if constexpr (OP == kOpInsert) {
                        st = kStDuplicateKey;
                        join |= kStDuplicateKey;
                        put_value<L>(t, sp, bucket * W + uint64_t(fh), val);
                    } else if constexpr (OP == kOpCount) {
                        st = kStDuplicateKey;
                        join |= kStDuplicateKey;
                        count_add<L>(sp, cnt_add, t.max_count, st, join);
                    } else {
                        if (erase_slot<L>(sp, key, tomb)) {
                            fp_store(t, bucket * W + uint64_t(fh), kFpTomb);
                            --live_delta;
                        }
                        st = kStNone;
                    }
                    pending = false;
                } else if (empty_bits) {
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
                        /* claim the free slots in slot order, from the next wave on */
                        claiming = true;
                        claim_bits = empty_bits;
                        claim_expect = 0;
                    }
                } else {
                    advance = true;
                }
            }
            if constexpr (OP == kOpInsert || OP == kOpCount) {
                if (did_cas) {
                    const int s = slot_of_bit<TPK, SPL>(lowest_slot_bit<TPK, SPL>(claim_bits));
                    unsigned char *const sp = slots + (bucket * W + uint64_t(s)) * SB;
                    if (cas_old == empty && cas_old_payload == claim_expect) {
                        fp_store(t, bucket * W + uint64_t(s), fingerprint(key));
                        if constexpr (kSoA) put_value<L>(t, sp, bucket * W + uint64_t(s), val);
                        ++live_delta;
                        st = kStNone;
                        pending = false;
                    } else if (cas_old == key) {
                        st = kStDuplicateKey;
                        join |= kStDuplicateKey;
                        if constexpr (OP == kOpInsert) put_value<L>(t, sp, bucket * W + uint64_t(s), val);
                        else count_add<L>(sp, cnt_add, t.max_count, st, join);
                        pending = false;
                    } else if (cas_old == empty) {
                        /* free slot with a stale payload: try again on it */
                        claim_expect = cas_old_payload;
                    } else {
                        claim_bits &= ~(1u << lowest_slot_bit<TPK, SPL>(claim_bits));
                        if (!claim_bits) {
                            claiming = false;
                            advance = true;
                        }
                    }
                }
            }
            if (pending && advance) {
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
}

template <class L, int W, int OP>
__global__ void __launch_bounds__(256, WC_TABLE_MIN_BLOCKS) table_op_kernel(const TableOpArgs a)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    const int wib = threadIdx.x >> 5;
    __shared__ uint64_t sh_bucket[8][32];
    __shared__ K sh_key[8][32];
    __shared__ uint32_t sh_off[8][32];

    /* this warp's contiguous range of keys */
    uint64_t per = (a.n + nwarps - 1) / nwarps;
    per = (per + 31) & ~uint64_t(31);
    const uint64_t wb = warp * per < a.n ? warp * per : a.n;
    const uint64_t we = wb + per < a.n ? wb + per : a.n;
    /* (a warp without keys runs the loop once and leaves it: every warp must
     * reach the block barriers of the counting cache below) */

    const K empty = K(a.t.empty_key);
    uint32_t join = 0;
    int live_delta = 0; /* claims minus erases of this warp's lanes */

    /* Counting inserts without per-key statuses go through a per-block
     * shared-memory count cache first: equal keys of the block add up there,
     * and each cached key reaches the table once, when the block flushes.
     * Skewed (Zipf) streams thus stop serialising atomics on hot slots. */
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

    group_range<L, W, OP>(a, wb, we, sh_bucket[wib], sh_key[wib], sh_off[wib], sc_key, sc_cnt,
                          use_cache, join, live_delta);

    if constexpr (OP == kOpCount) {
        if (use_cache) {
            /* flush: every cached key is counted into the table once */
            __syncthreads();
            for (int c = threadIdx.x; c < kCache; c += blockDim.x) {
                const K ck = sc_key[c];
                if (ck != empty)
                    count_one<L, W>(a.t, ck, uint32_t(sc_cnt[c]), a.max_windows, join, live_delta);
            }
        }
    }
    const uint32_t wjoin = __reduce_or_sync(kFull, join);
    const int wlive = int(__reduce_add_sync(kFull, unsigned(live_delta)));
    if (lane == 0) {
        join_status(a.t.status, wjoin);
        live_add(a.t, wlive);
    }
}

/* fill the slot array with empty slots (key = empty, payload = 0): the
 * reference's init_keys / init_values (storage.cuh:523-562) in one pass.
 * `pattern` is 16 bytes of slots; the array is 16-byte aligned. */
template <int kUnused = 0>
__global__ void __launch_bounds__(256) fill_kernel(uint32_t *p, uint64_t n_u32, uint4 pattern)
{
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t tid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    uint4 *p4 = reinterpret_cast<uint4 *>(p);
    const uint64_t n4 = n_u32 / 4;
    for (uint64_t i = tid; i < n4; i += stride) __stcg(p4 + i, pattern);
    const uint32_t pw[4] = {pattern.x, pattern.y, pattern.z, pattern.w};
    if (tid < n_u32 % 4) p[n4 * 4 + tid] = pw[tid];
}

/* size(): count slots whose key is neither empty nor tombstone
 * (single_value_hash_table.cuh:535-592) */
template <class L>
__global__ void __launch_bounds__(256) count_valid_kernel(const void *slots, uint64_t capacity,
                                                          uint64_t empty, uint64_t tomb,
                                                          unsigned long long *count)
{
    using K = typename L::key_t;
    constexpr int SB = L::kSlotBytes;
    constexpr int SPV = 16 / SB; /* slots per 16-byte vector */
    const uint64_t nvec = capacity / SPV;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    unsigned long long c = 0;
    for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < nvec; v += stride) {
        const LaneWords lw = load_lane<16>(reinterpret_cast<const unsigned char *>(slots) + v * 16);
#pragma unroll
        for (int s = 0; s < SPV; ++s) {
            const K k = slot_key<L>(lw, s);
            c += (k != K(empty) && k != K(tomb));
        }
    }
    /* ragged tail (capacity not a multiple of SPV) */
    if (blockIdx.x == 0 && threadIdx.x < capacity % SPV) {
        const uint64_t sidx = nvec * SPV + threadIdx.x;
        const K k = *reinterpret_cast<const K *>(reinterpret_cast<const unsigned char *>(slots) + sidx * SB);
        c += (k != K(empty) && k != K(tomb));
    }
    c = __reduce_add_sync(kFull, unsigned(c));
    __shared__ unsigned long long sm[8];
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) s += sm[w];
        if (s) atomicAdd(count, s);
    }
}

/* retrieve_all(): compact the valid slots into keys_out / values_out
 * (single_value_hash_table.cuh:391-417) by block tiles (wc_compact.cuh) */
template <class L>
__global__ void __launch_bounds__(256) dump_kernel(const void *slots, uint64_t capacity,
                                                   uint64_t empty, uint64_t tomb,
                                                   void *keys_out, void *values_out,
                                                   unsigned long long *count)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    constexpr int SB = L::kSlotBytes;
    const unsigned char *const base = reinterpret_cast<const unsigned char *>(slots);
    compact_tiles<K, V>(capacity, reinterpret_cast<K *>(keys_out),
                        L::kHasValue ? reinterpret_cast<V *>(values_out) : nullptr, count,
                        [&](uint64_t s, K &k, V &v) {
                            const unsigned char *sp = base + s * SB;
                            k = *reinterpret_cast<const K *>(sp);
                            if constexpr (L::kHasValue)
                                v = *slot_value_ptr<L>(const_cast<unsigned char *>(sp));
                            return k != K(empty) && k != K(tomb);
                        });
}

} // namespace b200
} // namespace warpcore

#endif /* WC_KERNELS_CUH */
