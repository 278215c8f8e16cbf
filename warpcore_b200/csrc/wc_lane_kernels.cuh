/*
 * wc_lane_kernels.cuh -- whole-window probing with one key per lane.
 *
 * Same bucket sequence, claim order (lowest free slot of a window first),
 * statuses and results as table_op_kernel (wc_kernels.cuh); the difference
 * is who reads a window.  table_op_kernel lets TPK lanes read one window
 * together and returns match / free masks to the owner lane with ballots:
 * for u64 pairs at CG 8 (TPK 8) a warp then spends about 35 instructions
 * per key on rounds of ballots and shuffles, and at 50 % issue-active the
 * insert is bound by instruction issue, not by memory.  Here every lane
 * reads its own key's window with 32-byte vector loads (sm_100; four for a
 * 128-byte window), tests the window's slots in registers and issues its
 * own compare-and-swap: no ballots, no shuffles, no shared memory.
 *
 * Each lane issues one memory operation per wave, a window read or a
 * claim's compare-and-swap, so a warp keeps 32 of them in flight.  Keys are
 * refilled in input order from a double-buffered prefetch of the warp's
 * contiguous key range, as in table_op_kernel.  Equal keys need no merging
 * before the atomics: every claim goes to the lowest free slot of the
 * window its lane read, so two claims of one key meet on one slot, and the
 * compare-and-swap that loses sees the key.  A claim that loses its slot to
 * another key reads the window again.
 *
 * Insert, retrieve and erase; counting inserts keep table_op_kernel and its
 * shared-memory count cache.
 */
#ifndef WC_LANE_KERNELS_CUH
#define WC_LANE_KERNELS_CUH

#include "wc_kernels.cuh"

namespace warpcore {
namespace b200 {

/* resident 256-thread blocks per SM the lane kernels are built for: 4 for
 * u32 pairs with windows of at most 64 bytes (64 registers, no spills; the
 * u32/u32 insert of 2^20 keys into 2 097 496 slots ran 21.2-21.4 against
 * 20.2 G keys/s with 3, the retrieve unchanged, and 5 spilled and lost),
 * 3 elsewhere, where 4 spills */
template <class L, int W>
constexpr int lane_min_blocks()
{
    return (L::kSlotBytes == 8 && L::kHasValue && W * L::kSlotBytes <= 64) ? 4 : 3;
}

/* a bucket's window of WB bytes, read by one lane from L2 (.cg: a claim by
 * another lane is seen): 32-byte vector loads for windows of 32 bytes or
 * more, else one load of the window */
template <int WB>
__device__ __forceinline__ void load_window(const unsigned char *p, uint32_t (&w)[WB / 4])
{
    if constexpr (WB >= 32) {
#pragma unroll
        for (int c = 0; c < WB / 32; ++c) {
            asm volatile("ld.global.cg.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(w[8 * c + 0]), "=r"(w[8 * c + 1]), "=r"(w[8 * c + 2]),
                           "=r"(w[8 * c + 3]), "=r"(w[8 * c + 4]), "=r"(w[8 * c + 5]),
                           "=r"(w[8 * c + 6]), "=r"(w[8 * c + 7])
                         : "l"(p + 32 * c));
        }
    } else if constexpr (WB == 16) {
        const uint4 v = __ldcg(reinterpret_cast<const uint4 *>(p));
        w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
    } else if constexpr (WB == 8) {
        const uint2 v = __ldcg(reinterpret_cast<const uint2 *>(p));
        w[0] = v.x; w[1] = v.y;
    } else {
        w[0] = __ldcg(reinterpret_cast<const unsigned int *>(p));
    }
}

/* key / payload of slot s of a window held as 32-bit words */
template <class L>
__device__ __forceinline__ typename L::key_t window_key(const uint32_t *w, int s)
{
    using K = typename L::key_t;
    constexpr int SB = L::kSlotBytes;
    if constexpr (SB == 16) {
        if constexpr (sizeof(K) == 8) return uint64_t(w[4 * s]) | (uint64_t(w[4 * s + 1]) << 32);
        else return w[4 * s];
    } else if constexpr (SB == 8 && L::kHasValue) {
        return w[2 * s];
    } else if constexpr (SB == 8) {
        return uint64_t(w[2 * s]) | (uint64_t(w[2 * s + 1]) << 32);
    } else {
        return w[s];
    }
}

template <class L>
__device__ __forceinline__ typename L::val_t window_val(const uint32_t *w, int s)
{
    using V = typename L::val_t;
    constexpr int SB = L::kSlotBytes;
    if constexpr (SB == 16) {
        if constexpr (sizeof(V) == 8) return uint64_t(w[4 * s + 2]) | (uint64_t(w[4 * s + 3]) << 32);
        else return w[4 * s + 2];
    } else if constexpr (SB == 8 && L::kHasValue) {
        return w[2 * s + 1];
    } else {
        return 0;
    }
}

/* payload of slot `target` (a run-time index): selected by an unrolled
 * loop, so that the window stays in registers */
template <class L, int W>
__device__ __forceinline__ typename L::val_t window_val_at(const uint32_t *w, int target)
{
    typename L::val_t v = 0;
#pragma unroll
    for (int s = 0; s < W; ++s)
        if (s == target) v = window_val<L>(w, s);
    return v;
}

template <class L, int W, int OP>
__global__ void __launch_bounds__(256, lane_min_blocks<L, W>()) lane_op_kernel(const TableOpArgs a)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    constexpr int SB = L::kSlotBytes;
    constexpr int WB = W * SB;
    static_assert(WB <= 128 && WB >= 4, "window of one lane");
    static_assert(OP == kOpInsert || OP == kOpRetrieve || OP == kOpErase, "operation");
    constexpr bool kValueIn = OP == kOpInsert && L::kHasValue;

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

    /* the key this lane owns: waiting for its window (claiming == false) or
     * for the compare-and-swap on slot claim_slot, expected to hold the
     * empty key with payload claim_expect */
    bool has = false, pending = false, flag = false, claiming = false;
    int claim_slot = 0;
    V claim_expect = 0;
    uint64_t i = 0, bucket = 0, step = 0, wins = 0;
    K key = empty;
    V val = 0;
    uint32_t st = kStNone, join = 0;
    int live_delta = 0;

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
            claiming = false;
            st = kStNone;
            wins = 0;
            step = 0;
            if (key == empty || key == tomb) {
                st = kStInvalidKey;
                join |= kStInvalidKey;
                pending = false;
            } else {
                bucket = probe_begin<K>(t, key);
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

        /* ---- one memory operation per pending lane: its window, or its
         * claim; all lanes' operations are in flight together ---- */
        unsigned char *const bptr = slots + bucket * uint64_t(W) * SB;
        uint32_t w[WB / 4];
        K cas_old = empty;
        V cas_old_payload = 0;
        if (pending) {
            if constexpr (OP == kOpInsert) {
                if (claiming)
                    cas_old = cas_slot<L>(bptr + claim_slot * SB, empty, claim_expect, key, val,
                                          &cas_old_payload);
                else
                    load_window<WB>(bptr, w);
            } else {
                load_window<WB>(bptr, w);
            }
        }

        bool advance = false;
        if (pending && !claiming) {
            uint32_t hit = 0, emp = 0;
#pragma unroll
            for (int s = 0; s < W; ++s) {
                const K sk = window_key<L>(w, s);
                hit |= uint32_t(sk == key) << s;
                emp |= uint32_t(sk == empty) << s;
            }
            if (hit) {
                const int s = __ffs(hit) - 1;
                unsigned char *const sp = bptr + s * SB;
                if constexpr (OP == kOpRetrieve) {
                    st = kStNone;
                    flag = true;
                    if constexpr (L::kHasValue) {
                        if (!a.is_set) {
                            V v = window_val_at<L, W>(w, s);
                            if (uint64_t(v) > t.max_count) v = V(t.max_count);
                            st_stream(reinterpret_cast<V *>(a.out) + i, v);
                        }
                    }
                } else if constexpr (OP == kOpInsert) {
                    st = kStDuplicateKey;
                    join |= kStDuplicateKey;
                    store_value<L>(sp, val);
                } else {
                    if (erase_slot<L>(sp, key, tomb)) {
                        fp_store(t, bucket * W + uint64_t(s), kFpTomb);
                        --live_delta;
                    }
                    st = kStNone;
                }
                pending = false;
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
                    /* claim the lowest free slot in the next wave */
                    claiming = true;
                    claim_slot = __ffs(emp) - 1;
                    claim_expect = window_val_at<L, W>(w, claim_slot);
                }
            } else {
                advance = true;
            }
        } else if (pending) {
            if constexpr (OP == kOpInsert) {
                if (cas_old == empty && cas_old_payload == claim_expect) {
                    fp_store(t, bucket * W + uint64_t(claim_slot), fingerprint(key));
                    ++live_delta;
                    st = kStNone;
                    pending = false;
                } else if (cas_old == key) {
                    st = kStDuplicateKey;
                    join |= kStDuplicateKey;
                    store_value<L>(bptr + claim_slot * SB, val);
                    pending = false;
                } else if (cas_old == empty) {
                    claim_expect = cas_old_payload; /* free slot, stale payload: again */
                } else {
                    claiming = false; /* taken by another key: read the window again */
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
    const uint32_t wjoin = __reduce_or_sync(kFull, join);
    const int wlive = int(__reduce_add_sync(kFull, unsigned(live_delta)));
    if (lane == 0) {
        join_status(t.status, wjoin);
        live_add(t, wlive);
    }
}

} // namespace b200
} // namespace warpcore

#endif /* WC_LANE_KERNELS_CUH */
