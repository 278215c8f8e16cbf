/*
 * wc_batch.cuh -- one launch for many requests on many tables.
 *
 * A batch is a list of requests; each names a table (its device view), an
 * operation (insert or retrieve), device buffers and a key count.  The keys
 * of all requests form one index space [0, total): request r owns
 * [begin_r, begin_r + n_r).  The kernel is the table kernel's warp-batched
 * probing (wc_kernels.cuh) with the table, operation and buffers looked up
 * per key, so requests of different sizes on tables of different capacities
 * share every wave and no request waits for a launch of its own.
 *
 * Requests of one batch must commute: the serving layer puts into one batch
 * only requests on distinct tables, or runs of requests of the same kind on
 * one table (retrieves, or inserts of distinct keys).
 */
#ifndef WC_BATCH_CUH
#define WC_BATCH_CUH

#include "wc_kernels.cuh"

namespace warpcore {
namespace b200 {

struct BatchDesc {
    TableView t;
    const void *keys;
    const void *values; /* insert */
    void *out;          /* retrieve */
    void *status_out;
    uint64_t begin;     /* first index of this request in the batch's key space */
    uint64_t n;
    uint64_t max_windows;
    uint32_t bool_mask;
    int op;             /* kOpInsert or kOpRetrieve */
    int handler;
    int pad;
};

struct BatchArgs {
    const BatchDesc *desc;
    uint64_t nreq;
    uint64_t total;
};

/* small batches carry their descriptors in the kernel parameters, so a
 * launch needs no descriptor copy */
constexpr int kBatchInline = 32;
struct BatchInlineArgs {
    uint64_t nreq;
    uint64_t total;
    BatchDesc desc[kBatchInline];
};

/* descriptors are read with plain loads: they live in global memory or in
 * the parameter space of the launch */
__device__ __forceinline__ uint64_t ldg_u64(const uint64_t *p) { return *p; }

/* request that owns flattened key index i (desc sorted by begin) */
__device__ __forceinline__ uint32_t find_request(const BatchDesc *d, uint64_t nreq, uint64_t i)
{
    uint64_t lo = 0, hi = nreq;
    while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (ldg_u64(&d[mid].begin) <= i) lo = mid;
        else hi = mid;
    }
    return uint32_t(lo);
}

template <class L, int W>
__device__ __forceinline__ void batch_body(const BatchArgs a)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    constexpr int SB = L::kSlotBytes;
    constexpr int WB = W * SB;
    constexpr int LB = WB < 16 ? WB : 16;
    constexpr int TPK = WB / LB;
    constexpr int SPL = LB / SB;
    constexpr int G = 32 / TPK;
    constexpr uint32_t kGroupMask = TPK == 32 ? kFull : ((1u << TPK) - 1u);
    static_assert(L::kHasValue, "batches serve single-value tables");

    const int lane = threadIdx.x & 31;
    const int g = lane / TPK;
    const int q = lane % TPK;
    const unsigned lanemask_lt = (1u << lane) - 1u;
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    const int wib = threadIdx.x >> 5;
    __shared__ uint64_t sh_slots[8][32]; /* byte address of the window's bucket */
    __shared__ K sh_key[8][32];
    __shared__ uint32_t sh_req[8][32];
    __shared__ uint64_t sh_idx[8][32];

    uint64_t per = (a.total + nwarps - 1) / nwarps;
    per = (per + 31) & ~uint64_t(31);
    const uint64_t wb = warp * per < a.total ? warp * per : a.total;
    const uint64_t we = wb + per < a.total ? wb + per : a.total;
    if (wb >= we) return;

    uint64_t cursor = wb;
    bool has = false, pending = false, claiming = false;
    uint32_t req = 0, claim_bits = 0, st = kStNone;
    uint64_t i = 0, bucket = 0, step = 0, wins = 0;
    K key = 0, empty = 0;
    V val = 0, claim_expect = 0;

    for (;;) {
        const unsigned need = __ballot_sync(kFull, !has);
        const uint64_t avail = we - cursor;
        const int take = int(uint64_t(__popc(need)) < avail ? uint64_t(__popc(need)) : avail);
        if (take == 0 && need == kFull) break;
        const int r = __popc(need & lanemask_lt);
        const bool refill = !has && r < take;
        if (refill) {
            i = cursor + r;
            req = find_request(a.desc, a.nreq, i);
            const BatchDesc &d = a.desc[req];
            const uint64_t j = i - d.begin;
            key = ld_stream(reinterpret_cast<const K *>(d.keys) + j);
            empty = K(d.t.empty_key);
            const int op = d.op;
            val = op == kOpInsert ? ld_stream(reinterpret_cast<const V *>(d.values) + j) : V(0);
            has = true;
            pending = true;
            claiming = false;
            claim_bits = 0;
            claim_expect = 0;
            st = kStNone;
            wins = 0;
            step = 0;
            if (key == empty || key == K(d.t.tombstone_key)) {
                st = kStInvalidKey;
                pending = false;
            } else {
                bucket = probe_begin<K>(d.t, key);
            }
        }
        cursor += uint64_t(take);

        const bool loading = pending && !claiming;
        const unsigned pmask = __ballot_sync(kFull, loading);
        bool did_cas = false;
        K cas_old = 0;
        V cas_old_payload = 0;
        if (__any_sync(kFull, pending)) {
            const int cnt = __popc(pmask);
            const int rounds = (cnt + G - 1) / G;
            const int my_rank = __popc(pmask & lanemask_lt);
            const int my_round = my_rank / G;
            const int my_g = my_rank % G;
            __syncwarp();
            if (loading) {
                const BatchDesc &d = a.desc[req];
                sh_slots[wib][my_rank] = reinterpret_cast<uint64_t>(d.t.slots) + bucket * uint64_t(WB);
                sh_key[wib][my_rank] = key;
                sh_req[wib][my_rank] = req;
                sh_idx[wib][my_rank] = i;
            }
            __syncwarp();

            LaneWords win[TPK];
#pragma unroll
            for (int rr = 0; rr < TPK; ++rr) {
                if (rr < rounds) {
                    const int idx = rr * G + g;
                    if (idx < cnt)
                        win[rr] = load_lane<LB>(reinterpret_cast<const unsigned char *>(sh_slots[wib][idx]) + q * LB);
                    else
                        win[rr] = LaneWords{{0u, 0u, 0u, 0u}};
                }
            }

            if (pending && claiming) {
                const BatchDesc &d = a.desc[req];
                const int s = slot_of_bit<TPK, SPL>(lowest_slot_bit<TPK, SPL>(claim_bits));
                unsigned char *const sp = reinterpret_cast<unsigned char *>(d.t.slots) +
                                          (bucket * W + uint64_t(s)) * SB;
                cas_old = cas_slot<L>(sp, empty, claim_expect, key, val, &cas_old_payload);
                did_cas = true;
            }

            uint32_t hit_bits = 0, empty_bits = 0;
#pragma unroll
            for (int rr = 0; rr < TPK; ++rr) {
                if (rr < rounds) {
                    const int idx = rr * G + g;
                    const bool served = idx < cnt;
                    const K kr = served ? sh_key[wib][idx] : K(0);
                    const uint32_t rq = served ? sh_req[wib][idx] : 0u;
                    const K em = served ? K(ldg_u64(&a.desc[rq].t.empty_key)) : K(0);
#pragma unroll
                    for (int s = 0; s < SPL; ++s) {
                        const K sk = slot_key<L>(win[rr], s);
                        const bool h = served && sk == kr;
                        const unsigned hb = __ballot_sync(kFull, h);
                        const unsigned eb = __ballot_sync(kFull, served && sk == em);
                        if (loading && my_round == rr) {
                            hit_bits |= window_bits<TPK, SPL>((hb >> (my_g * TPK)) & kGroupMask, s);
                            empty_bits |= window_bits<TPK, SPL>((eb >> (my_g * TPK)) & kGroupMask, s);
                        }
                        if (h && a.desc[rq].op == kOpRetrieve) {
                            const BatchDesc &d = a.desc[rq];
                            V v = slot_val<L>(win[rr], s);
                            if (uint64_t(v) > d.t.max_count) v = V(d.t.max_count);
                            st_stream(reinterpret_cast<V *>(d.out) + (sh_idx[wib][idx] - d.begin), v);
                        }
                    }
                }
            }

            bool advance = false;
            if (loading) {
                const BatchDesc &d = a.desc[req];
                unsigned char *const bptr = reinterpret_cast<unsigned char *>(d.t.slots) + bucket * uint64_t(WB);
                if (d.op == kOpRetrieve) {
                    if (hit_bits) {
                        st = kStNone;
                        pending = false;
                    } else if (empty_bits) {
                        st = kStKeyNotFound;
                        pending = false;
                    } else {
                        advance = true;
                    }
                } else {
                    if (hit_bits) {
                        store_value<L>(bptr + slot_of_bit<TPK, SPL>(__ffs(hit_bits) - 1) * SB, val);
                        st = kStDuplicateKey;
                        pending = false;
                    } else if (empty_bits) {
                        claiming = true;
                        claim_bits = empty_bits;
                        claim_expect = 0;
                    } else {
                        advance = true;
                    }
                }
            }
            if (did_cas) {
                const BatchDesc &d = a.desc[req];
                const int s = slot_of_bit<TPK, SPL>(lowest_slot_bit<TPK, SPL>(claim_bits));
                unsigned char *const sp = reinterpret_cast<unsigned char *>(d.t.slots) +
                                          (bucket * W + uint64_t(s)) * SB;
                if (cas_old == empty && cas_old_payload == claim_expect) {
                    fp_store(d.t, bucket * W + uint64_t(s), fingerprint(key));
                    live_add(d.t, 1);
                    st = kStNone;
                    pending = false;
                } else if (cas_old == key) {
                    store_value<L>(sp, val);
                    st = kStDuplicateKey;
                    pending = false;
                } else if (cas_old == empty) {
                    claim_expect = cas_old_payload;
                } else {
                    claim_bits &= ~(1u << lowest_slot_bit<TPK, SPL>(claim_bits));
                    if (!claim_bits) {
                        claiming = false;
                        advance = true;
                    }
                }
            }
            if (pending && advance) {
                const BatchDesc &d = a.desc[req];
                if (++wins >= d.max_windows) {
                    pending = false;
                    st = kStProbingLengthExceeded;
                } else {
                    if (wins == 1) step = probe_step<K>(d.t, key);
                    bucket = probe_next(d.t, bucket, step);
                }
            }
        }

        if (has && !pending) {
            const BatchDesc &d = a.desc[req];
            if (d.status_out) {
                const uint64_t j = i - d.begin;
                if (d.handler == kHandlerStatus)
                    st_stream(reinterpret_cast<uint32_t *>(d.status_out) + j, st);
                else if (d.handler == kHandlerBoolean)
                    reinterpret_cast<unsigned char *>(d.status_out)[j] =
                        (unsigned char)((st & d.bool_mask) != 0);
            }
            /* table status: the reference joins every status except a
             * retrieve's none (single_value_hash_table.cuh:285-306, 743-823) */
            const uint32_t jn = st & (kStInvalidKey | kStDuplicateKey | kStKeyNotFound |
                                      kStProbingLengthExceeded);
            if (jn) join_status(d.t.status, jn);
            has = false;
        }
    }
}

template <class L, int W>
__global__ void __launch_bounds__(256, WC_TABLE_MIN_BLOCKS) batch_op_kernel(const BatchArgs a)
{
    batch_body<L, W>(a);
}

template <class L, int W>
__global__ void __launch_bounds__(256, WC_TABLE_MIN_BLOCKS)
    batch_op_kernel_inline(const __grid_constant__ BatchInlineArgs a)
{
    BatchArgs b;
    b.desc = a.desc;
    b.nreq = a.nreq;
    b.total = a.total;
    batch_body<L, W>(b);
}

} // namespace b200
} // namespace warpcore

#endif /* WC_BATCH_CUH */
