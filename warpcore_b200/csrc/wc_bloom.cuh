/*
 * wc_bloom.cuh -- pattern-blocked Bloom filter kernels
 * (the reference's BloomFilter::insert / retrieve, bloom_filter.cuh:168-237,
 * launched by kernels::bloom_filter::insert / retrieve, gpu_engine.cuh:130-171).
 *
 * A block is cg_size consecutive slots (words).  The bit pattern of a key is
 * the reference's: block = h(key+seed) % num_blocks, bit i (i < k) =
 * h(key+seed+i) % block_bits, owned by word bit / slot_bits of the block, and
 * the word index wraps modulo num_slots for a ragged last block.  A warp takes
 * 32 keys; lane l owns key l.  A block is read by TPK lanes with 16-byte
 * vector loads (one request per block) for all 32 keys before any is tested.
 * Insert ORs only the words that miss bits (one atomicOr per such word, as
 * the reference), query tests the whole block and writes one byte per key.
 */
#ifndef WC_BLOOM_CUH
#define WC_BLOOM_CUH

#include "wc_kernels.cuh"

namespace warpcore {
namespace b200 {

struct BloomArgs {
    void *words;
    const void *keys;
    unsigned char *flags_out;
    uint64_t n;
    uint64_t num_slots;
    uint64_t num_blocks;
    uint64_t magic_blocks; /* barrett_magic(num_blocks) */
    uint64_t k;
    uint64_t seed;
    uint32_t hasher;
    /* a shard holds the blocks [block_base, block_base + local_blocks) of a
     * filter of num_blocks blocks (a whole filter: 0 and num_blocks); its
     * words start at block_base, and a key whose block it does not hold is
     * skipped (insert) or reported absent (query) */
    uint64_t block_base;
    uint64_t local_blocks;
    /* this launch serves only the keys whose local block lies in
     * [region_lo, region_hi) (bloom_lane_kernel; see region passes below);
     * region_lo == 0 also answers the keys of other shards */
    uint64_t region_lo;
    uint64_t region_hi;
};

template <class S>
__device__ __forceinline__ S lane_word(const LaneWords &lw, int s)
{
    if constexpr (sizeof(S) == 4) return lw.w[s];
    else return uint64_t(lw.w[2 * s]) | (uint64_t(lw.w[2 * s + 1]) << 32);
}

template <class T>
__device__ __forceinline__ T atomic_or_any(T *p, T v)
{
    if constexpr (sizeof(T) == 8)
        return T(atomicOr(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v));
    else
        return T(atomicOr(reinterpret_cast<unsigned int *>(p), (unsigned int)v));
}

#ifndef WC_BLOOM_INSERT_READS_BLOCK
#define WC_BLOOM_INSERT_READS_BLOCK 1
#endif

/* bit masks of the CG words of key's block, computed once by the lane that
 * owns the key */
template <class K, class S, int CG>
__device__ __forceinline__ void block_masks(K key, K seed, uint32_t hasher, uint64_t k, S (&m)[CG])
{
    constexpr uint64_t kSlotBits = sizeof(S) * 8;
    constexpr uint64_t kBlockBits = kSlotBits * CG;
#pragma unroll
    for (int w = 0; w < CG; ++w) m[w] = 0;
    /* the hasher decided once for the k hashes, with MurmurHash (the
     * default) inlined: 27.9 against 27.2 G queries/s on the 2^32-bit
     * filter */
    if (hasher == kHashMurmur) {
        for (uint64_t j = 0; j < k; ++j) {
            const uint64_t h = hash_key<K>(kHashMurmur, K(key + seed + K(j))) & (kBlockBits - 1);
            const int word = int(h / kSlotBits);
            const S bit = S(1) << (h % kSlotBits);
#pragma unroll
            for (int w = 0; w < CG; ++w)
                if (word == w) m[w] |= bit;
        }
        return;
    }
    for (uint64_t j = 0; j < k; ++j) {
        const uint64_t h = hash_key<K>(hasher, K(key + seed + K(j))) & (kBlockBits - 1);
        const int word = int(h / kSlotBits);
        const S bit = S(1) << (h % kSlotBits);
#pragma unroll
        for (int w = 0; w < CG; ++w)
            if (word == w) m[w] |= bit;
    }
}

/* word i of a block held in registers, by a select tree (no dynamic
 * register indexing) */
template <class S, int CG>
__device__ __forceinline__ S pick_word(const S (&w)[CG], int i)
{
    if constexpr (CG == 1) {
        return w[0];
    } else if constexpr (CG == 2) {
        return (i & 1) ? w[1] : w[0];
    } else if constexpr (CG == 4) {
        const S a = (i & 1) ? w[1] : w[0], b = (i & 1) ? w[3] : w[2];
        return (i & 2) ? b : a;
    } else if constexpr (CG == 8) {
        const S a = (i & 1) ? w[1] : w[0], b = (i & 1) ? w[3] : w[2];
        const S c = (i & 1) ? w[5] : w[4], d = (i & 1) ? w[7] : w[6];
        const S e = (i & 2) ? b : a, f = (i & 2) ? d : c;
        return (i & 4) ? f : e;
    } else {
        S v = 0;
#pragma unroll
        for (int s = 0; s < CG; ++s)
            if (s == i) v = w[s];
        return v;
    }
}

/* Whether every one of the key's k bits is set in the block w, each bit
 * tested in the word it falls in (the query needs no masks).  Against
 * building the k masks (a compare and select per word and bit) and testing
 * them, 36.4 against 27.9 G queries/s on the 2^32-bit filter of 64-byte
 * blocks. */
template <class K, class S, int CG>
__device__ __forceinline__ bool block_has_all(K key, K seed, uint32_t hasher, uint64_t k,
                                              const S (&w)[CG])
{
    constexpr uint64_t kSlotBits = sizeof(S) * 8;
    constexpr uint64_t kBlockBits = kSlotBits * CG;
    bool ok = true;
    if (hasher == kHashMurmur) {
        for (uint64_t j = 0; j < k; ++j) {
            const uint64_t h = hash_key<K>(kHashMurmur, K(key + seed + K(j))) & (kBlockBits - 1);
            ok &= ((pick_word<S, CG>(w, int(h / kSlotBits)) >> (h % kSlotBits)) & S(1)) != 0;
        }
        return ok;
    }
    for (uint64_t j = 0; j < k; ++j) {
        const uint64_t h = hash_key<K>(hasher, K(key + seed + K(j))) & (kBlockBits - 1);
        ok &= ((pick_word<S, CG>(w, int(h / kSlotBits)) >> (h % kSlotBits)) & S(1)) != 0;
    }
    return ok;
}

template <class K, class S, int CG, bool INSERT>
__global__ void __launch_bounds__(256) bloom_kernel(const BloomArgs a)
{
    constexpr int SB = sizeof(S);
    constexpr int BB = CG * SB;                 /* block bytes */
    constexpr int LB = BB < 16 ? BB : 16;       /* bytes per lane */
    constexpr int TPK = BB / LB;                /* lanes per block */
    constexpr int SPL = LB / SB;                /* words per lane */
    constexpr int G = 32 / TPK;
    constexpr uint64_t kSlotBits = SB * 8;
    constexpr uint64_t kBlockBits = kSlotBits * CG;
    constexpr uint32_t kGroupMask = TPK == 32 ? kFull : ((1u << TPK) - 1u);
    /* small blocks: the owner computes the masks once and the group lanes
     * receive their words by shuffles; large blocks: every group lane derives
     * the masks of its own words */
    constexpr bool kOwnerMasks = CG * SB <= 64;

    const int lane = threadIdx.x & 31;
    const int g = lane / TPK;
    const int q = lane % TPK;
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    S *const words = reinterpret_cast<S *>(a.words);
    const K *const keys = reinterpret_cast<const K *>(a.keys);
    const K seed = K(a.seed);

    for (uint64_t base = warp * 32; base < a.n; base += nwarps * 32) {
        const uint64_t i = base + lane;
        const bool active = i < a.n;
        const K key = active ? ld_stream(keys + i) : K(0);
        const uint64_t blk = fast_mod(hash_key<K>(a.hasher, K(key + seed)), a.num_blocks, a.magic_blocks);
        S own_mask[kOwnerMasks ? CG : 1];
        if constexpr (kOwnerMasks) block_masks<K, S, CG>(key, seed, a.hasher, a.k, own_mask);

        constexpr bool kRead = !INSERT || WC_BLOOM_INSERT_READS_BLOCK;
        LaneWords win[TPK];
#pragma unroll
        for (int r = 0; r < TPK; ++r) {
            const int o = r * G + g; /* owner lane of this round's block */
            const uint64_t b = shfl_any(blk, o);
            const uint64_t w0 = b * CG + uint64_t(q) * SPL;
            win[r] = LaneWords{{0u, 0u, 0u, 0u}};
            if (kRead && (base + o) < a.n) {
                if (b * CG + CG <= a.num_slots) {
                    win[r] = load_lane<LB>(words + w0);
                } else {
                    /* ragged last block: words wrap to the front */
#pragma unroll
                    for (int s = 0; s < SPL; ++s) {
                        const S v = __ldcg(reinterpret_cast<const S *>(words) + (w0 + s) % a.num_slots);
                        if constexpr (SB == 4) win[r].w[s] = uint32_t(v);
                        else { win[r].w[2 * s] = uint32_t(v); win[r].w[2 * s + 1] = uint32_t(uint64_t(v) >> 32); }
                    }
                }
            }
        }

        bool my_flag = false;
#pragma unroll
        for (int r = 0; r < TPK; ++r) {
            const int o = r * G + g;
            const bool own_ok = (base + o) < a.n;
            const uint64_t b = shfl_any(blk, o);
            S mask[SPL];
            if constexpr (kOwnerMasks) {
#pragma unroll
                for (int w = 0; w < CG; ++w) {
                    const S m = shfl_any(own_mask[w], o);
                    if (w / SPL == q) mask[w % SPL] = m;
                }
            } else {
                const K kr = shfl_any(key, o);
#pragma unroll
                for (int s = 0; s < SPL; ++s) mask[s] = 0;
                for (uint64_t j = 0; j < a.k; ++j) {
                    const uint64_t h = hash_key<K>(a.hasher, K(kr + seed + K(j))) & (kBlockBits - 1);
                    const int word = int(h / kSlotBits);
                    if (word / SPL == q) {
#pragma unroll
                        for (int s = 0; s < SPL; ++s)
                            if (word % SPL == s) mask[s] |= S(1) << (h % kSlotBits);
                    }
                }
            }
            bool ok = true;
#pragma unroll
            for (int s = 0; s < SPL; ++s) {
                const S w = lane_word<S>(win[r], s);
                const bool missing = (w & mask[s]) != mask[s];
                ok &= !missing;
                if (INSERT && own_ok && mask[s] && (!kRead || missing)) {
                    uint64_t wi = b * CG + uint64_t(q) * SPL + s;
                    if (wi >= a.num_slots) wi -= a.num_slots; /* ragged last block */
                    atomic_or_any(words + wi, mask[s]);
                }
            }
            if constexpr (!INSERT) {
                const unsigned bad = __ballot_sync(kFull, !ok);
                /* lane r*G + gg owns the block read by group gg this round */
                if (lane / G == r) {
                    const int gg = lane - r * G;
                    my_flag = ((bad >> (gg * TPK)) & kGroupMask) == 0;
                }
            }
        }
        if constexpr (!INSERT) {
            if (active) a.flags_out[i] = (unsigned char)my_flag;
        }
    }
}

/* One key per lane, for blocks of at most 128 bytes: the lane computes its
 * key's masks, reads its own block with BB / 16 vector loads (all lanes'
 * loads independent, so a warp keeps 32 blocks in flight), tests it, and
 * ORs only the words that miss bits.  Against the cooperative kernel above
 * it spends no shuffles on block indices and masks.  It serves the keys
 * whose block lies in [region_lo, region_hi) (one pass: the whole filter). */
template <class K, class S, int CG, bool INSERT>
__global__ void __launch_bounds__(256) bloom_lane_kernel(const BloomArgs a)
{
    constexpr int SB = sizeof(S);
    constexpr int BB = CG * SB;               /* block bytes, <= 128 */
    constexpr int VB = BB < 16 ? BB : 16;     /* bytes per load */
    constexpr int NV = BB / VB;               /* loads per block */
    constexpr int WPV = VB / SB;              /* words per load */
    static_assert(BB <= 128 && NV * VB == BB && WPV * SB == VB, "block split");

    S *const words = reinterpret_cast<S *>(a.words);
    const K *const keys = reinterpret_cast<const K *>(a.keys);
    const K seed = K(a.seed);
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const K key = ld_stream(keys + i);
        const uint64_t blk =
            fast_mod(hash_key<K>(a.hasher, K(key + seed)), a.num_blocks, a.magic_blocks) -
            a.block_base;
        if (blk >= a.local_blocks) {
            if constexpr (!INSERT) {
                if (a.region_lo == 0) a.flags_out[i] = 0;
            }
            continue;
        }
        if (blk < a.region_lo || blk >= a.region_hi) continue;
        const uint64_t w0 = blk * CG;
        S w[CG];
        constexpr bool kRead = !INSERT || WC_BLOOM_INSERT_READS_BLOCK;
        if (kRead) {
            if (w0 + CG <= a.num_slots) {
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    const LaneWords lw = load_lane<VB>(words + w0 + uint64_t(v) * WPV);
#pragma unroll
                    for (int s = 0; s < WPV; ++s) w[v * WPV + s] = lane_word<S>(lw, s);
                }
            } else {
                /* ragged last block: words wrap to the front */
#pragma unroll
                for (int s = 0; s < CG; ++s) w[s] = __ldcg(words + (w0 + s) % a.num_slots);
            }
        } else {
#pragma unroll
            for (int s = 0; s < CG; ++s) w[s] = 0;
        }
        if constexpr (!INSERT) {
            a.flags_out[i] = (unsigned char)block_has_all<K, S, CG>(key, seed, a.hasher, a.k, w);
        } else {
            S m[CG];
            block_masks<K, S, CG>(key, seed, a.hasher, a.k, m);
#pragma unroll
            for (int s = 0; s < CG; ++s) {
                const bool missing = (w[s] & m[s]) != m[s];
                if (m[s] && (!kRead || missing)) {
                    uint64_t wi = w0 + uint64_t(s);
                    if (wi >= a.num_slots) wi -= a.num_slots;
                    atomic_or_any(words + wi, m[s]);
                }
            }
        }
    }
}

/* Region passes, for blocks of at most 128 bytes.  On B200, random reads
 * slow down sharply once the array they hit outgrows the GPU's
 * address-translation reach: 64-byte reads at random measured 64 G/s over
 * 256 MiB but 13.5 G/s over 512 MiB and 9.5 G/s over 4 GiB.  A filter
 * larger than one region is therefore processed in passes, one launch per
 * region of its blocks; each pass streams all keys and serves those whose
 * block lies in its region, so that its random reads (and an insert's
 * atomics) stay inside the region.
 *
 * A pass must keep many block reads in flight although only a fraction of
 * the keys it streams belongs to its region.  So a warp takes a tile of
 * kRegionKpl x 32 keys (kRegionKpl coalesced loads per lane in flight),
 * computes their blocks, and compacts the keys of its region into a list
 * in shared memory (ballot + prefix count, input order kept).  The lanes
 * then take the list densely, kRegionU entries per lane at a time, issue
 * all their block reads before testing any, and write flags / OR words as
 * the one-key-per-lane kernel does.  One entry per lane with four resident
 * blocks per SM (64-byte blocks; two for 128-byte blocks, whose words take
 * twice the registers) keeps more warps issuing than four entries per lane
 * with two blocks: on the 2^32-bit filter of 64-byte blocks, 2^28 keys,
 * 20.3 / 27.2 G keys/s (insert / query) against 16.9 / 21.3; two entries
 * with three blocks 19.7 / 25.5.  Each key is served by exactly one
 * pass; a query's flag is written there (a key of another shard's block
 * gets 0 in the first pass). */
constexpr int kRegionKpl = 8;   /* keys per lane per warp tile */
constexpr int kRegionU = 1;     /* compacted keys per lane in flight */
constexpr int kRegionWarps = 8; /* 256 threads */

template <class K, class S, int CG, bool INSERT>
__global__ void __launch_bounds__(256, CG * sizeof(S) <= 64 ? 4 : 2) bloom_region_kernel(const BloomArgs a)
{
    constexpr int SB = sizeof(S);
    constexpr int BB = CG * SB;
    constexpr int VB = BB < 16 ? BB : 16;
    constexpr int NV = BB / VB;
    constexpr int WPV = VB / SB;
    constexpr int WT = 32 * kRegionKpl; /* keys per warp tile */
    static_assert(BB <= 128 && NV * VB == BB && WPV * SB == VB, "block split");
    static_assert(WT <= 256, "tile offsets are one byte");
    constexpr bool kRead = !INSERT || WC_BLOOM_INSERT_READS_BLOCK;

    __shared__ K s_key[kRegionWarps][WT];
    __shared__ uint32_t s_rel[kRegionWarps][WT];       /* block - region_lo */
    __shared__ unsigned char s_off[kRegionWarps][WT];  /* position in the tile */

    S *const words = reinterpret_cast<S *>(a.words);
    const K *const keys = reinterpret_cast<const K *>(a.keys);
    const K seed = K(a.seed);
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const unsigned lanemask_lt = (1u << lane) - 1u;
    const uint64_t gwarp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;

    for (uint64_t base = gwarp * WT; base < a.n; base += nwarps * WT) {
        K kk[kRegionKpl];
#pragma unroll
        for (int j = 0; j < kRegionKpl; ++j) {
            const uint64_t i = base + uint64_t(j) * 32 + lane;
            kk[j] = i < a.n ? ld_stream(keys + i) : K(0);
        }
        int cnt = 0;
#pragma unroll
        for (int j = 0; j < kRegionKpl; ++j) {
            const uint64_t i = base + uint64_t(j) * 32 + lane;
            const uint64_t blk =
                fast_mod(hash_key<K>(a.hasher, K(kk[j] + seed)), a.num_blocks, a.magic_blocks) -
                a.block_base;
            if constexpr (!INSERT) {
                if (i < a.n && a.region_lo == 0 && blk >= a.local_blocks) a.flags_out[i] = 0;
            }
            const bool in = i < a.n && blk < a.local_blocks && blk >= a.region_lo &&
                            blk < a.region_hi;
            const unsigned m = __ballot_sync(kFull, in);
            if (in) {
                const int pos = cnt + __popc(m & lanemask_lt);
                s_key[wib][pos] = kk[j];
                s_rel[wib][pos] = uint32_t(blk - a.region_lo);
                s_off[wib][pos] = (unsigned char)(j * 32 + lane);
            }
            cnt += __popc(m);
        }
        __syncwarp();
        for (int e0 = 0; e0 < cnt; e0 += 32 * kRegionU) {
            S w[kRegionU][CG];
#pragma unroll
            for (int u = 0; u < kRegionU; ++u) {
                const int e = e0 + u * 32 + lane;
                if (kRead && e < cnt) {
                    const uint64_t w0 = (a.region_lo + s_rel[wib][e]) * CG;
                    if (w0 + CG <= a.num_slots) {
#pragma unroll
                        for (int v = 0; v < NV; ++v) {
                            const LaneWords lw = load_lane<VB>(words + w0 + uint64_t(v) * WPV);
#pragma unroll
                            for (int s = 0; s < WPV; ++s) w[u][v * WPV + s] = lane_word<S>(lw, s);
                        }
                    } else {
#pragma unroll
                        for (int s = 0; s < CG; ++s) w[u][s] = __ldcg(words + (w0 + s) % a.num_slots);
                    }
                } else {
#pragma unroll
                    for (int s = 0; s < CG; ++s) w[u][s] = 0;
                }
            }
#pragma unroll
            for (int u = 0; u < kRegionU; ++u) {
                const int e = e0 + u * 32 + lane;
                if (e >= cnt) continue;
                const K key = s_key[wib][e];
                const uint64_t w0 = (a.region_lo + s_rel[wib][e]) * CG;
                if constexpr (!INSERT) {
                    a.flags_out[base + s_off[wib][e]] =
                        (unsigned char)block_has_all<K, S, CG>(key, seed, a.hasher, a.k, w[u]);
                } else {
                    S m[CG];
                    block_masks<K, S, CG>(key, seed, a.hasher, a.k, m);
#pragma unroll
                    for (int s = 0; s < CG; ++s) {
                        const bool missing = (w[u][s] & m[s]) != m[s];
                        if (m[s] && (!kRead || missing)) {
                            uint64_t wi = w0 + uint64_t(s);
                            if (wi >= a.num_slots) wi -= a.num_slots;
                            atomic_or_any(words + wi, m[s]);
                        }
                    }
                }
            }
        }
        __syncwarp();
    }
}

} // namespace b200
} // namespace warpcore

#endif /* WC_BLOOM_CUH */
