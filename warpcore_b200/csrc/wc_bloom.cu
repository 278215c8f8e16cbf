/* Bloom filter kernels and the table-wide scan kernels (size, retrieve_all) */
#include "wc_internal.h"

namespace warpcore {
namespace b200 {

/* blocks of at most 128 bytes: one key per lane (bloom_lane_kernel);
 * larger blocks: the cooperative kernel */
#ifndef WC_BLOOM_LANE
#define WC_BLOOM_LANE 1
#endif

/* a single pass runs the one-key-per-lane kernel, region passes the
 * compacting region kernel */
template <class K, class S, int CG, bool INSERT>
static BloomKernel pick_lane(bool multi_pass)
{
    return multi_pass ? bloom_region_kernel<K, S, CG, INSERT> : bloom_lane_kernel<K, S, CG, INSERT>;
}

template <class K, class S, int CG>
static BloomKernel pick_bloom(bool insert, bool multi_pass, bool *lane)
{
    if constexpr (WC_BLOOM_LANE && CG * sizeof(S) <= 128) {
        *lane = true;
        return insert ? pick_lane<K, S, CG, true>(multi_pass) : pick_lane<K, S, CG, false>(multi_pass);
    } else {
        *lane = false;
        return insert ? bloom_kernel<K, S, CG, true> : bloom_kernel<K, S, CG, false>;
    }
}

template <class K, class S>
static BloomKernel pick_bloom_cg(int cg, bool insert, bool multi_pass, bool *lane)
{
    switch (cg) {
    case 1: return pick_bloom<K, S, 1>(insert, multi_pass, lane);
    case 2: return pick_bloom<K, S, 2>(insert, multi_pass, lane);
    case 4: return pick_bloom<K, S, 4>(insert, multi_pass, lane);
    case 8: return pick_bloom<K, S, 8>(insert, multi_pass, lane);
    case 16: return pick_bloom<K, S, 16>(insert, multi_pass, lane);
    case 32: return pick_bloom<K, S, 32>(insert, multi_pass, lane);
    default: return nullptr;
    }
}

BloomKernel bloom_kernel_ptr(int key_bytes, int slot_bytes, int cg, bool insert, bool multi_pass,
                             bool *lane_kernel)
{
    bool lane = false;
    BloomKernel k = nullptr;
    if (key_bytes == 4 && slot_bytes == 4) k = pick_bloom_cg<uint32_t, uint32_t>(cg, insert, multi_pass, &lane);
    if (key_bytes == 4 && slot_bytes == 8) k = pick_bloom_cg<uint32_t, uint64_t>(cg, insert, multi_pass, &lane);
    if (key_bytes == 8 && slot_bytes == 4) k = pick_bloom_cg<uint64_t, uint32_t>(cg, insert, multi_pass, &lane);
    if (key_bytes == 8 && slot_bytes == 8) k = pick_bloom_cg<uint64_t, uint64_t>(cg, insert, multi_pass, &lane);
    if (lane_kernel) *lane_kernel = lane;
    return k;
}

CountKernel count_kernel(int layout)
{
    switch (layout) {
    case kLayoutKV32: return count_valid_kernel<LayoutKV32>;
    case kLayoutKV64: return count_valid_kernel<LayoutKV64>;
    case kLayoutSet32: return count_valid_kernel<LayoutSet32>;
    case kLayoutSet64: return count_valid_kernel<LayoutSet64>;
    case kLayoutK32V64: return count_valid_kernel<LayoutK32V64>;
    case kLayoutK64V32: return count_valid_kernel<LayoutK64V32>;
    default: return nullptr;
    }
}

RebuildKernel fp_rebuild_kernel_ptr(int layout)
{
    switch (layout) {
    case kLayoutKV32: return fp_rebuild_kernel<LayoutKV32>;
    case kLayoutKV64: return fp_rebuild_kernel<LayoutKV64>;
    case kLayoutSet32: return fp_rebuild_kernel<LayoutSet32>;
    case kLayoutSet64: return fp_rebuild_kernel<LayoutSet64>;
    case kLayoutK32V64: return fp_rebuild_kernel<LayoutK32V64>;
    case kLayoutK64V32: return fp_rebuild_kernel<LayoutK64V32>;
    default: return nullptr;
    }
}

DumpKernel dump_kernel_ptr(int layout)
{
    switch (layout) {
    case kLayoutKV32: return dump_kernel<LayoutKV32>;
    case kLayoutKV64: return dump_kernel<LayoutKV64>;
    case kLayoutSet32: return dump_kernel<LayoutSet32>;
    case kLayoutSet64: return dump_kernel<LayoutSet64>;
    case kLayoutK32V64: return dump_kernel<LayoutK32V64>;
    case kLayoutK64V32: return dump_kernel<LayoutK64V32>;
    default: return nullptr;
    }
}

} // namespace b200
} // namespace warpcore
