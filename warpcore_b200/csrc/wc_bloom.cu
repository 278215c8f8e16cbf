/* Bloom filter kernels and the table-wide scan kernels (size, retrieve_all) */
#include "wc_internal.h"

namespace warpcore {
namespace b200 {

/* blocks of at most 128 bytes: one key per lane (bloom_lane_kernel);
 * larger blocks: the cooperative kernel */
#ifndef WC_BLOOM_LANE
#define WC_BLOOM_LANE 1
#endif

template <class K, class S, int CG>
static BloomKernel pick_bloom(bool insert)
{
    if constexpr (WC_BLOOM_LANE && CG * sizeof(S) <= 128)
        return insert ? bloom_lane_kernel<K, S, CG, true> : bloom_lane_kernel<K, S, CG, false>;
    else
        return insert ? bloom_kernel<K, S, CG, true> : bloom_kernel<K, S, CG, false>;
}

template <class K, class S>
static BloomKernel pick_bloom_cg(int cg, bool insert)
{
    switch (cg) {
    case 1: return pick_bloom<K, S, 1>(insert);
    case 2: return pick_bloom<K, S, 2>(insert);
    case 4: return pick_bloom<K, S, 4>(insert);
    case 8: return pick_bloom<K, S, 8>(insert);
    case 16: return pick_bloom<K, S, 16>(insert);
    case 32: return pick_bloom<K, S, 32>(insert);
    default: return nullptr;
    }
}

BloomKernel bloom_kernel_ptr(int key_bytes, int slot_bytes, int cg, bool insert)
{
    if (key_bytes == 4 && slot_bytes == 4) return pick_bloom_cg<uint32_t, uint32_t>(cg, insert);
    if (key_bytes == 4 && slot_bytes == 8) return pick_bloom_cg<uint32_t, uint64_t>(cg, insert);
    if (key_bytes == 8 && slot_bytes == 4) return pick_bloom_cg<uint64_t, uint32_t>(cg, insert);
    if (key_bytes == 8 && slot_bytes == 8) return pick_bloom_cg<uint64_t, uint64_t>(cg, insert);
    return nullptr;
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
