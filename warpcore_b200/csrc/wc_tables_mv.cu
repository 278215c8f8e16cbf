/* MultiValueHashTable kernels for the u32/u32 and u64/u64 layouts (see wc_mv.cuh) */
#include "wc_internal.h"

namespace warpcore {
namespace b200 {

template <class L, int W>
static MvKernels mv_pick()
{
    MvKernels k;
    k.insert = reinterpret_cast<const void *>(mv_insert_kernel<L, W>);
    k.count = reinterpret_cast<const void *>(mv_find_kernel<L, W, false>);
    k.values = reinterpret_cast<const void *>(mv_find_kernel<L, W, true>);
    k.unique = reinterpret_cast<const void *>(mv_unique_keys_kernel<L, W>);
    return k;
}

template <class L>
static MvKernels mv_pick_w(int W)
{
    switch (W) {
    case 1: return mv_pick<L, 1>();
    case 2: return mv_pick<L, 2>();
    case 4: return mv_pick<L, 4>();
    case 8: return mv_pick<L, 8>();
    case 16: return mv_pick<L, 16>();
    case 32: return mv_pick<L, 32>();
    default: return MvKernels{};
    }
}

MvKernels mv_kernels(int layout, int W)
{
    if (layout == kLayoutKV32) return mv_pick_w<LayoutKV32>(W);
    if (layout == kLayoutKV64) return mv_pick_w<LayoutKV64>(W);
    return MvKernels{};
}

MvScanKernels mv_scan_kernels()
{
    MvScanKernels k;
    k.tile_sums = reinterpret_cast<const void *>(scan_tile_sums_kernel<0>);
    k.tile_offsets = reinterpret_cast<const void *>(scan_tile_offsets_kernel<0>);
    k.apply = reinterpret_cast<const void *>(scan_apply_kernel<0>);
    k.dry_status = reinterpret_cast<const void *>(mv_dry_status_kernel<0>);
    return k;
}

} // namespace b200
} // namespace warpcore
