/* MultiValueHashTable kernels for the u32/u32 and u64/u64 layouts (see wc_mv.cuh) */
#include "wc_mv_pick.cuh"

namespace warpcore {
namespace b200 {

MvKernels mv_kernels(int layout, int W)
{
    if (layout == kLayoutKV32) return mv_pick_w<LayoutKV32>(W);
    if (layout == kLayoutKV64) return mv_pick_w<LayoutKV64>(W);
    if (layout == kLayoutK32V64 || layout == kLayoutK64V32) return mv_kernels_mixed(layout, W);
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
