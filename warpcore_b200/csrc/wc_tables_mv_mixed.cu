/* MultiValueHashTable kernels for the u32/u64 and u64/u32 layouts (see wc_mv.cuh) */
#include "wc_mv_pick.cuh"

namespace warpcore {
namespace b200 {

MvKernels mv_kernels_mixed(int layout, int W)
{
    if (layout == kLayoutK32V64) return mv_pick_w<LayoutK32V64>(W);
    if (layout == kLayoutK64V32) return mv_pick_w<LayoutK64V32>(W);
    return MvKernels{};
}

} // namespace b200
} // namespace warpcore
