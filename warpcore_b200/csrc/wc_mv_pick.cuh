/*
 * wc_mv_pick.cuh -- the MultiValueHashTable kernels of one slot layout, by
 * window width; wc_tables_mv.cu (equal widths) and wc_tables_mv_mixed.cu
 * (mixed widths) instantiate it, so the layouts compile in parallel.
 */
#ifndef WC_MV_PICK_CUH
#define WC_MV_PICK_CUH

#include "wc_internal.h"

namespace warpcore {
namespace b200 {

template <class L, int W>
MvKernels mv_pick()
{
    MvKernels k;
    k.insert = reinterpret_cast<const void *>(mv_insert_kernel<L, W>);
    k.count = reinterpret_cast<const void *>(mv_find_kernel<L, W, false>);
    k.values = reinterpret_cast<const void *>(mv_find_kernel<L, W, true>);
    k.unique = reinterpret_cast<const void *>(mv_unique_keys_kernel<L, W>);
    return k;
}

template <class L>
MvKernels mv_pick_w(int W)
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

} // namespace b200
} // namespace warpcore

#endif /* WC_MV_PICK_CUH */
