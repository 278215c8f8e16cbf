/*
 * wc_tables_pick.cuh -- the (window width, operation, fingerprints) table
 * of bulk table kernels for one slot layout; each wc_tables_*.cu
 * translation unit instantiates it for its layout, so the layouts compile
 * in parallel.
 */
#ifndef WC_TABLES_PICK_CUH
#define WC_TABLES_PICK_CUH

#include "wc_internal.h"

namespace warpcore {
namespace b200 {

template <class L, int W>
TableKernel pick_table_op(int op, bool fp)
{
    switch (op) {
    case kOpInsert: return fp ? fp_op_kernel<L, W, kOpInsert> : table_op_kernel<L, W, kOpInsert>;
    case kOpCount: return fp ? fp_op_kernel<L, W, kOpCount> : table_op_kernel<L, W, kOpCount>;
    case kOpRetrieve: return fp ? fp_op_kernel<L, W, kOpRetrieve> : table_op_kernel<L, W, kOpRetrieve>;
    case kOpErase: return fp ? fp_op_kernel<L, W, kOpErase> : table_op_kernel<L, W, kOpErase>;
    default: return nullptr;
    }
}

template <class L>
TableKernel pick_table_kernel_for(int W, int op, bool fp)
{
    switch (W) {
    case 1: return pick_table_op<L, 1>(op, fp);
    case 2: return pick_table_op<L, 2>(op, fp);
    case 4: return pick_table_op<L, 4>(op, fp);
    case 8: return pick_table_op<L, 8>(op, fp);
    case 16: return pick_table_op<L, 16>(op, fp);
    case 32: return pick_table_op<L, 32>(op, fp);
    default: return nullptr;
    }
}

/* the one-key-per-lane window kernel (wc_lane_kernels.cuh) for insert,
 * retrieve and erase, where a window is at most 128 bytes; else nullptr */
template <class L, int W>
TableKernel pick_lane_op(int op)
{
    if constexpr (W * L::kSlotBytes > 128) {
        return nullptr;
    } else {
        switch (op) {
        case kOpInsert: return lane_op_kernel<L, W, kOpInsert>;
        case kOpRetrieve: return lane_op_kernel<L, W, kOpRetrieve>;
        case kOpErase: return lane_op_kernel<L, W, kOpErase>;
        default: return nullptr;
        }
    }
}

template <class L>
TableKernel pick_lane_kernel_for(int W, int op)
{
    switch (W) {
    case 1: return pick_lane_op<L, 1>(op);
    case 2: return pick_lane_op<L, 2>(op);
    case 4: return pick_lane_op<L, 4>(op);
    case 8: return pick_lane_op<L, 8>(op);
    case 16: return pick_lane_op<L, 16>(op);
    case 32: return pick_lane_op<L, 32>(op);
    default: return nullptr;
    }
}

} // namespace b200
} // namespace warpcore

#endif /* WC_TABLES_PICK_CUH */
