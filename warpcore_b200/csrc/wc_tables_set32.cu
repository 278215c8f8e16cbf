/* bulk table kernels for the LayoutSet32 slot layout (see wc_kernels.cuh) */
#include "wc_internal.h"

namespace warpcore {
namespace b200 {

template <int W, class L = LayoutSet32>
static TableKernel pick_set32(int op, bool fp)
{
    switch (op) {
    case kOpInsert: return fp ? fp_op_kernel<L, W, kOpInsert> : table_op_kernel<L, W, kOpInsert>;
    case kOpRetrieve: return fp ? fp_op_kernel<L, W, kOpRetrieve> : table_op_kernel<L, W, kOpRetrieve>;
    case kOpErase: return fp ? fp_op_kernel<L, W, kOpErase> : table_op_kernel<L, W, kOpErase>;
    default: return nullptr;
    }
}

TableKernel table_kernel_set32(int W, int op, bool fp)
{
    switch (W) {
    case 1: return pick_set32<1>(op, fp);
    case 2: return pick_set32<2>(op, fp);
    case 4: return pick_set32<4>(op, fp);
    case 8: return pick_set32<8>(op, fp);
    case 16: return pick_set32<16>(op, fp);
    case 32: return pick_set32<32>(op, fp);
    default: return nullptr;
    }
}

} // namespace b200
} // namespace warpcore
