/* bulk table kernels for the LayoutSet64 slot layout (see wc_kernels.cuh) */
#include "wc_internal.h"

namespace warpcore {
namespace b200 {

template <int W, class L = LayoutSet64>
static TableKernel pick_set64(int op)
{
    switch (op) {
    case kOpInsert: return table_op_kernel<L, W, kOpInsert>;
    case kOpRetrieve: return table_op_kernel<L, W, kOpRetrieve>;
    case kOpErase: return table_op_kernel<L, W, kOpErase>;
    default: return nullptr;
    }
}

TableKernel table_kernel_set64(int W, int op)
{
    switch (W) {
    case 1: return pick_set64<1>(op);
    case 2: return pick_set64<2>(op);
    case 4: return pick_set64<4>(op);
    case 8: return pick_set64<8>(op);
    case 16: return pick_set64<16>(op);
    case 32: return pick_set64<32>(op);
    default: return nullptr;
    }
}

} // namespace b200
} // namespace warpcore
