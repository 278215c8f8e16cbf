/* bulk table kernels for the LayoutKV32 slot layout (see wc_kernels.cuh) */
#include "wc_internal.h"

namespace warpcore {
namespace b200 {

template <int W, class L = LayoutKV32>
static TableKernel pick_kv32(int op)
{
    switch (op) {
    case kOpInsert: return table_op_kernel<L, W, kOpInsert>;
    case kOpCount: return table_op_kernel<L, W, kOpCount>;
    case kOpRetrieve: return table_op_kernel<L, W, kOpRetrieve>;
    case kOpErase: return table_op_kernel<L, W, kOpErase>;
    default: return nullptr;
    }
}

TableKernel table_kernel_kv32(int W, int op)
{
    switch (W) {
    case 1: return pick_kv32<1>(op);
    case 2: return pick_kv32<2>(op);
    case 4: return pick_kv32<4>(op);
    case 8: return pick_kv32<8>(op);
    case 16: return pick_kv32<16>(op);
    case 32: return pick_kv32<32>(op);
    default: return nullptr;
    }
}

} // namespace b200
} // namespace warpcore
