/* bulk table kernels for the LayoutKV64 slot layout (see wc_kernels.cuh) */
#include "wc_internal.h"

namespace warpcore {
namespace b200 {

template <int W, class L = LayoutKV64>
static TableKernel pick_kv64(int op)
{
    switch (op) {
    case kOpInsert: return table_op_kernel<L, W, kOpInsert>;
    case kOpCount: return table_op_kernel<L, W, kOpCount>;
    case kOpRetrieve: return table_op_kernel<L, W, kOpRetrieve>;
    case kOpErase: return table_op_kernel<L, W, kOpErase>;
    default: return nullptr;
    }
}

TableKernel table_kernel_kv64(int W, int op)
{
    switch (W) {
    case 1: return pick_kv64<1>(op);
    case 2: return pick_kv64<2>(op);
    case 4: return pick_kv64<4>(op);
    case 8: return pick_kv64<8>(op);
    case 16: return pick_kv64<16>(op);
    case 32: return pick_kv64<32>(op);
    default: return nullptr;
    }
}

} // namespace b200
} // namespace warpcore
