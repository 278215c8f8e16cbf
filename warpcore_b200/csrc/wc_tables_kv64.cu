/* bulk table kernels for the LayoutKV64 slot layout (see wc_kernels.cuh) */
#include "wc_internal.h"

namespace warpcore {
namespace b200 {

template <int W, class L = LayoutKV64>
static TableKernel pick_kv64(int op, bool fp)
{
    switch (op) {
    case kOpInsert: return fp ? fp_op_kernel<L, W, kOpInsert> : table_op_kernel<L, W, kOpInsert>;
    case kOpCount: return fp ? fp_op_kernel<L, W, kOpCount> : table_op_kernel<L, W, kOpCount>;
    case kOpRetrieve: return fp ? fp_op_kernel<L, W, kOpRetrieve> : table_op_kernel<L, W, kOpRetrieve>;
    case kOpErase: return fp ? fp_op_kernel<L, W, kOpErase> : table_op_kernel<L, W, kOpErase>;
    default: return nullptr;
    }
}

TableKernel table_kernel_kv64(int W, int op, bool fp)
{
    switch (W) {
    case 1: return pick_kv64<1>(op, fp);
    case 2: return pick_kv64<2>(op, fp);
    case 4: return pick_kv64<4>(op, fp);
    case 8: return pick_kv64<8>(op, fp);
    case 16: return pick_kv64<16>(op, fp);
    case 32: return pick_kv64<32>(op, fp);
    default: return nullptr;
    }
}

} // namespace b200
} // namespace warpcore
