/* multi-table batch kernels (see wc_batch.cuh) */
#include "wc_internal.h"

namespace warpcore {
namespace b200 {

template <class L>
static const void *pick_batch(int W, bool inl)
{
#define WC_PICK(w)                                                                            \
    case w:                                                                                   \
        return inl ? reinterpret_cast<const void *>(batch_op_kernel_inline<L, w>)             \
                   : reinterpret_cast<const void *>(batch_op_kernel<L, w>);
    switch (W) {
        WC_PICK(1)
        WC_PICK(2)
        WC_PICK(4)
        WC_PICK(8)
        WC_PICK(16)
        WC_PICK(32)
    default: return nullptr;
    }
#undef WC_PICK
}

const void *batch_kernel_ptr(int layout, int W, bool inline_desc)
{
    if (layout == kLayoutKV32) return pick_batch<LayoutKV32>(W, inline_desc);
    if (layout == kLayoutKV64) return pick_batch<LayoutKV64>(W, inline_desc);
    return nullptr;
}

} // namespace b200
} // namespace warpcore
