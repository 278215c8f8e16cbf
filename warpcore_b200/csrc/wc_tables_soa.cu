/* bulk table kernels for single-value tables stored as a struct of arrays
 * (LayoutSoA; SoAStore, storage.cuh:218-432): the key array is probed like a
 * hash set's slot array by table_op_kernel, which writes and reads values
 * in the separate value array at the slot index.  No fingerprint or
 * one-key-per-lane variants: those tables use the window kernel only. */
#include "wc_tables_pick.cuh"

namespace warpcore {
namespace b200 {

namespace {

template <class L, int W>
TableKernel pick_soa_op(int op)
{
    switch (op) {
    case kOpInsert: return table_op_kernel<L, W, kOpInsert>;
    case kOpRetrieve: return table_op_kernel<L, W, kOpRetrieve>;
    case kOpErase: return table_op_kernel<L, W, kOpErase>;
    default: return nullptr;
    }
}

template <class L>
TableKernel pick_soa_for(int W, int op)
{
    switch (W) {
    case 1: return pick_soa_op<L, 1>(op);
    case 2: return pick_soa_op<L, 2>(op);
    case 4: return pick_soa_op<L, 4>(op);
    case 8: return pick_soa_op<L, 8>(op);
    case 16: return pick_soa_op<L, 16>(op);
    case 32: return pick_soa_op<L, 32>(op);
    default: return nullptr;
    }
}

/* every valid (key, value) of the key array and the value array, compacted
 * by block tiles as dump_kernel does (compact_tiles); both arrays are streamed */
template <class K, class V>
__global__ void __launch_bounds__(256) soa_dump_kernel(const void *keys, const void *values,
                                                       uint64_t capacity, uint64_t empty,
                                                       uint64_t tomb, void *keys_out,
                                                       void *values_out,
                                                       unsigned long long *count)
{
    const K *const kin = reinterpret_cast<const K *>(keys);
    const V *const vin = reinterpret_cast<const V *>(values);
    const bool want_values = values_out != nullptr;
    compact_tiles<K, V>(capacity, reinterpret_cast<K *>(keys_out),
                        reinterpret_cast<V *>(values_out), count, [&](uint64_t s, K &k, V &v) {
                            k = kin[s];
                            if (want_values) v = vin[s];
                            return k != K(empty) && k != K(tomb);
                        });
}

} // namespace

TableKernel table_kernel_soa(uint32_t key_bytes, uint32_t value_bytes, int W, int op)
{
    if (key_bytes == 4 && value_bytes == 4) return pick_soa_for<LayoutSoA<uint32_t, uint32_t>>(W, op);
    if (key_bytes == 8 && value_bytes == 8) return pick_soa_for<LayoutSoA<uint64_t, uint64_t>>(W, op);
    if (key_bytes == 4 && value_bytes == 8) return pick_soa_for<LayoutSoA<uint32_t, uint64_t>>(W, op);
    if (key_bytes == 8 && value_bytes == 4) return pick_soa_for<LayoutSoA<uint64_t, uint32_t>>(W, op);
    return nullptr;
}

SoaDumpKernel soa_dump_kernel_ptr(uint32_t key_bytes, uint32_t value_bytes)
{
    if (key_bytes == 4 && value_bytes == 4) return soa_dump_kernel<uint32_t, uint32_t>;
    if (key_bytes == 8 && value_bytes == 8) return soa_dump_kernel<uint64_t, uint64_t>;
    if (key_bytes == 4 && value_bytes == 8) return soa_dump_kernel<uint32_t, uint64_t>;
    if (key_bytes == 8 && value_bytes == 4) return soa_dump_kernel<uint64_t, uint32_t>;
    return nullptr;
}

} // namespace b200
} // namespace warpcore
