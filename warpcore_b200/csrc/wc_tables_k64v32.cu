/* bulk table kernels for the LayoutK64V32 slot layout (see wc_kernels.cuh) */
#include "wc_tables_pick.cuh"

namespace warpcore {
namespace b200 {

TableKernel table_kernel_k64v32(int W, int op, bool fp) { return pick_table_kernel_for<LayoutK64V32>(W, op, fp); }
TableKernel lane_kernel_k64v32(int W, int op) { return pick_lane_kernel_for<LayoutK64V32>(W, op); }

} // namespace b200
} // namespace warpcore
