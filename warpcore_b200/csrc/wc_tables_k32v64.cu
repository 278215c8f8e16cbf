/* bulk table kernels for the LayoutK32V64 slot layout (see wc_kernels.cuh) */
#include "wc_tables_pick.cuh"

namespace warpcore {
namespace b200 {

TableKernel table_kernel_k32v64(int W, int op, bool fp) { return pick_table_kernel_for<LayoutK32V64>(W, op, fp); }
TableKernel lane_kernel_k32v64(int W, int op) { return pick_lane_kernel_for<LayoutK32V64>(W, op); }

} // namespace b200
} // namespace warpcore
