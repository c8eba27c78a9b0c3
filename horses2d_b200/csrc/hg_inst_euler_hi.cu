// hg_inst_euler_hi.cu -- explicit instantiations: Euler stage and trace kernels, orders 9-12 (the
// high orders of p-refined meshes), FP64.
#include "hg_launch.cuh"

template void launch_stage_PV<10, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<10, double>(hg_ctx*);
template void launch_stage_PV<11, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<11, double>(hg_ctx*);
template void launch_stage_PV<12, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<12, double>(hg_ctx*);
template void launch_stage_PV<13, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<13, double>(hg_ctx*);
