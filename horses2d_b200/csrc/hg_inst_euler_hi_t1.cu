// hg_inst_euler_hi_t1.cu -- explicit instantiations: Euler stage kernels, tiling variant 1 (one
// element per CTA), orders 9-12, FP64.
#include "hg_launch.cuh"

template void launch_stage_PV<10, double, 1>(hg_ctx*, const StageArgs<double>&);
template void launch_stage_PV<11, double, 1>(hg_ctx*, const StageArgs<double>&);
template void launch_stage_PV<12, double, 1>(hg_ctx*, const StageArgs<double>&);
template void launch_stage_PV<13, double, 1>(hg_ctx*, const StageArgs<double>&);
