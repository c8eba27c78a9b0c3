// hg_inst_euler_t1.cu -- explicit instantiations: Euler stage kernels, tiling variant 1 (small CTAs),
// orders 1-8, FP64.
#include "hg_launch.cuh"

template void launch_stage_PV<2, double, 1>(hg_ctx*, const StageArgs<double>&);
template void launch_stage_PV<3, double, 1>(hg_ctx*, const StageArgs<double>&);
template void launch_stage_PV<4, double, 1>(hg_ctx*, const StageArgs<double>&);
template void launch_stage_PV<5, double, 1>(hg_ctx*, const StageArgs<double>&);
template void launch_stage_PV<6, double, 1>(hg_ctx*, const StageArgs<double>&);
template void launch_stage_PV<7, double, 1>(hg_ctx*, const StageArgs<double>&);
template void launch_stage_PV<8, double, 1>(hg_ctx*, const StageArgs<double>&);
template void launch_stage_PV<9, double, 1>(hg_ctx*, const StageArgs<double>&);
