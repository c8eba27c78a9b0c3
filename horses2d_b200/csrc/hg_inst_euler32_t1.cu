// hg_inst_euler32_t1.cu -- explicit instantiations: Euler stage kernels, tiling variant 1 (small CTAs),
// orders 1-8, FP32.
// Compiled with approximate FP32 quotients and square roots (FP32_FLAGS in build.py).
#include "hg_launch.cuh"

template void launch_stage_PV<2, float, 1>(hg_ctx*, const StageArgs<float>&);
template void launch_stage_PV<3, float, 1>(hg_ctx*, const StageArgs<float>&);
template void launch_stage_PV<4, float, 1>(hg_ctx*, const StageArgs<float>&);
template void launch_stage_PV<5, float, 1>(hg_ctx*, const StageArgs<float>&);
template void launch_stage_PV<6, float, 1>(hg_ctx*, const StageArgs<float>&);
template void launch_stage_PV<7, float, 1>(hg_ctx*, const StageArgs<float>&);
template void launch_stage_PV<8, float, 1>(hg_ctx*, const StageArgs<float>&);
template void launch_stage_PV<9, float, 1>(hg_ctx*, const StageArgs<float>&);
