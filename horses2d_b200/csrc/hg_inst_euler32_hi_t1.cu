// hg_inst_euler32_hi_t1.cu -- explicit instantiations: Euler stage kernels, tiling variant 1 (one
// element per CTA), orders 9-12, FP32.
// Compiled with approximate FP32 quotients and square roots (FP32_FLAGS in build.py).
#include "hg_launch.cuh"

template void launch_stage_PV<10, float, 1>(hg_ctx*, const StageArgs<float>&);
template void launch_stage_PV<11, float, 1>(hg_ctx*, const StageArgs<float>&);
template void launch_stage_PV<12, float, 1>(hg_ctx*, const StageArgs<float>&);
template void launch_stage_PV<13, float, 1>(hg_ctx*, const StageArgs<float>&);
