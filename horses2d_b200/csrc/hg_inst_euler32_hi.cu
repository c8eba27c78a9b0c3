// hg_inst_euler32_hi.cu -- explicit instantiations: Euler stage and trace kernels, orders 9-12 (the
// high orders of p-refined meshes), FP32.
// Compiled with approximate FP32 quotients and square roots (FP32_FLAGS in build.py).
#include "hg_launch.cuh"

template void launch_stage_PV<10, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<10, float>(hg_ctx*);
template void launch_stage_PV<11, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<11, float>(hg_ctx*);
template void launch_stage_PV<12, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<12, float>(hg_ctx*);
template void launch_stage_PV<13, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<13, float>(hg_ctx*);
