// hg_inst_euler32.cu -- explicit instantiations: Euler stage and trace kernels, orders 1-8, FP32.
// Compiled with approximate FP32 quotients and square roots (FP32_FLAGS in build.py).
#include "hg_launch.cuh"

template void launch_stage_PV<2, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<2, float>(hg_ctx*);
template void launch_stage_PV<3, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<3, float>(hg_ctx*);
template void launch_stage_PV<4, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<4, float>(hg_ctx*);
template void launch_stage_PV<5, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<5, float>(hg_ctx*);
template void launch_stage_PV<6, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<6, float>(hg_ctx*);
template void launch_stage_PV<7, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<7, float>(hg_ctx*);
template void launch_stage_PV<8, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<8, float>(hg_ctx*);
template void launch_stage_PV<9, float, 0>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<9, float>(hg_ctx*);
