// hg_inst_euler.cu -- explicit instantiations: Euler stage and trace kernels, orders 1-8, FP64 and FP32.
#include "hg_launch.cuh"

template void launch_stage_P<2, double>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<2, double>(hg_ctx*);
template void launch_stage_P<3, double>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<3, double>(hg_ctx*);
template void launch_stage_P<4, double>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<4, double>(hg_ctx*);
template void launch_stage_P<5, double>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<5, double>(hg_ctx*);
template void launch_stage_P<6, double>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<6, double>(hg_ctx*);
template void launch_stage_P<7, double>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<7, double>(hg_ctx*);
template void launch_stage_P<8, double>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<8, double>(hg_ctx*);
template void launch_stage_P<9, double>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<9, double>(hg_ctx*);
template void launch_stage_P<2, float>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<2, float>(hg_ctx*);
template void launch_stage_P<3, float>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<3, float>(hg_ctx*);
template void launch_stage_P<4, float>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<4, float>(hg_ctx*);
template void launch_stage_P<5, float>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<5, float>(hg_ctx*);
template void launch_stage_P<6, float>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<6, float>(hg_ctx*);
template void launch_stage_P<7, float>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<7, float>(hg_ctx*);
template void launch_stage_P<8, float>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<8, float>(hg_ctx*);
template void launch_stage_P<9, float>(hg_ctx*, const StageArgs<float>&);
template void launch_trace_P<9, float>(hg_ctx*);
