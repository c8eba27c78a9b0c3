// hg_inst_euler.cu -- explicit instantiations: Euler stage and trace kernels, orders 1-8, FP64.
#include "hg_launch.cuh"

template void launch_stage_PV<2, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<2, double>(hg_ctx*);
template void launch_stage_PV<3, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<3, double>(hg_ctx*);
template void launch_stage_PV<4, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<4, double>(hg_ctx*);
template void launch_stage_PV<5, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<5, double>(hg_ctx*);
template void launch_stage_PV<6, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<6, double>(hg_ctx*);
template void launch_stage_PV<7, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<7, double>(hg_ctx*);
template void launch_stage_PV<8, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<8, double>(hg_ctx*);
template void launch_stage_PV<9, double, 0>(hg_ctx*, const StageArgs<double>&);
template void launch_trace_P<9, double>(hg_ctx*);
