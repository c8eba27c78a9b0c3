// hg_inst_sensor.cu -- explicit instantiations: sensor evaluation kernels, orders 1-8, FP64 and FP32.
#include "hg_launch.cuh"

template void launch_sensor_eval_P<2, double>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<3, double>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<4, double>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<5, double>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<6, double>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<7, double>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<8, double>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<9, double>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<2, float>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<3, float>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<4, float>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<5, float>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<6, float>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<7, float>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<8, float>(hg_ctx*, float*, double*);
template void launch_sensor_eval_P<9, float>(hg_ctx*, float*, double*);
