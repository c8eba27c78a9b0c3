// hg_inst_ns32d_t1.cu -- explicit instantiations: Navier-Stokes kernels, tiling variant 1, P = 8, 9, float.
// Compiled with approximate FP32 quotients and square roots (FP32_FLAGS in build.py).
#include "hg_launch.cuh"

template void launch_ns_PV<8, float, 1>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_PV<9, float, 1>(hg_ctx*, const NSArgs<float>&);
