// hg_inst_ns32b_t1.cu -- explicit instantiations: Navier-Stokes kernels, tiling variant 1, P = 4, 5, float.
// Compiled with approximate FP32 quotients and square roots (FP32_FLAGS in build.py).
#include "hg_launch.cuh"

template void launch_ns_PV<4, float, 1>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_PV<5, float, 1>(hg_ctx*, const NSArgs<float>&);
