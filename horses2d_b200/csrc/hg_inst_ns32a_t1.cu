// hg_inst_ns32a_t1.cu -- explicit instantiations: Navier-Stokes kernels, tiling variant 1, P = 2, 3, float.
// Compiled with approximate FP32 quotients and square roots (FP32_FLAGS in build.py).
#include "hg_launch.cuh"

template void launch_ns_PV<2, float, 1>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_PV<3, float, 1>(hg_ctx*, const NSArgs<float>&);
