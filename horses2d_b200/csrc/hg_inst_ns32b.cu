// hg_inst_ns32b.cu -- explicit instantiations: Navier-Stokes kernels, P = 4, 5, float.
// Compiled with approximate FP32 quotients and square roots (FP32_FLAGS in build.py).
#include "hg_launch.cuh"

template void launch_ns_PV<4, float, 0>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_PV<5, float, 0>(hg_ctx*, const NSArgs<float>&);
