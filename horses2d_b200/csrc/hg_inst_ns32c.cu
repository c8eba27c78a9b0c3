// hg_inst_ns32c.cu -- explicit instantiations: Navier-Stokes kernels, P = 6, 7, float.
// Compiled with approximate FP32 quotients and square roots (FP32_FLAGS in build.py).
#include "hg_launch.cuh"

template void launch_ns_PV<6, float, 0>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_PV<7, float, 0>(hg_ctx*, const NSArgs<float>&);
