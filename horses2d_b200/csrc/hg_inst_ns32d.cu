// hg_inst_ns32d.cu -- explicit instantiations: Navier-Stokes kernels, P = 8, 9, float.
// Compiled with approximate FP32 quotients and square roots (FP32_FLAGS in build.py).
#include "hg_launch.cuh"

template void launch_ns_PV<8, float, 0>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_PV<9, float, 0>(hg_ctx*, const NSArgs<float>&);
