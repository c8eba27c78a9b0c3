// hg_inst_ns32_hi.cu -- explicit instantiations: Navier-Stokes kernels, P = 10, 11 (orders 9, 10 of
// p-refined meshes; one element per CTA in both tilings), float.
// Compiled with approximate FP32 quotients and square roots (FP32_FLAGS in build.py).
#include "hg_launch.cuh"

template void launch_ns_PV<10, float, 0>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_PV<11, float, 0>(hg_ctx*, const NSArgs<float>&);
