// hg_inst_ns32b_t1.cu -- explicit instantiations: Navier-Stokes kernels, tiling variant 1, P = 4, 5, float.
#include "hg_launch.cuh"

template void launch_ns_PV<4, float, 1>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_PV<5, float, 1>(hg_ctx*, const NSArgs<float>&);
