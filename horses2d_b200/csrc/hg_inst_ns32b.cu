// hg_inst_ns32b.cu -- explicit instantiations: Navier-Stokes kernels, P = 4, 5, float.
#include "hg_launch.cuh"

template void launch_ns_PV<4, float, 0>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_PV<5, float, 0>(hg_ctx*, const NSArgs<float>&);
