// hg_inst_ns32b.cu -- explicit instantiations: Navier-Stokes kernels, P = 4, 5, float.
#include "hg_launch.cuh"

template void launch_ns_P<4, float>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_P<5, float>(hg_ctx*, const NSArgs<float>&);
