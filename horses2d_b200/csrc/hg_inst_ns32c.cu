// hg_inst_ns32c.cu -- explicit instantiations: Navier-Stokes kernels, P = 6, 7, float.
#include "hg_launch.cuh"

template void launch_ns_P<6, float>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_P<7, float>(hg_ctx*, const NSArgs<float>&);
