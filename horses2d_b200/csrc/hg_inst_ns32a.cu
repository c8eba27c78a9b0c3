// hg_inst_ns32a.cu -- explicit instantiations: Navier-Stokes kernels, P = 2, 3, float.
#include "hg_launch.cuh"

template void launch_ns_P<2, float>(hg_ctx*, const NSArgs<float>&);
template void launch_ns_P<3, float>(hg_ctx*, const NSArgs<float>&);
