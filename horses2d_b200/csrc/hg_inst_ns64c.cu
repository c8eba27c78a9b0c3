// hg_inst_ns64c.cu -- explicit instantiations: Navier-Stokes kernels, P = 6, 7, double.
#include "hg_launch.cuh"

template void launch_ns_P<6, double>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_P<7, double>(hg_ctx*, const NSArgs<double>&);
