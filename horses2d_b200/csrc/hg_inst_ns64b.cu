// hg_inst_ns64b.cu -- explicit instantiations: Navier-Stokes kernels, P = 4, 5, double.
#include "hg_launch.cuh"

template void launch_ns_P<4, double>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_P<5, double>(hg_ctx*, const NSArgs<double>&);
