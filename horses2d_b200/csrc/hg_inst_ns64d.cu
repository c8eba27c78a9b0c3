// hg_inst_ns64d.cu -- explicit instantiations: Navier-Stokes kernels, P = 8, 9, double.
#include "hg_launch.cuh"

template void launch_ns_P<8, double>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_P<9, double>(hg_ctx*, const NSArgs<double>&);
