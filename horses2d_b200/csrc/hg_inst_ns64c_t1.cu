// hg_inst_ns64c_t1.cu -- explicit instantiations: Navier-Stokes kernels, tiling variant 1, P = 6, 7, double.
#include "hg_launch.cuh"

template void launch_ns_PV<6, double, 1>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_PV<7, double, 1>(hg_ctx*, const NSArgs<double>&);
