// hg_inst_ns64a_t1.cu -- explicit instantiations: Navier-Stokes kernels, tiling variant 1, P = 2, 3, double.
#include "hg_launch.cuh"

template void launch_ns_PV<2, double, 1>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_PV<3, double, 1>(hg_ctx*, const NSArgs<double>&);
