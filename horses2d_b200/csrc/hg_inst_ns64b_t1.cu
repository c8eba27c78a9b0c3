// hg_inst_ns64b_t1.cu -- explicit instantiations: Navier-Stokes kernels, tiling variant 1, P = 4, 5, double.
#include "hg_launch.cuh"

template void launch_ns_PV<4, double, 1>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_PV<5, double, 1>(hg_ctx*, const NSArgs<double>&);
