// hg_inst_ns64d_t1.cu -- explicit instantiations: Navier-Stokes kernels, tiling variant 1, P = 8, 9, double.
#include "hg_launch.cuh"

template void launch_ns_PV<8, double, 1>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_PV<9, double, 1>(hg_ctx*, const NSArgs<double>&);
