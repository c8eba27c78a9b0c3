// hg_inst_ns64d.cu -- explicit instantiations: Navier-Stokes kernels, P = 8, 9, double.
#include "hg_launch.cuh"

template void launch_ns_PV<8, double, 0>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_PV<9, double, 0>(hg_ctx*, const NSArgs<double>&);
