// hg_inst_ns64c.cu -- explicit instantiations: Navier-Stokes kernels, P = 6, 7, double.
#include "hg_launch.cuh"

template void launch_ns_PV<6, double, 0>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_PV<7, double, 0>(hg_ctx*, const NSArgs<double>&);
