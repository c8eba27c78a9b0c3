// hg_inst_ns64a.cu -- explicit instantiations: Navier-Stokes kernels, P = 2, 3, double.
#include "hg_launch.cuh"

template void launch_ns_PV<2, double, 0>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_PV<3, double, 0>(hg_ctx*, const NSArgs<double>&);
