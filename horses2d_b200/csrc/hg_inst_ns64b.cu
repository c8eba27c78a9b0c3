// hg_inst_ns64b.cu -- explicit instantiations: Navier-Stokes kernels, P = 4, 5, double.
#include "hg_launch.cuh"

template void launch_ns_PV<4, double, 0>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_PV<5, double, 0>(hg_ctx*, const NSArgs<double>&);
