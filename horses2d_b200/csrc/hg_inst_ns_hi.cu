// hg_inst_ns_hi.cu -- explicit instantiations: Navier-Stokes kernels, P = 10, 11 (orders 9, 10 of
// p-refined meshes; one element per CTA in both tilings), double.
#include "hg_launch.cuh"

template void launch_ns_PV<10, double, 0>(hg_ctx*, const NSArgs<double>&);
template void launch_ns_PV<11, double, 0>(hg_ctx*, const NSArgs<double>&);
