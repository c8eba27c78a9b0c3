// hg_exact.cu -- face fluxes of the exact Riemann solver for one stage.
//
// The exact solver (Physics/RiemannSolvers.f90:33-187) iterates on the star pressure and calls pow
// throughout; folded into the fused stage kernels it would widen their register budget for every
// solver.  It therefore runs here, one thread per element-side node, ahead of the stage kernel: the
// arguments are exactly those the stage kernel would pass (this element's trace and the
// neighbour's, or the boundary ghost state, in LEFT-RIGHT order with LEFT's normal), taken from
// the trace buffer of the current state, and the flux goes to FX[n_el*4][P][4], which the stage
// kernel reads for every face whose solver (global, or its zone's override) is the exact one.
#include "hg_ctx.h"

namespace hg {

template <typename real>
__global__ void __launch_bounds__(128) exact_flux_kernel(int n_sides, const int* sides, int P, int affine, int riemann,
                                                         const int4* side, const real* side_geo, const Zone* zones,
                                                         const double* bq, const real* T, PhysConst pc, real* FX) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= int64_t(n_sides) * P) return;
  const int kk = int(idx % P);
  const int64_t es = sides[idx / P];   // element * 4 + side of a face that uses the exact solver
  const int4 sd = side[es];
  const int kind = sd.y & 15;
  if (kind == SIDE_WALL || kind == SIDE_FLUX) return;   // prescribed wall flux / mortar face: no Riemann problem here
  int solver = riemann;
  if (sd.z >= 0) {
    const int zr = zones[sd.z].riemann;
    if (zr >= 0) solver = zr;
  }
  if (solver != RIEMANN_EXACT) return;
  Phys<real> ph;
  ph.load(pc);
  const real* g3 = affine ? side_geo + es * 3 : side_geo + (es * P + kk) * 3;
  const real nx = g3[0], ny = g3[1];
  real qo[4], qn[4], F[4];
  const real* to = T + (es * P + kk) * 4;
#pragma unroll
  for (int k = 0; k < 4; ++k) qo[k] = to[k];
  if (kind == SIDE_STATE) {
    real us[4];
    bc_states(ph, zones[sd.z], qo, nx, ny, qn, us, sd.w >= 0 ? bq + (size_t(sd.w) * P + kk) * 4 : nullptr);
    exact(ph, qo, qn, nx, ny, F);
  } else {
    const int kn = (sd.y & SIDE_REVERSED) ? (P - 1 - kk) : kk;
    const real* tp = T + (size_t(sd.x) * P + kn) * 4;
#pragma unroll
    for (int k = 0; k < 4; ++k) qn[k] = tp[k];
    if (kind == SIDE_RIGHT) exact(ph, qn, qo, nx, ny, F);
    else exact(ph, qo, qn, nx, ny, F);
  }
  real* out = FX + (es * P + kk) * 4;
#pragma unroll
  for (int k = 0; k < 4; ++k) out[k] = F[k];
}

}  // namespace hg

// One thread per node of the element sides whose face uses the exact solver (a list built at
// hg_create: all Riemann faces when it is the interior solver, else the sides of the zones that
// select it).
template <typename real>
void launch_exact_flux(hg_ctx* c) {
  if (c->n_exact_sides == 0) return;
  const int64_t n = int64_t(c->n_exact_sides) * c->P;
  const unsigned grid = unsigned((n + 127) / 128);
  timed(c, HG_KERNEL_FACEFLUX, [&] {
    exact_flux_kernel<real><<<grid, 128, 0, c->stream>>>(
        c->n_exact_sides, c->d_exact_sides, c->P, c->affine ? 1 : 0, c->riemann, c->d_side,
        static_cast<const real*>(c->d_side_geo), c->d_zones, c->d_bq, static_cast<const real*>(c->d_T[c->cur]), c->pc,
        static_cast<real*>(c->d_FX));
  });
  ++c->launches;
}

template void launch_exact_flux<double>(hg_ctx*);
template void launch_exact_flux<float>(hg_ctx*);
