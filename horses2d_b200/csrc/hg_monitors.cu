// hg_monitors.cu -- surface integrals of a boundary zone on the device (the mesh functions behind the
// reference's surface monitors, Mesh/QuadMesh_Integrals.incf:67-346, with ComputeViscousTensor of
// Physics/ViscousFluxes.f90:416-461).
//
// They run over the traces of the state of the last residual evaluation (after a time step, the
// last stage's input state, as the reference's monitors see its edge storage) and, for the viscous
// tensor, over the gradient traces of that evaluation.  One CTA per call: each thread accumulates a
// fixed subset of the zone's side nodes, then a fixed-order tree sums the eight values, so repeated
// calls give identical results.
#include "hg_ctx.h"
#include <cfloat>

namespace hg {

constexpr int SI_THREADS = 256;

template <typename real>
__global__ void __launch_bounds__(SI_THREADS) surface_integral_kernel(int n_sides, const int* sides, int P, int affine,
                                                                      const real* side_geo, const real* T,
                                                                      const real* GT, const double* w, PhysConst pc,
                                                                      int viscous, double* out) {
  __shared__ double red[8][SI_THREADS];
  double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const double gm1 = pc.gm1, mu = pc.mu, lambda = pc.lambda;
  for (int idx = threadIdx.x; idx < n_sides * P; idx += SI_THREADS) {
    const int k = idx % P;
    const size_t es = size_t(sides[idx / P]);
    const real* g3 = affine ? side_geo + es * 3 : side_geo + (es * P + k) * 3;
    const double nx = double(g3[0]), ny = double(g3[1]), dS = double(g3[2]);
    const real* q = T + (es * P + k) * 4;
    const double Q0 = double(q[0]), Q1 = double(q[1]), Q2 = double(q[2]), Q3 = double(q[3]);
    const double wk = w[k];
    const double p = gm1 * (Q3 - 0.5 * (Q1 * Q1 + Q2 * Q2) / Q0);
    acc[0] += wk * dS;
    acc[1] += p * dS * wk;
    acc[2] += p * wk * nx * dS;
    acc[3] += p * wk * ny * dS;
    acc[6] += wk * (Q1 * nx + Q2 * ny) * dS;
    acc[7] += wk * (Q1 * nx + Q2 * ny) * dS / Q0;
    if (viscous) {
      const real* g = GT + (es * P + k) * 8;
      const double gx0 = double(g[0]), gx1 = double(g[1]), gx2 = double(g[2]);
      const double gy0 = double(g[4]), gy1 = double(g[5]), gy2 = double(g[6]);
      const double invRho = 1.0 / Q0;
      const double u = Q1 * invRho, v = Q2 * invRho;
      const double uDivRho = u * invRho, vDivRho = v * invRho;
      const double divV = -uDivRho * gx0 + invRho * gx1 - vDivRho * gy0 + invRho * gy2;
      const double txx = 2.0 * mu * (-uDivRho * gx0 + invRho * gx1) + lambda * mu * divV;
      const double tyy = 2.0 * mu * (-vDivRho * gy0 + invRho * gy2) + lambda * mu * divV;
      const double txy = -mu * vDivRho * gx0 - mu * uDivRho * gy0 + mu * invRho * gy1 + mu * invRho * gx2;
      acc[4] += wk * (txx * nx + txy * ny) * dS;
      acc[5] += wk * (txy * nx + tyy * ny) * dS;
    }
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int half = SI_THREADS / 2; half > 0; half >>= 1) {
    if (threadIdx.x < half)
#pragma unroll
      for (int c = 0; c < 8; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + half];
    __syncthreads();
  }
  if (threadIdx.x < 8) out[threadIdx.x] = red[threadIdx.x][0];
}

// Probes (Monitors.f90:740-830): the resident state at reference coordinates (xi, eta) of an element,
// BilinearForm(Q, l_xi, l_eta) = sum_i l_xi(i) sum_j Q(i,j) l_eta(j) (Generic/MatrixOperations.f90:185-209)
// with the barycentric Lagrange basis of the element's nodes (exact at the nodes).  One thread per probe.
__device__ __forceinline__ void lagrange_at(double x, int P, const double* nodes, const double* wb, double* l) {
  bool match = false;
  for (int j = 0; j < P; ++j) {
    const double a = x, b = nodes[j];
    const bool eq = (a == 0.0 || b == 0.0) ? fabs(a - b) <= 2.0 * DBL_EPSILON
                                           : fabs(b - a) <= 2.0 * DBL_EPSILON * fmax(fabs(a), fabs(b));
    l[j] = eq ? 1.0 : 0.0;
    match = match || eq;
  }
  if (match) return;
  double d = 0.0;
  for (int j = 0; j < P; ++j) { const double t = wb[j] / (x - nodes[j]); l[j] = t; d += t; }
  for (int j = 0; j < P; ++j) l[j] /= d;
}

__global__ void probe_kernel(int n, const int* elements, const double* xi_eta, const double* nodes, const double* wb,
                             int P, const double* Q, double* out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double lx[10], ly[10];
  lagrange_at(xi_eta[2 * k], P, nodes, wb, lx);
  lagrange_at(xi_eta[2 * k + 1], P, nodes, wb, ly);
  const double* q = Q + size_t(elements[k]) * P * P * 4;
  for (int v = 0; v < 4; ++v) {
    double b = 0.0;
    for (int i = 0; i < P; ++i) {
      double t = 0.0;
      for (int j = 0; j < P; ++j) t += q[(j * P + i) * 4 + v] * ly[j];
      b += lx[i] * t;
    }
    out[4 * k + v] = b;
  }
}

}  // namespace hg

void launch_probes(hg_ctx* c, int n, const int* d_elements, const double* d_xi_eta, double* d_out) {
  const int NP = c->P * c->P;
  const double* nodes = c->d_mats + 3 * NP + 7 * c->P;   // after hatD lb0 lb1 lbw0 lbw1 D dlbw0 dlbw1 w Vinv
  probe_kernel<<<(n + 127) / 128, 128, 0, c->stream>>>(n, d_elements, d_xi_eta, nodes, nodes + c->P, c->P, c->d_Q,
                                                      d_out);
  ++c->launches;
}

template <typename real>
void launch_surface_integrals(hg_ctx* c, int zone, double* d_out) {
  const int z = zone - 1;
  const int n_sides = int(c->zone_sides[z].size());
  const int NP = c->P * c->P;
  const double* w = c->d_mats + 2 * NP + 6 * c->P;   // hatD lb0 lb1 lbw0 lbw1 D dlbw0 dlbw1 w Vinv
  const int viscous = (c->ns && c->pc.mu != 0.0 && c->d_GT[c->last_T]) ? 1 : 0;
  surface_integral_kernel<real><<<1, SI_THREADS, 0, c->stream>>>(
      n_sides, c->d_zone_sides[z], c->P, c->affine ? 1 : 0, static_cast<const real*>(c->d_side_geo),
      static_cast<const real*>(c->d_T[c->last_T]), static_cast<const real*>(c->d_GT[c->last_T]), w, c->pc, viscous, d_out);
  ++c->launches;
}

template void launch_surface_integrals<double>(hg_ctx*, int, double*);
template void launch_surface_integrals<float>(hg_ctx*, int, double*);
