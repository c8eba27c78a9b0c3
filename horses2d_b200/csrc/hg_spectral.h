// hg_spectral.h -- host-side nodal operators for one polynomial order.
//
// Definitions match the reference's NodesAndWeights_t
// (Approximation/NodesAndWeightsClass.f90:251-332): Legendre-Gauss or
// Legendre-Gauss-Lobatto nodes mapped to [0,1] with weights halved, the
// barycentric derivative matrix D (Spectral/InterpolationAndDerivatives.f90:440-475),
// hatD = M^-1 (M D)^T, boundary interpolants lb at 0 and 1 and lbw = lb / w.
// Roots are found by Newton's method on the Legendre recurrence
// (Kopriva, "Implementing Spectral Methods for PDEs", Alg. 23-25).
#pragma once
#include <vector>

namespace hg {

struct NodalOps {
  int N = 0, P = 0;
  std::vector<double> xi, w, wb, D, hatD, lb0, lb1, lbw0, lbw1, dlbw0, dlbw1;
  // nodal -> modal transform: Vinv = V^-1 with V(i,k) = sqrt(2k+1) L_k(2 xi_i - 1), the orthonormal
  // Legendre basis on [0,1]; modal coefficients u_hat(k) = sum_i Vinv(k,i) u(xi_i)   [k*P+i]
  std::vector<double> Vinv;
};

NodalOps make_nodal_ops(int N, int node_type);   // node_type: 1 LG, 2 LGL
std::vector<double> lagrange_basis(const NodalOps& ops, double x);

}  // namespace hg
