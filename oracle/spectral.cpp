/*
 * spectral.cpp -- nodes, weights and matrices of the oracle (TEST INFRASTRUCTURE).
 *
 * Restates:
 *   GaussLegendreNodesAndWeights          Spectral/LegendreAlgorithms.f90:106-175
 *   LegendreGaussLobattoNodesAndWeights   Spectral/LegendreAlgorithms.f90:185-256
 *   BarycentricWeights / PolynomialDerivativeMatrix / PolynomialInterpolationMatrix /
 *   LagrangeInterpolatingPolynomialBarycentric   Spectral/InterpolationAndDerivatives.f90
 *   computeNodesAndWeights (nodes mapped to [0,1], hatD = M^-1 (M D)^T, lb, lbw, dlb, dlbw)
 *                                          Approximation/NodesAndWeightsClass.f90:251-332
 *   AlmostEqual                            Generic/Utilities.f90:37-64
 */
#include "oracle_internal.h"
#include <cfloat>
#include <cstdlib>

namespace orc {

bool almost_equal(double a, double b) {
  const double eps = DBL_EPSILON;
  if (a == 0.0 || b == 0.0) return std::fabs(a - b) <= 2.0 * eps;
  return std::fabs(b - a) <= 2.0 * eps * std::fmax(std::fabs(a), std::fabs(b));
}

static void legendre_poly_and_derivative(int N, double x, double& L, double& Lp) {
  if (N == 0) { L = 1.0; Lp = 0.0; return; }
  if (N == 1) { L = x; Lp = 1.0; return; }
  double Lm2 = 1.0, Lpm2 = 0.0, Lm1 = x, Lpm1 = 1.0;
  for (int k = 2; k <= N; ++k) {
    L = ((2.0 * k - 1.0) * x * Lm1 - (k - 1.0) * Lm2) / k;
    Lp = Lpm2 + (2.0 * k - 1.0) * Lm1;
    Lm2 = Lm1; Lm1 = L; Lpm2 = Lpm1; Lpm1 = Lp;
  }
}

void legendre_gauss(int N, double* x, double* w) {
  const double tol = 4.0 * DBL_EPSILON;
  double L, Lp;
  if (N == 0) { x[0] = 0.0; w[0] = 2.0; return; }
  if (N == 1) {
    x[0] = -std::sqrt(1.0 / 3.0); w[0] = 1.0; x[1] = -x[0]; w[1] = w[0];
  } else {
    const int half = (N + 1) / 2;
    for (int j = 0; j < half; ++j) {
      double xj = -std::cos((2 * j + 1) * PI / (2 * N + 2));
      for (int k = 0; k <= 100; ++k) {
        legendre_poly_and_derivative(N + 1, xj, L, Lp);
        const double delta = -L / Lp;
        xj += delta;
        if (std::fabs(delta) <= tol * std::fabs(xj)) break;
      }
      legendre_poly_and_derivative(N + 1, xj, L, Lp);
      x[j] = xj;
      w[j] = 2.0 / ((1.0 - xj * xj) * Lp * Lp);
      x[N - j] = -xj;
      w[N - j] = w[j];
    }
  }
  if (N % 2 == 0) {
    legendre_poly_and_derivative(N + 1, 0.0, L, Lp);
    x[N / 2] = 0.0;
    w[N / 2] = 2.0 / (Lp * Lp);
  }
}

// q = L_{N+1} - L_{N-1} and its derivative, plus L_N (qAndLEvaluation)
static void q_and_L(int N, double x, double& q, double& dq, double& LN) {
  double Lm2 = 1.0, Lm1 = x, dLm2 = 0.0, dLm1 = 1.0, dLN = 0.0;
  LN = 0.0;
  for (int k = 2; k <= N; ++k) {
    LN = (2.0 * k - 1.0) * x * Lm1 / k - (1.0 * k - 1.0) * Lm2 / k;
    dLN = dLm2 + (2.0 * k - 1.0) * Lm1;
    Lm2 = Lm1; Lm1 = LN; dLm2 = dLm1; dLm1 = dLN;
  }
  const int k = N + 1;
  const double Lp1 = (2.0 * k - 1.0) * x * LN / k - (1.0 * k - 1.0) * Lm2 / k;
  const double dLp1 = dLm2 + (2.0 * k - 1.0) * LN;
  q = Lp1 - Lm2;
  dq = dLp1 - dLm2;
}

void legendre_gauss_lobatto(int N, double* x, double* w) {
  const double pi = std::acos(-1.0), tol = 1e-10;
  double q, dq, LN;
  if (N == 1) { x[0] = -1; x[1] = 1; w[0] = 1; w[1] = 1; return; }
  x[0] = -1.0; w[0] = 2.0 / (1.0 * N * (1.0 * N + 1.0)); x[N] = 1.0; w[N] = w[0];
  for (int j = 1; j <= (N + 1) / 2 - 1; ++j) {
    x[j] = -std::cos((j + 0.25) * pi / N - 3.0 / (8.0 * N * pi * (j + 0.25)));
    for (int k = 0; k <= 10; ++k) {
      q_and_L(N, x[j], q, dq, LN);
      const double delta = -q / dq;
      x[j] += delta;
      if (std::fabs(delta) < tol * std::fabs(x[j])) break;
    }
    q_and_L(N, x[j], q, dq, LN);
    x[N - j] = -x[j];
    w[j] = 2.0 / (1.0 * N * (N + 1.0) * LN * LN);
    w[N - j] = w[j];
  }
  if (N % 2 == 0) {
    q_and_L(N, 0.0, q, dq, LN);
    x[N / 2] = 0.0;
    w[N / 2] = 2.0 / (1.0 * N * (N + 1.0) * LN * LN);
  }
}

void barycentric_weights(int N, const double* x, double* w) {
  for (int j = 0; j <= N; ++j) w[j] = 1.0;
  for (int j = 1; j <= N; ++j)
    for (int k = 0; k <= j - 1; ++k) {
      w[k] = w[k] * (x[k] - x[j]);
      w[j] = w[j] * (x[j] - x[k]);
    }
  for (int j = 0; j <= N; ++j) w[j] = 1.0 / w[j];
}

// T: (M+1) x (N+1), row-major [k*(N+1)+j]
void interp_matrix(int N, int M, const double* oldNodes, const double* wb, const double* newNodes, double* T) {
  for (int k = 0; k <= M; ++k) {
    bool match = false;
    for (int j = 0; j <= N; ++j) {
      T[k * (N + 1) + j] = 0.0;
      if (almost_equal(newNodes[k], oldNodes[j])) { match = true; T[k * (N + 1) + j] = 1.0; }
    }
    if (!match) {
      double s = 0.0;
      for (int j = 0; j <= N; ++j) {
        const double t = wb[j] / (newNodes[k] - oldNodes[j]);
        T[k * (N + 1) + j] = t;
        s += t;
      }
      for (int j = 0; j <= N; ++j) T[k * (N + 1) + j] /= s;
    }
  }
}

static void lagrange_barycentric(double x, int N, const double* nodes, const double* wb, double* p) {
  bool match = false;
  for (int j = 0; j <= N; ++j) {
    p[j] = 0.0;
    if (almost_equal(x, nodes[j])) { p[j] = 1.0; match = true; }
  }
  if (match) return;
  double d = 0.0;
  for (int j = 0; j <= N; ++j) { const double t = wb[j] / (x - nodes[j]); p[j] = t; d += t; }
  for (int j = 0; j <= N; ++j) p[j] /= d;
}

std::vector<double> Spectral::lj(double x) const {
  std::vector<double> v(P);
  lagrange_barycentric(x, N, xi.data(), wb.data(), v.data());
  return v;
}

void build_spectral(Spectral& s, int N, int nodes) {
  s.N = N; s.P = N + 1; s.nodes = nodes;
  const int P = N + 1;
  s.xi.assign(P, 0); s.w.assign(P, 0); s.wb.assign(P, 0);
  if (nodes == OR_NODES_LG) legendre_gauss(N, s.xi.data(), s.w.data());
  else legendre_gauss_lobatto(N, s.xi.data(), s.w.data());
  for (int i = 0; i < P; ++i) { s.xi[i] = 0.5 + 0.5 * s.xi[i]; s.w[i] = 0.5 * s.w[i]; }
  barycentric_weights(N, s.xi.data(), s.wb.data());
  // D(i,j) = wb(j) / (wb(i) (x_i - x_j)), D(i,i) = -sum   (PolynomialDerivativeMatrix)
  std::vector<double> bw(P);
  barycentric_weights(N, s.xi.data(), bw.data());
  s.D.assign(P * P, 0.0);
  for (int i = 0; i < P; ++i) {
    s.D[i * P + i] = 0.0;
    for (int j = 0; j < P; ++j)
      if (j != i) {
        s.D[i * P + j] = bw[j] / (bw[i] * (s.xi[i] - s.xi[j]));
        s.D[i * P + i] = s.D[i * P + i] - s.D[i * P + j];
      }
  }
  // MD = M D; trMD = (MD)^T; hatD = Minv trMD  -> hatD(i,l) = (1/w_i) * (w_l * D(l,i))
  s.hatD.assign(P * P, 0.0);
  for (int i = 0; i < P; ++i)
    for (int l = 0; l < P; ++l) s.hatD[i * P + l] = (1.0 / s.w[i]) * (s.w[l] * s.D[l * P + i]);
  for (int side = 0; side < 2; ++side) {
    s.lb[side].assign(P, 0); s.lbw[side].assign(P, 0); s.dlb[side].assign(P, 0); s.dlbw[side].assign(P, 0);
    lagrange_barycentric(side == 0 ? 0.0 : 1.0, N, s.xi.data(), s.wb.data(), s.lb[side].data());
    for (int i = 0; i < P; ++i) s.lbw[side][i] = s.lb[side][i] / s.w[i];
    // dlb = DT * lb  ->  dlb(i) = sum_j D(j,i) lb(j)
    for (int i = 0; i < P; ++i) {
      double t = 0.0;
      for (int j = 0; j < P; ++j) t += s.D[j * P + i] * s.lb[side][j];
      s.dlb[side][i] = t;
    }
    for (int i = 0; i < P; ++i) s.dlbw[side][i] = s.dlb[side][i] / s.w[i];
  }
}

const Spectral* Oracle::spectral(int N) {
  auto it = spectra.find(N);
  if (it != spectra.end()) return it->second.get();
  auto s = std::make_unique<Spectral>();
  build_spectral(*s, N, cas.nodes);
  const Spectral* r = s.get();
  spectra[N] = std::move(s);
  return r;
}

}  // namespace orc
