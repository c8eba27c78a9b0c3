// hg_spectral.cpp -- nodes, weights and nodal matrices on [0,1] (host code).
#include "hg_spectral.h"
#include <cmath>
#include <cfloat>
#include <stdexcept>
#include <utility>

namespace hg {

namespace {

// L_n(x) and L_n'(x) by the three-term recurrence
void legendre(int n, double x, double& L, double& dL) {
  double l0 = 1.0, l1 = x, d0 = 0.0, d1 = 1.0;
  if (n == 0) { L = 1.0; dL = 0.0; return; }
  for (int k = 2; k <= n; ++k) {
    const double l2 = ((2.0 * k - 1.0) * x * l1 - (k - 1.0) * l0) / k;
    const double d2 = d0 + (2.0 * k - 1.0) * l1;
    l0 = l1; l1 = l2; d0 = d1; d1 = d2;
  }
  L = l1; dL = d1;
}

void gauss(int N, std::vector<double>& x, std::vector<double>& w) {
  const double pi = 3.14159265358979323846;
  x.assign(N + 1, 0.0); w.assign(N + 1, 0.0);
  if (N == 0) { x[0] = 0.0; w[0] = 2.0; return; }
  for (int j = 0; j <= N / 2; ++j) {
    double r = -std::cos((2.0 * j + 1.0) * pi / (2.0 * N + 2.0));
    double L, dL;
    for (int it = 0; it < 100; ++it) {
      legendre(N + 1, r, L, dL);
      const double d = -L / dL;
      r += d;
      if (std::fabs(d) <= 4.0 * DBL_EPSILON * std::fabs(r)) break;
    }
    legendre(N + 1, r, L, dL);
    x[j] = r; x[N - j] = -r;
    w[j] = w[N - j] = 2.0 / ((1.0 - r * r) * dL * dL);
  }
  if (N % 2 == 0) {
    double L, dL;
    legendre(N + 1, 0.0, L, dL);
    x[N / 2] = 0.0;
    w[N / 2] = 2.0 / (dL * dL);
  }
}

// interior LGL nodes are the roots of L_N'(x); Newton on q = L_{N+1} - L_{N-1} (proportional to (1-x^2) L_N')
void lobatto(int N, std::vector<double>& x, std::vector<double>& w) {
  const double pi = 3.14159265358979323846;
  x.assign(N + 1, 0.0); w.assign(N + 1, 0.0);
  x[0] = -1.0; x[N] = 1.0;
  w[0] = w[N] = 2.0 / (N * (N + 1.0));
  for (int j = 1; j <= (N + 1) / 2 - 1; ++j) {
    double r = -std::cos((j + 0.25) * pi / N - 3.0 / (8.0 * N * pi * (j + 0.25)));
    for (int it = 0; it < 50; ++it) {
      double Lp, dLp, Lm, dLm;
      legendre(N + 1, r, Lp, dLp);
      legendre(N - 1, r, Lm, dLm);
      const double d = -(Lp - Lm) / (dLp - dLm);
      r += d;
      if (std::fabs(d) <= 1e-15 * std::fabs(r)) break;
    }
    double LN, dLN;
    legendre(N, r, LN, dLN);
    x[j] = r; x[N - j] = -r;
    w[j] = w[N - j] = 2.0 / (N * (N + 1.0) * LN * LN);
  }
  if (N % 2 == 0) {
    double LN, dLN;
    legendre(N, 0.0, LN, dLN);
    x[N / 2] = 0.0;
    w[N / 2] = 2.0 / (N * (N + 1.0) * LN * LN);
  }
}

bool same_point(double a, double b) {
  if (a == 0.0 || b == 0.0) return std::fabs(a - b) <= 2.0 * DBL_EPSILON;
  return std::fabs(a - b) <= 2.0 * DBL_EPSILON * std::fmax(std::fabs(a), std::fabs(b));
}

}  // namespace

std::vector<double> lagrange_basis(const NodalOps& o, double x) {
  std::vector<double> l(o.P, 0.0);
  for (int j = 0; j < o.P; ++j)
    if (same_point(x, o.xi[j])) { l[j] = 1.0; return l; }
  double s = 0.0;
  for (int j = 0; j < o.P; ++j) { l[j] = o.wb[j] / (x - o.xi[j]); s += l[j]; }
  for (int j = 0; j < o.P; ++j) l[j] /= s;
  return l;
}

NodalOps make_nodal_ops(int N, int node_type) {
  if (N < 1 || N > 16) throw std::runtime_error("polynomial order out of range");
  NodalOps o;
  o.N = N; o.P = N + 1;
  const int P = o.P;
  if (node_type == 1) gauss(N, o.xi, o.w);
  else if (node_type == 2) lobatto(N, o.xi, o.w);
  else throw std::runtime_error("unknown node type");
  for (int i = 0; i < P; ++i) { o.xi[i] = 0.5 * (1.0 + o.xi[i]); o.w[i] *= 0.5; }
  o.wb.assign(P, 1.0);
  for (int j = 0; j < P; ++j)
    for (int k = 0; k < P; ++k)
      if (k != j) o.wb[j] *= (o.xi[j] - o.xi[k]);
  for (int j = 0; j < P; ++j) o.wb[j] = 1.0 / o.wb[j];
  o.D.assign(P * P, 0.0);
  for (int i = 0; i < P; ++i) {
    double diag = 0.0;
    for (int j = 0; j < P; ++j)
      if (j != i) {
        o.D[i * P + j] = o.wb[j] / (o.wb[i] * (o.xi[i] - o.xi[j]));
        diag -= o.D[i * P + j];
      }
    o.D[i * P + i] = diag;
  }
  o.hatD.assign(P * P, 0.0);
  for (int i = 0; i < P; ++i)
    for (int l = 0; l < P; ++l) o.hatD[i * P + l] = o.w[l] * o.D[l * P + i] / o.w[i];
  o.lb0 = lagrange_basis(o, 0.0);
  o.lb1 = lagrange_basis(o, 1.0);
  o.lbw0.resize(P); o.lbw1.resize(P);
  for (int i = 0; i < P; ++i) { o.lbw0[i] = o.lb0[i] / o.w[i]; o.lbw1[i] = o.lb1[i] / o.w[i]; }
  // dlb = D^T lb (derivative of the boundary interpolant), dlbw = dlb / w
  o.dlbw0.assign(P, 0.0); o.dlbw1.assign(P, 0.0);
  for (int i = 0; i < P; ++i) {
    double s0 = 0.0, s1 = 0.0;
    for (int j = 0; j < P; ++j) { s0 += o.D[j * P + i] * o.lb0[j]; s1 += o.D[j * P + i] * o.lb1[j]; }
    o.dlbw0[i] = s0 / o.w[i];
    o.dlbw1[i] = s1 / o.w[i];
  }
  // modal transform (orthonormal Legendre on [0,1]) by Gauss-Jordan elimination with pivoting
  {
    std::vector<double> V(P * P), A(P * 2 * P, 0.0);
    for (int i = 0; i < P; ++i)
      for (int k = 0; k < P; ++k) {
        double L, dL;
        legendre(k, 2.0 * o.xi[i] - 1.0, L, dL);
        V[i * P + k] = std::sqrt(2.0 * k + 1.0) * L;
      }
    for (int r = 0; r < P; ++r) {
      for (int c = 0; c < P; ++c) A[r * 2 * P + c] = V[r * P + c];
      A[r * 2 * P + P + r] = 1.0;
    }
    for (int c = 0; c < P; ++c) {
      int piv = c;
      for (int r = c + 1; r < P; ++r)
        if (std::fabs(A[r * 2 * P + c]) > std::fabs(A[piv * 2 * P + c])) piv = r;
      if (piv != c) for (int q = 0; q < 2 * P; ++q) std::swap(A[c * 2 * P + q], A[piv * 2 * P + q]);
      const double d = A[c * 2 * P + c];
      for (int q = 0; q < 2 * P; ++q) A[c * 2 * P + q] /= d;
      for (int r = 0; r < P; ++r)
        if (r != c) {
          const double f = A[r * 2 * P + c];
          for (int q = 0; q < 2 * P; ++q) A[r * 2 * P + q] -= f * A[c * 2 * P + q];
        }
    }
    o.Vinv.assign(P * P, 0.0);
    for (int k = 0; k < P; ++k)
      for (int i = 0; i < P; ++i) o.Vinv[k * P + i] = A[k * 2 * P + P + i];
  }
  return o;
}

}  // namespace hg
