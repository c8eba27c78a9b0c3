/*
 * dissipation.cpp -- artificial dissipation of the oracle (TEST INFRASTRUCTURE).
 *
 * Restates Approximation/DGArtificialDissipation.f90 (Navier-Stokes build only):
 *   JumpsBasedElementViscosity   :277-338   element viscosity from the interface jumps of rho, rhoE
 *   JumpsBasedEdgeViscosity      :340-363   mean of the adjacent elements' viscosities
 *   LaplaceDissipation_*         :208-249   F_a = mu dQ_local (volume), -mu Area (QL - QR) (faces)
 *   PhysicalDissipation_*        :251-269   mu_a added to mu in every viscous flux
 * and the edge jumps Edge_ComputeJumps / CurvedEdge_ / SubdividedEdge_ / CurvedSubdividedEdge_ /
 * StraightBdryEdge_ / CurvedBdryEdge_ComputeJumps (Mesh/QuadElement_EdgeProcedures.incf:1348-1619).
 *
 * Two indicators without a reference counterpart feed the same viscosity law Ceps sqrt(V)/(N+1) G:
 * the modal-decay indicator (Persson & Peraire, "Sub-cell shock capturing for discontinuous Galerkin
 * methods", AIAA 2006-112): s = max over rho and p of log10(E_N/E), E the energy of the element's
 * modal coefficients in the orthonormal Legendre basis of [0,1] and E_N that of the modes whose higher
 * index is N, G = the reference's sine ramp around s0 of half width kappa; and an external G per
 * element (the library's learned sensor, checked through it).  These two are evaluated on the first
 * stage of each time step and held for its other stages (the library's rule for its sensors); the
 * reference's jumps indicator is evaluated at every residual, as in the reference.
 */
#include "oracle_internal.h"
#include "viscous.h"
#include <cfloat>
#include <cmath>

namespace orc {

// ProjectSolution (types 1-6) of one variable onto the edge nodes
static void project_var(const Edge& f, int var, std::vector<double>& QL, std::vector<double>& QR) {
  const int P = f.P();
  const EdgeStorage& sL = f.storage[SLOT_LEFT];
  const EdgeStorage& sR = f.storage[SLOT_RIGHT];
  const int PL = sL.sp->P, PR = sR.sp->P;
  QL.assign(P, 0.0);
  QR.assign(P, 0.0);
  if (f.transform[SLOT_LEFT]) {
    for (int l = 0; l <= f.NLow; ++l) for (int i = 0; i < P; ++i) QL[i] = QL[i] + f.T_forward[i * PL + l] * sL.Q[4 * l + var];
  } else {
    for (int i = 0; i < P; ++i) QL[i] = sL.Q[4 * i + var];
  }
  if (f.transform[SLOT_RIGHT]) {
    for (int l = 0; l <= f.NLow; ++l) for (int i = 0; i < P; ++i) {
      const int dst = f.inverse ? (P - 1 - i) : i;
      QR[dst] = QR[dst] + f.T_forward[i * PR + l] * sR.Q[4 * l + var];
    }
  } else if (f.inverse) {
    for (int i = 0; i < P; ++i) QR[i] = sR.Q[4 * (P - 1 - i) + var];
  } else {
    for (int i = 0; i < P; ++i) QR[i] = sR.Q[4 * i + var];
  }
}

static double jumps_sum(const Spectral& sp, const std::vector<double>& QL, const std::vector<double>& QR,
                        const double* dS, bool per_node) {
  double s = 0.0;
  for (int i = 0; i < sp.P; ++i) {
    const double j = 2.0 * (QL[i] - QR[i]) / (QL[i] + QR[i]);
    s = s + sp.w[i] * j * j * (per_node ? dS[i] : dS[0]);
  }
  return s;
}

double edge_jumps(const Oracle& o, const Edge& f, int var) {
  (void)o;
  std::vector<double> QL, QR;
  if (f.kind == E_STRAIGHT || f.kind == E_CURVED) {
    project_var(f, var, QL, QR);
    return jumps_sum(*f.sp, QL, QR, f.dS.data(), f.kind == E_CURVED);
  }
  if (f.is_subdiv()) {
    auto proj = [&](const std::vector<double>& T, int rows, int slot) {
      const EdgeStorage& s = f.storage[slot];
      const int cols = s.sp->P;
      std::vector<double> out(rows, 0.0);
      for (int l = 0; l < cols; ++l) for (int i = 0; i < rows; ++i) out[i] = out[i] + T[i * cols + l] * s.Q[4 * l + var];
      return out;
    };
    const int PN = f.spN->P, PS = f.spS->P;
    const std::vector<double> QLN = proj(f.T_LN_FWD, PN, SLOT_LEFT), QLS = proj(f.T_LS_FWD, PS, SLOT_LEFT);
    const std::vector<double> QRN = proj(f.T_RN_FWD, PN, SLOT_RN), QRS = proj(f.T_RS_FWD, PS, SLOT_RS);
    const bool curved = f.kind == E_CURVED_SUBDIV;
    return jumps_sum(*f.spN, QLN, QRN, f.dS_N.data(), curved) + jumps_sum(*f.spS, QLS, QRS, f.dS_S.data(), curved);
  }
  // boundary edges: the viscous boundary state; both straight and curved kinds use dS(0)
  const int P = f.P();
  const std::vector<double>& uS = *f.uSB;
  QL.assign(P, 0.0);
  QR.assign(P, 0.0);
  for (int i = 0; i < P; ++i) {
    QL[i] = f.storage[0].Q[4 * i + var];
    QR[i] = f.inverse ? uS[4 * (P - 1 - i) + var] : uS[4 * i + var];
  }
  return jumps_sum(*f.sp, QL, QR, f.dS.data(), false);
}

double av_element_viscosity(const Oracle& o, const Element& e) {
  const double k = 5.0;
  const Edge& eb = o.ed[e.edges[0]];
  const Edge& er = o.ed[e.edges[1]];
  const Edge& et = o.ed[e.edges[2]];
  const Edge& el = o.ed[e.edges[3]];
  const double gkRHO = edge_jumps(o, eb, IRHO) + edge_jumps(o, er, IRHO) + edge_jumps(o, et, IRHO) + edge_jumps(o, el, IRHO);
  const double gkRHOE =
      edge_jumps(o, eb, IRHOE) + edge_jumps(o, er, IRHOE) + edge_jumps(o, et, IRHOE) + edge_jumps(o, el, IRHOE);
  double gk = std::fmax(gkRHO, gkRHOE);
  gk = gk / (eb.Area + er.Area + et.Area + el.Area);
  if (gk > 1.0e-8) gk = std::log10(gk);
  else gk = -DBL_MAX;
  const double maxVisc = std::sqrt(e.volume) / (e.N + 1);
  const double s0 = std::log10(1.0 / std::pow(double(e.N + 1), 4.0)) + 1;
  double G;
  if (gk < s0 - k) G = 0.0;
  else if (gk < s0 + k) G = 0.5 * std::sin(0.5 * PI * (gk - s0) / k) + 0.5;
  else G = 1.0;
  return o.cas.av_intensity * maxVisc * G;
}

// nodal -> modal matrix of the orthonormal Legendre basis sqrt(2k+1) L_k(2x-1) at the element nodes
static std::vector<double> modal_matrix(const Spectral& sp) {
  const int P = sp.P;
  std::vector<double> A(size_t(P) * 2 * P, 0.0);
  for (int i = 0; i < P; ++i) {
    const double x = 2.0 * sp.xi[i] - 1.0;
    double l0 = 1.0, l1 = x;
    for (int k = 0; k < P; ++k) {
      double Lk;
      if (k == 0) Lk = 1.0;
      else if (k == 1) Lk = x;
      else { const double l2 = ((2.0 * k - 1.0) * x * l1 - (k - 1.0) * l0) / k; l0 = l1; l1 = l2; Lk = l2; }
      A[size_t(i) * 2 * P + k] = std::sqrt(2.0 * k + 1.0) * Lk;
    }
    A[size_t(i) * 2 * P + P + i] = 1.0;
  }
  for (int c = 0; c < P; ++c) {   // Gauss-Jordan with partial pivoting
    int piv = c;
    for (int r = c + 1; r < P; ++r) if (std::fabs(A[size_t(r) * 2 * P + c]) > std::fabs(A[size_t(piv) * 2 * P + c])) piv = r;
    if (piv != c) for (int q = 0; q < 2 * P; ++q) std::swap(A[size_t(c) * 2 * P + q], A[size_t(piv) * 2 * P + q]);
    const double d = A[size_t(c) * 2 * P + c];
    for (int q = 0; q < 2 * P; ++q) A[size_t(c) * 2 * P + q] /= d;
    for (int r = 0; r < P; ++r)
      if (r != c) {
        const double f = A[size_t(r) * 2 * P + c];
        for (int q = 0; q < 2 * P; ++q) A[size_t(r) * 2 * P + q] -= f * A[size_t(c) * 2 * P + q];
      }
  }
  std::vector<double> Vinv(size_t(P) * P);
  for (int k = 0; k < P; ++k) for (int i = 0; i < P; ++i) Vinv[size_t(k) * P + i] = A[size_t(k) * 2 * P + P + i];
  return Vinv;
}

static double ramp(double s, double s0, double k) {
  if (s < s0 - k) return 0.0;
  if (s < s0 + k) return 0.5 * std::sin(0.5 * PI * (s - s0) / k) + 0.5;
  return 1.0;
}

double modal_indicator(const Oracle& o, const Element& e) {
  const int P = e.P, N = e.N, NP = P * P;
  const std::vector<double> Vinv = modal_matrix(*e.sp);
  const double* Q = &o.Q[e.offset];
  double smax = -DBL_MAX;
  for (int v = 0; v < 2; ++v) {
    std::vector<double> u(NP);
    for (int q = 0; q < NP; ++q) {
      const double* qq = &Q[4 * q];
      u[q] = v == 0 ? qq[0] : o.ph.gm1 * (qq[3] - 0.5 * (qq[1] * qq[1] + qq[2] * qq[2]) / qq[0]);
    }
    double E = 0.0, EN = 0.0;
    for (int n = 0; n < P; ++n)
      for (int m = 0; m < P; ++m) {
        double c = 0.0;
        for (int j = 0; j < P; ++j) {
          double a = 0.0;
          for (int i = 0; i < P; ++i) a += Vinv[size_t(m) * P + i] * u[j * P + i];
          c += Vinv[size_t(n) * P + j] * a;
        }
        E += c * c;
        if (m == N || n == N) EN += c * c;
      }
    const double s = (E > 0.0 && EN > 0.0) ? std::log10(EN / E) : -DBL_MAX;
    smax = std::fmax(smax, s);
  }
  return ramp(smax, o.cas.av_s0, o.cas.av_kappa);
}

void compute_av_viscosity(Oracle& o) {
  if (o.av_hold && o.cas.av_indicator != OR_IND_JUMPS && o.av_mu.size() == o.el.size()) return;
  o.av_mu.assign(o.el.size(), 0.0);
  if (!o.cas.navier_stokes || o.cas.av_type == OR_AV_NONE) return;
#pragma omp parallel for schedule(static)
  for (size_t e = 0; e < o.el.size(); ++e) {
    const Element& E = o.el[e];
    if (o.cas.av_indicator == OR_IND_JUMPS) {
      o.av_mu[e] = av_element_viscosity(o, E);
    } else {
      const double G = o.cas.av_indicator == OR_IND_MODAL ? modal_indicator(o, E)
                                                          : (e < o.av_g_ext.size() ? o.av_g_ext[e] : 0.0);
      const double maxVisc = std::sqrt(E.volume) / (E.N + 1);
      o.av_mu[e] = o.cas.av_intensity * maxVisc * G;
    }
  }
}

double av_edge_viscosity(const Oracle& o, const Edge& f) {
  if (f.is_bdry()) return o.av_mu[f.quads[0]] / 1.0;
  if (f.is_subdiv()) return (o.av_mu[f.quads[SLOT_RN]] + o.av_mu[f.quads[SLOT_LEFT]] + o.av_mu[f.quads[SLOT_RS]]) / 3.0;
  return (o.av_mu[f.quads[SLOT_RIGHT]] + o.av_mu[f.quads[SLOT_LEFT]]) / 2.0;
}

// Physical type: mu_a of the elements (volume loop) and edges (face loops)
void set_physical_av(Oracle& o) {
  const bool phys = o.cas.navier_stokes && o.cas.av_type == OR_AV_PHYSICAL;
  for (size_t e = 0; e < o.el.size(); ++e) o.el[e].mu_a = phys ? o.av_mu[e] : 0.0;
  for (auto& f : o.ed) f.mu_a = phys ? av_edge_viscosity(o, f) : 0.0;
}

bool laplacian_av(const Oracle& o) { return o.cas.navier_stokes && o.cas.av_type == OR_AV_LAPLACIAN; }

// LaplaceDissipation_ComputeVolumeFluxes: F -= mu_e * dQ_local   (F[q*8 + d*4 + k])
void av_volume_flux(Oracle& o, Element& e, std::vector<double>& F) {
  if (!laplacian_av(o)) return;
  const int NP = e.P * e.P;
  std::vector<double> dQ(size_t(8) * NP);
  interior_gradient(o, e, dQ.data());
  const double mu = o.av_mu[e.id];
  for (int q = 0; q < NP; ++q)
    for (int d = 0; d < 2; ++d)
      for (int k = 0; k < 4; ++k) F[q * 8 + d * 4 + k] = F[q * 8 + d * 4 + k] - mu * dQ[(size_t(d) * NP + q) * 4 + k];
}

// LaplaceDissipation_ComputeFaceFluxes at one point: Fa[k] = -mu Area (qL - qR)
void av_face_flux(const Oracle& o, const Edge& f, const double* qL, const double* qR, double* Fa) {
  if (!laplacian_av(o)) { for (int k = 0; k < 4; ++k) Fa[k] = 0.0; return; }
  const double mu = av_edge_viscosity(o, f);
  for (int k = 0; k < 4; ++k) Fa[k] = -(mu * f.Area * (qL[k] - qR[k]));
}

}  // namespace orc
