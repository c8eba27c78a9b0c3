/*
 * residual.cpp -- DGSEM time derivative of the oracle (TEST INFRASTRUCTURE).
 *
 * Restates (Euler part; the viscous terms live in viscous.cpp):
 *   InitializePhysics (_DIMENSIONLESS_TAU)        Physics/PhysicsNS.f90:405-481
 *   InviscidFlux2D                                Physics/InviscidFluxes.f90:104-147
 *   RoeFlux / HLLFlux / ExactRiemannSolver        Physics/RiemannSolvers.f90:33-459
 *   DGSpatial_computeTimeDerivative / newTimeStep / computeQDot / face loops /
 *   ComputeRiemannSolver_* / interpolateSolutionToBoundaries
 *                                                 Approximation/DGSpatialDiscretizationMethods.f90
 *   Scalar_StdVolumeGreen / Scalar_StdFace        Approximation/DGWeakIntegrals.f90:111-266
 *   Edge_ProjectSolutionType1..6 / Edge_ProjectFluxesType1..6
 *                                                 Mesh/QuadElement_EdgeProcedures.incf:749-1206
 *   Zone_LinkPeriodicZones / checkIfAreInverted   Mesh/QuadMesh_Zones.incf:22-131
 *   EulerWall_UpdateSolution                      BoundaryConditions/EulerWall.incf:71-158
 *   Dirichlet / Farfield / PressureOutlet UpdateSolution (inviscid part),
 *                                                 BoundaryConditions/{Dirichlet,Farfield,PressureOutlet}.incf
 * The LxF (Rusanov) flux has no reference counterpart; it uses the same
 * rotation and 1/(sqrt(gamma) M) scaling as the reference solvers.
 */
#include "oracle_internal.h"
#include "viscous.h"
#include <stdexcept>
#include <algorithm>

namespace orc {

void init_physics(Oracle& o) {
  Physics& ph = o.ph;
  const or_case& c = o.cas;
  ph.gamma = 1.4; ph.R = 287.15; ph.gm1 = 0.4; ph.gogm1 = 3.5; ph.invgm1 = 2.5;
  ph.L = c.reynolds_length;
  ph.T = c.temperature_ref;
  ph.p = c.pressure_ref;
  ph.rho = ph.p / (ph.R * ph.T);
  ph.a = std::sqrt(ph.p / ph.rho);
  ph.Mach = c.mach;
  ph.V = std::sqrt(ph.gamma) * ph.Mach * ph.a;
  ph.mu_ref = (c.reynolds == 0.0) ? 0.0 : ph.rho * ph.V * ph.L / c.reynolds;
  ph.kappa_ref = ph.mu_ref * (ph.R * 3.5) / c.prandtl;
  ph.sqrtGammaMach = std::sqrt(ph.gamma) * ph.Mach;
  ph.gammaMach2 = ph.gamma * ph.Mach * ph.Mach;
  ph.invSqrtGammaMach = 1.0 / (std::sqrt(ph.gamma) * ph.Mach);
  if (c.reynolds == 0.0) { ph.mu = 0.0; ph.kappa = 0.0; }
  else { ph.mu = 1.0 / c.reynolds; ph.kappa = ph.gogm1 / (c.prandtl * c.reynolds); }
  ph.cp = ph.gogm1; ph.cv = ph.invgm1; ph.Re = c.reynolds; ph.Pr = c.prandtl;
}

// ---------------------------------------------------------------- Riemann solvers
static inline void flux_normal(double rho, double u, double v, double p, double H, double* F) {
  F[0] = rho * u; F[1] = F[0] * u + p; F[2] = F[0] * v; F[3] = H * F[0];
}

static inline void rotate_back(double* F, double nx, double ny) {
  const double Ft = F[1] * nx - F[2] * ny;
  F[2] = F[1] * ny + F[2] * nx;
  F[1] = Ft;
}

static void roe(const Physics& ph, const double* qL, const double* qR, double nx, double ny, double* F) {
  const double rhoL = qL[0], invRhoL = 1.0 / rhoL, sqrtRhoL = std::sqrt(rhoL);
  const double uL = (qL[1] * nx + qL[2] * ny) * invRhoL, vL = (-qL[1] * ny + qL[2] * nx) * invRhoL;
  const double pL = ph.gm1 * (qL[3] - 0.5 * rhoL * (uL * uL + vL * vL));
  const double HL = ph.cp * pL * invRhoL + 0.5 * (uL * uL + vL * vL);
  const double rhoR = qR[0], invRhoR = 1.0 / rhoR, sqrtRhoR = std::sqrt(rhoR);
  const double uR = (qR[1] * nx + qR[2] * ny) * invRhoR, vR = (-qR[1] * ny + qR[2] * nx) * invRhoR;
  const double pR = ph.gm1 * (qR[3] - 0.5 * rhoR * (uR * uR + vR * vR));
  const double HR = ph.cp * pR * invRhoR + 0.5 * (uR * uR + vR * vR);
  const double invrho = 1.0 / (sqrtRhoL + sqrtRhoR);
  const double u = (sqrtRhoL * uL + sqrtRhoR * uR) * invrho;
  const double v = (sqrtRhoL * vL + sqrtRhoR * vR) * invrho;
  const double H = (sqrtRhoL * HL + sqrtRhoR * HR) * invrho;
  const double a = std::sqrt(ph.gm1 * (H - 0.5 * (u * u + v * v)));
  const double lam[4] = {u - a, u, u, u + a};
  int nw;
  if (lam[0] > 0.0) nw = 0; else if (lam[1] > 0.0) nw = 1; else if (lam[3] > 0.0) nw = 3; else nw = 4;
  const double K[4][4] = {{1.0, u - a, v, H - u * a}, {1.0, u, v, 0.5 * (u * u + v * v)},
                          {0.0, 0.0, 1.0, v}, {1.0, u + a, v, H + u * a}};
  const double dq0 = rhoR - rhoL, dq1 = rhoR * uR - rhoL * uL, dq2 = rhoR * vR - rhoL * vL, dq3 = qR[3] - qL[3];
  double al[4];
  al[2] = dq2 - v * dq0;
  al[1] = ph.gm1 * (dq0 * (H - u * u) + u * dq1 - dq3 + (dq2 - v * dq0) * v) / (a * a);
  al[0] = (dq0 * (u + a) - dq1 - a * al[1]) / (2.0 * a);
  al[3] = dq0 - (al[0] + al[1]);
  flux_normal(rhoL, uL, vL, pL, HL, F);
  for (int w = 0; w < nw; ++w)
    for (int k = 0; k < 4; ++k) F[k] = F[k] + al[w] * lam[w] * K[w][k];
  rotate_back(F, nx, ny);
  for (int k = 0; k < 4; ++k) F[k] *= ph.invSqrtGammaMach;
}

static void hll(const Physics& ph, const double* qL, const double* qR, double nx, double ny, double* F) {
  const double rhoL = qL[0], invRhoL = 1.0 / rhoL;
  const double uL = (qL[1] * nx + qL[2] * ny) * invRhoL, vL = (-qL[1] * ny + qL[2] * nx) * invRhoL;
  const double pL = ph.gm1 * (qL[3] - 0.5 * rhoL * (uL * uL + vL * vL));
  const double HL = ph.cp * pL * invRhoL + 0.5 * (uL * uL + vL * vL);
  const double aL = std::sqrt(ph.gamma * pL * invRhoL), rhoeL = qL[3];
  const double rhoR = qR[0], invRhoR = 1.0 / rhoR;
  const double uR = (qR[1] * nx + qR[2] * ny) * invRhoR, vR = (-qR[1] * ny + qR[2] * nx) * invRhoR;
  const double pR = ph.gm1 * (qR[3] - 0.5 * rhoR * (uR * uR + vR * vR));
  const double HR = ph.cp * pR * invRhoR + 0.5 * (uR * uR + vR * vR);
  const double aR = std::sqrt(ph.gamma * pR * invRhoR), rhoeR = qR[3];
  const double sqrtRhoL = std::sqrt(rhoL), sqrtRhoR = std::sqrt(rhoR);
  const double invrho = 1.0 / (sqrtRhoL + sqrtRhoR);
  const double u = (sqrtRhoL * uL + sqrtRhoR * uR) * invrho;
  const double v = (sqrtRhoL * vL + sqrtRhoR * vR) * invrho;
  const double H = (sqrtRhoL * HL + sqrtRhoR * HR) * invrho;
  const double a = std::sqrt(ph.gm1 * (H - 0.5 * (u * u + v * v)));
  const double SL = std::min(uL - aL, u - a), SR = std::max(uR + aR, u + a);
  if (SL >= 0.0) flux_normal(rhoL, uL, vL, pL, HL, F);
  else if (SR <= 0.0) flux_normal(rhoR, uR, vR, pR, HR, F);
  else {
    const double invdS = 1.0 / (SR - SL);
    F[0] = (SR * rhoL * uL - SL * rhoR * uR + SL * SR * (rhoR - rhoL)) * invdS;
    F[1] = (SR * (rhoL * uL * uL + pL) - SL * (rhoR * uR * uR + pR) + SL * SR * (rhoR * uR - rhoL * uL)) * invdS;
    F[2] = (SR * rhoL * uL * vL - SL * rhoR * uR * vR + SR * SL * (rhoR * vR - rhoL * vL)) * invdS;
    F[3] = (SR * uL * rhoL * HL - SL * uR * rhoR * HR + SR * SL * (rhoeR - rhoeL)) * invdS;
  }
  rotate_back(F, nx, ny);
  for (int k = 0; k < 4; ++k) F[k] *= ph.invSqrtGammaMach;
}

static void lxf(const Physics& ph, const double* qL, const double* qR, double nx, double ny, double* F) {
  const double rhoL = qL[0], invRhoL = 1.0 / rhoL;
  const double uL = (qL[1] * nx + qL[2] * ny) * invRhoL, vL = (-qL[1] * ny + qL[2] * nx) * invRhoL;
  const double pL = ph.gm1 * (qL[3] - 0.5 * rhoL * (uL * uL + vL * vL));
  const double HL = ph.cp * pL * invRhoL + 0.5 * (uL * uL + vL * vL);
  const double aL = std::sqrt(ph.gamma * pL * invRhoL);
  const double rhoR = qR[0], invRhoR = 1.0 / rhoR;
  const double uR = (qR[1] * nx + qR[2] * ny) * invRhoR, vR = (-qR[1] * ny + qR[2] * nx) * invRhoR;
  const double pR = ph.gm1 * (qR[3] - 0.5 * rhoR * (uR * uR + vR * vR));
  const double HR = ph.cp * pR * invRhoR + 0.5 * (uR * uR + vR * vR);
  const double aR = std::sqrt(ph.gamma * pR * invRhoR);
  const double lam = std::max(std::fabs(uL) + aL, std::fabs(uR) + aR);
  double FL[4], FR[4];
  flux_normal(rhoL, uL, vL, pL, HL, FL);
  flux_normal(rhoR, uR, vR, pR, HR, FR);
  const double dq[4] = {rhoR - rhoL, rhoR * uR - rhoL * uL, rhoR * vR - rhoL * vL, qR[3] - qL[3]};
  for (int k = 0; k < 4; ++k) F[k] = 0.5 * (FL[k] + FR[k]) - 0.5 * lam * dq[k];
  rotate_back(F, nx, ny);
  for (int k = 0; k < 4; ++k) F[k] *= ph.invSqrtGammaMach;
}

static void exact_f(const Physics& ph, double p, const double* W, double& F, double& dF) {
  const double gamma = ph.gamma;
  if (p > W[3]) {
    const double A = 2.0 / (W[0] * (gamma + 1.0));
    const double B = ph.gm1 * W[3] / (gamma + 1.0);
    const double s = std::sqrt(A / (p + B));
    F = (p - W[3]) * s;
    dF = s * (1.0 - 0.5 * (p - W[3]) / (B + p));
  } else {
    F = 2.0 * ph.cv * W[4] * (std::pow(p / W[3], 0.5 / ph.cp) - 1);
    dF = 1.0 / (W[0] * W[4]) * std::pow(p / W[3], -0.5 * (gamma + 1.0) / gamma);
  }
}

// W = {rho, u, v, p, a}
static void exact_pstar(const Physics& ph, const double* WL, const double* WR, double& pstar, double& ustar) {
  const double cp = ph.cp;
  pstar = std::pow((WL[4] + WR[4] - 0.5 * ph.gm1 * (WR[1] - WL[1])) /
                       (WL[4] / std::pow(WL[3], 0.5 / cp) + WR[4] / std::pow(WR[3], 0.5 / cp)),
                   2.0 * cp);
  double FL, dFL, FR, dFR;
  for (int it = 1; it <= 50; ++it) {
    exact_f(ph, pstar, WL, FL, dFL);
    exact_f(ph, pstar, WR, FR, dFR);
    const double F = FL + FR + WR[1] - WL[1], dF = dFL + dFR;
    const double pold = pstar;
    pstar = pold - F / dF;
    const double cha = 0.5 * std::fabs(pstar - pold) / (pstar + pold);
    if (std::fabs(cha) < 1.0e-6) {
      exact_f(ph, pstar, WL, FL, dFL);
      exact_f(ph, pstar, WR, FR, dFR);
      ustar = 0.5 * (WL[1] + WR[1] + FR - FL);
      return;
    }
  }
  // the reference leaves ustar undefined when Newton does not converge
  ustar = 0.5 * (WL[1] + WR[1] + FR - FL);
}

static void exact(const Physics& ph, const double* qL, const double* qR, double nx, double ny, double* F) {
  const double gamma = ph.gamma, gm1 = ph.gm1, cp = ph.cp, cv = ph.cv;
  double qnL[4] = {qL[0], qL[1] * nx + qL[2] * ny, -qL[1] * ny + qL[2] * nx, qL[3]};
  double qnR[4] = {qR[0], qR[1] * nx + qR[2] * ny, -qR[1] * ny + qR[2] * nx, qR[3]};
  double wL[5], wR[5];
  wL[0] = qnL[0]; wL[1] = qnL[1] / qnL[0]; wL[2] = qnL[2] / qnL[0];
  wL[3] = gm1 * (qnL[3] - 0.5 * (qnL[1] * wL[1] + qnL[2] * wL[2])); wL[4] = std::sqrt(gamma * wL[3] / wL[0]);
  wR[0] = qnR[0]; wR[1] = qnR[1] / qnR[0]; wR[2] = qnR[2] / qnR[0];
  wR[3] = gm1 * (qnR[3] - 0.5 * (qnR[1] * wR[1] + qnR[2] * wR[2])); wR[4] = std::sqrt(gamma * wR[3] / wR[0]);
  double pstar, ustar;
  exact_pstar(ph, wL, wR, pstar, ustar);
  for (int k = 0; k < 4; ++k) F[k] = 0.0;
  auto upwind = [&](const double* qn, const double* w) {
    F[0] = qn[1]; F[1] = qn[1] * w[1] + w[3]; F[2] = qn[2] * w[1];
    F[3] = w[1] * (cp * w[3] + 0.5 * (qn[1] * w[1] + qn[2] * w[2]));
  };
  if (ustar >= 0.0) {
    const double* w = wL;
    if (pstar <= w[3] && w[1] >= w[4]) upwind(qnL, wL);
    else if (pstar <= w[3] && w[1] < w[4] && ustar < w[4] * std::pow(pstar / w[3], 0.5 / cp)) {
      const double rs = w[0] * std::pow(pstar / w[3], 1.0 / gamma);
      F[0] = rs * ustar; F[1] = rs * ustar * ustar + pstar; F[2] = F[0] * w[2];
      F[3] = ustar * (cp * pstar + 0.5 * rs * (ustar * ustar + w[2] * w[2]));
    } else if (pstar <= w[3] && w[1] < w[4] && ustar >= w[4] * std::pow(pstar / w[3], 0.5 / cp)) {
      const double uFan = 2.0 * w[4] / (gamma + 1.0) + (gamma - 1.0) / (gamma + 1.0) * w[1];
      const double rs = w[0] * std::pow(uFan / w[4], 2.0 * cv);
      const double pFan = w[3] * std::pow(rs / w[0], gamma);
      F[0] = rs * uFan; F[1] = rs * uFan * uFan + pFan; F[2] = rs * uFan * w[2];
      F[3] = uFan * (cp * pFan + 0.5 * rs * (uFan * uFan + w[2] * w[2]));
    } else if (pstar > w[3] && w[1] >= w[4] * std::sqrt((gamma + 1.0) / (2.0 * gamma) * pstar / w[3] + 0.5 / cp)) {
      upwind(qnL, wL);
    } else if (pstar > w[3] && w[1] < w[4] * std::sqrt((gamma + 1.0) / (2.0 * gamma) * pstar / w[3] + 0.5 / cp)) {
      const double rs = w[0] * ((pstar / w[3] + (gamma - 1.0) / (gamma + 1.0)) / (pstar / w[3] * (gamma - 1.0) / (gamma + 1.0) + 1.0));
      F[0] = rs * ustar; F[1] = rs * ustar * ustar + pstar; F[2] = rs * ustar * w[2];
      F[3] = ustar * (cp * pstar + 0.5 * rs * (ustar * ustar + w[2] * w[2]));
    }
  } else {
    const double* w = wR;
    if (pstar <= w[3] && w[1] + w[4] <= 0.0) upwind(qnR, wR);
    else if (pstar <= w[3] && w[1] + w[4] >= 0.0 && ustar + w[4] * std::pow(pstar / w[3], 0.5 / cp) >= 0.0) {
      const double rs = w[0] * std::pow(pstar / w[3], 1.0 / gamma);
      F[0] = rs * ustar; F[1] = rs * ustar * ustar + pstar; F[2] = F[0] * w[2];
      F[3] = ustar * (cp * pstar + 0.5 * rs * (ustar * ustar + w[2] * w[2]));
    } else if (pstar <= w[3] && w[1] + w[4] > 0.0 && ustar + w[4] * std::pow(pstar / w[3], 0.5 / cp) < 0.0) {
      const double uFan = -2.0 * w[4] / (gamma + 1.0) + (gamma - 1.0) / (gamma + 1.0) * w[1];
      const double rs = w[0] * std::pow(-uFan / w[4], 2.0 * cv);
      const double pFan = w[3] * std::pow(rs / w[0], gamma);
      F[0] = rs * uFan; F[1] = rs * uFan * uFan + pFan; F[2] = rs * uFan * w[2];
      F[3] = uFan * (cp * pFan + 0.5 * rs * (uFan * uFan + w[2] * w[2]));
    } else if (pstar > w[3] && w[1] + w[4] * (0.5 * (gamma + 1.0) / gamma * pstar / w[3] + 0.5 / cp) <= 0.0) {
      upwind(qnR, wR);
    } else if (pstar > w[3] && w[1] + w[4] * ((gamma + 1.0) / (2.0 * gamma) * pstar / w[3] + 0.5 / cp) > 0.0) {
      const double rs = w[0] * ((pstar / w[3] + (gamma - 1.0) / (gamma + 1.0)) / (pstar / w[3] * (gamma - 1.0) / (gamma + 1.0) + 1.0));
      F[0] = rs * ustar; F[1] = rs * ustar * ustar + pstar; F[2] = rs * ustar * w[2];
      F[3] = ustar * (cp * pstar + 0.5 * rs * (ustar * ustar + w[2] * w[2]));
    }
  }
  rotate_back(F, nx, ny);
  for (int k = 0; k < 4; ++k) F[k] *= ph.invSqrtGammaMach;
}

void riemann(const Physics& ph, int which, const double* qL, const double* qR, double nx, double ny, double* F) {
  switch (which) {
    case OR_RIEMANN_ROE: roe(ph, qL, qR, nx, ny, F); break;
    case OR_RIEMANN_HLL: hll(ph, qL, qR, nx, ny, F); break;
    case OR_RIEMANN_EXACT: exact(ph, qL, qR, nx, ny, F); break;
    case OR_RIEMANN_LXF: lxf(ph, qL, qR, nx, ny, F); break;
    default: throw std::runtime_error("unknown Riemann solver");
  }
}

// InviscidFlux (0-D form with invRho products as in the 2-D routine)
void inviscid_flux(const Physics& ph, const double* u, double* f, double* g) {
  const double invRho = 1.0 / u[0];
  const double vx = u[1] * invRho, vy = u[2] * invRho;
  const double p = ph.gm1 * (u[3] - 0.5 * u[1] * vx - 0.5 * u[2] * vy);
  f[0] = u[1]; f[1] = u[1] * vx + p; f[2] = u[1] * vy; f[3] = (u[3] + p) * vx;
  g[0] = u[2]; g[1] = f[2]; g[2] = u[2] * vy + p; g[3] = (u[3] + p) * vy;
  for (int k = 0; k < 4; ++k) { f[k] *= ph.invSqrtGammaMach; g[k] *= ph.invSqrtGammaMach; }
}

double pressure(const Physics& ph, const double* Q) {
  return ph.gm1 * (Q[3] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) / Q[0]);
}

// ---------------------------------------------------------------- zones / BCs
static std::vector<double> dimensionless(const Physics& ph, const double* q) {
  return {q[0] / ph.rho, q[1] / (ph.rho * ph.a), q[2] / (ph.rho * ph.a), q[3] / ph.p};
}

// Dirichlet/Farfield/Outlet constant state: pressure, temperature, Mach, AoA (BC Construct)
static std::vector<double> bc_state(const Oracle& o, const or_bc& b) {
  const Physics& ph = o.ph;
  const double p = b.pressure > 0 ? b.pressure : o.cas.pressure_ref;
  const double T = b.temperature > 0 ? b.temperature : o.cas.temperature_ref;
  const double M = b.mach >= 0 ? b.mach : ph.Mach;
  const double aoa = b.aoa_deg * PI / 180.0;
  const double V = M * std::sqrt(ph.gamma * ph.R * T);
  const double rho = p / (ph.R * T);
  const double q[4] = {rho, rho * V * std::cos(aoa), rho * V * std::sin(aoa), ph.cv * p + 0.5 * rho * V * V};
  return dimensionless(ph, q);
}

void setup_zones(Oracle& o) {
  const int M = o.cas.n_markers;
  o.zones.assign(M + 1, Zone{});
  for (int z = 0; z <= M; ++z) {
    Zone& Z = o.zones[z];
    Z.marker = z;
    for (auto& f : o.ed) if (f.edgeType == z) Z.edges.push_back(f.id);
    if (z == 0) continue;
    Z.bc = o.bcs[z - 1];
    const int P0 = 0; (void)P0;
    for (int id : Z.edges) {
      Edge& f = o.ed[id];
      f.zone = z;
      const int P = f.P();
      f.riemannOverride = Z.bc.riemann;
      f.viscousBCType.assign(P, VBC_UNDEFINED);
      switch (Z.bc.type) {
        case OR_BC_PERIODIC: break;
        case OR_BC_EULERWALL:
          f.inviscidBCType = WEAK_PRESCRIBED;
          f.FB.assign(4 * P, 0.0); f.uB_own.assign(4 * P, 0.0); f.uB = &f.uB_own;
          f.uSB_own.assign(4 * P, 0.0); f.uSB = &f.uSB_own;
          f.viscousBCType.assign(P, VBC_ADIABATIC);
          break;
        case OR_BC_DIRICHLET:
        case OR_BC_FARFIELD:
        case OR_BC_PRESSUREOUTLET: {
          Z.q = bc_state(o, Z.bc);
          f.inviscidBCType = WEAK_RIEMANN;
          f.uB_own.assign(4 * P, 0.0);
          for (int i = 0; i < P; ++i) for (int k = 0; k < 4; ++k) f.uB_own[4 * i + k] = Z.q[k];
          f.uB = &f.uB_own;
          f.uSB_own.assign(4 * P, 0.0); f.uSB = &f.uSB_own;
          break;
        }
        case OR_BC_VISCOUSWALL:
          viscous_wall_associate(o, Z, f);
          break;
        case OR_BC_NEWDIRICHLET:   // newDirichletBC_Associate; uSB aliases uB (newDirichlet.incf)
          Z.q = bc_state(o, Z.bc);
          f.inviscidBCType = WEAK_RIEMANN;
          f.uB_own.assign(4 * P, 0.0);
          f.uB = &f.uB_own;
          f.uSB = &f.uB_own;
          f.viscousBCType.assign(P, VBC_DIRICHLET);
          break;
        default: throw std::runtime_error("boundary condition not supported by the oracle");
      }
    }
  }
  // periodic linking (Mesh_ConstructZones + Zone_LinkPeriodicZones)
  for (int z = 1; z <= M; ++z) {
    Zone& Z1 = o.zones[z];
    if (Z1.bc.type != OR_BC_PERIODIC || Z1.associated) continue;
    Zone& Z2 = o.zones[Z1.bc.connected_marker];
    const int coord = (Z1.bc.periodic_dir == 1 && Z2.bc.periodic_dir == 1) ? 1 : 0;
    for (int id1 : Z1.edges) {
      Edge& e1 = o.ed[id1];
      for (int id2 : Z2.edges) {
        Edge& e2 = o.ed[id2];
        if (e2.associated) continue;
        const double a1 = o.nodeX[2 * e1.nodes[0] + coord], b1 = o.nodeX[2 * e1.nodes[1] + coord];
        const double a2 = o.nodeX[2 * e2.nodes[0] + coord], b2 = o.nodeX[2 * e2.nodes[1] + coord];
        const bool same = (almost_equal(a1, a2) && almost_equal(b1, b2)) || (almost_equal(a1, b2) && almost_equal(b1, a2));
        if (!same) continue;
        const double dot = e1.dX[0] * e2.dX[0] + e1.dX[1] * e2.dX[1];
        const bool inv = !(dot >= 0.0);
        e1.inverse = e2.inverse = inv;
        e1.associated = e2.associated = true;
        e1.inviscidBCType = e2.inviscidBCType = WEAK_RIEMANN;
        e1.uB = &e2.storage[0].Q; e2.uB = &e1.storage[0].Q;
        e1.periodic_partner = id2; e2.periodic_partner = id1;
        e1.uSB = &e2.storage[0].Q; e2.uSB = &e1.storage[0].Q;
        e1.gB = &e2.storage[0].dQ; e2.gB = &e1.storage[0].dQ;
        e1.viscousBCType.assign(e1.P(), VBC_PERIODIC);
        e2.viscousBCType.assign(e2.P(), VBC_PERIODIC);
      }
    }
    Z1.associated = Z2.associated = true;
  }
}

static void euler_wall_update(const Oracle& o, Edge& f) {
  const Physics& ph = o.ph;
  const int P = f.P();
  const std::vector<double>& Q = f.storage[0].Q;
  for (int i = 0; i < P; ++i) {
    const double nx = f.nx(i), ny = f.ny(i);
    const double* q0 = &Q[4 * i];
    const double rhovn = q0[1] * nx + q0[2] * ny;
    const double rhovt = f.straight_like() ? (-q0[1] * ny + q0[2] * nx) : (q0[1] * ny - q0[2] * nx);
    const double p = ph.gm1 * (q0[3] - 0.5 * (q0[1] * q0[1] + q0[2] * q0[2]) / q0[0]);
    double q[4] = {q0[0], q0[1] - rhovn * nx, q0[2] - rhovn * ny, ph.cv * p + 0.5 * rhovt * rhovt / q0[0]};
    double F[4], G[4];
    // InviscidFlux1D uses invRho products
    inviscid_flux(ph, q, F, G);
    const double dS = f.straight_like() ? f.dS[0] : f.dS[i];
    for (int k = 0; k < 4; ++k) {
      double s = 0.0;
      s = s + F[k] * nx * dS;
      s = s + G[k] * ny * dS;
      f.FB[4 * i + k] = s;
    }
    f.uB_own[4 * i + 0] = q0[0];
    f.uB_own[4 * i + 1] = q0[1] - 2.0 * rhovn * nx;
    f.uB_own[4 * i + 2] = q0[2] - 2.0 * rhovn * ny;
    f.uB_own[4 * i + 3] = q0[3];
    for (int k = 0; k < 4; ++k) f.uSB_own[4 * i + k] = q[k];
  }
}

// newDirichletBC_UpdateSolution (BoundaryConditions/newDirichlet.incf): characteristic in/outflow
// state per node from the zone state (no boundary-condition function).
static double gf_norm2(double a, double b) {   // NORM2 of two values, scaled sum of squares
  double scale = 0.0, ssq = 1.0;
  for (double x : {a, b}) {
    if (x != 0.0) {
      const double ax = std::fabs(x);
      if (scale < ax) { ssq = 1.0 + ssq * (scale / ax) * (scale / ax); scale = ax; }
      else ssq = ssq + (ax / scale) * (ax / scale);
    }
  }
  return scale * std::sqrt(ssq);
}

static void newdirichlet_update(Oracle& o, Zone& Z, Edge& f) {
  const Physics& ph = o.ph;
  const int P = f.P();
  const double gamma = ph.gamma, gm1 = ph.gm1, cp = ph.cp, cv = ph.cv;
  const double* q = Z.q.data();
  const std::vector<double>& Q = f.storage[0].Q;
  for (int i = 0; i < P; ++i) {
    const double uExt = q[1] / q[0], vExt = q[2] / q[0];
    const double nrm = gf_norm2(uExt, vExt);
    const double nInf[2] = {uExt / nrm, vExt / nrm};
    const double pExt = gm1 * (q[3] - 0.5 * (q[1] * uExt + q[2] * vExt));
    const double MExtSq = (uExt * uExt + vExt * vExt) / (gamma * pExt) * q[0];
    const double sExt = pExt / std::pow(q[0], gamma);
    const double ptExt = pExt * std::pow(1.0 + 0.5 * gm1 * MExtSq, cp);
    const double* qL = &Q[4 * i];
    double* uB = &f.uB_own[4 * i];
    const double rhoL = qL[0], uL = qL[1] / rhoL, vL = qL[2] / rhoL;
    const double vnL = uL * f.nx(i) + vL * f.ny(i);
    const double pL = gm1 * (qL[3] - 0.5 * (qL[1] * uL + qL[2] * vL));
    const double aL = std::sqrt(gamma * pL / rhoL);
    const double ML = std::sqrt(uL * uL + vL * vL) / aL;
    int vbc;
    if (vnL <= 0.0) {
      if (ML > 1.0) {
        for (int k = 0; k < 4; ++k) uB[k] = q[k];
      } else {
        const double pR = pL;
        const double rhoR = std::pow(pR / sExt, 1.0 / gamma);
        const double aR = std::sqrt(gamma * pR / rhoR);
        if (Z.bc.nd_mode == 0) {
          uB[0] = q[0]; uB[1] = q[1]; uB[2] = q[2];
          uB[3] = cv * pR + 0.5 * (uB[1] * uB[1] + uB[2] * uB[2]) / uB[0];
        } else {
          double MR;
          if (pR >= ptExt) MR = -std::sqrt(2.0 / gm1 * (std::pow(pR / ptExt, gm1 / gamma) - 1.0));
          else MR = std::sqrt(2.0 / gm1 * (std::pow(ptExt / pR, gm1 / gamma) - 1.0));
          uB[0] = rhoR;
          uB[1] = rhoR * aR * MR * nInf[0];
          uB[2] = rhoR * aR * MR * nInf[1];
          uB[3] = cv * pR + 0.5 * rhoR * aR * aR * MR * MR;
        }
      }
      vbc = VBC_DIRICHLET;
    } else {
      if (ML > 1.0) {
        for (int k = 0; k < 4; ++k) uB[k] = qL[k];
        vbc = VBC_NEUMANN;
      } else {
        uB[0] = qL[0]; uB[1] = qL[1]; uB[2] = qL[2];
        const double pb = Z.bc.nd_outflow_total ? ptExt : pExt;
        uB[3] = cv * (2.0 * pb - pL) + 0.5 * (uB[1] * uL + uB[2] * vL);
        vbc = VBC_DIRICHLET;
      }
    }
    if (o.cas.navier_stokes) f.viscousBCType[i] = vbc;
  }
}

static void update_zones(Oracle& o, double t) {
  for (size_t z = 1; z < o.zones.size(); ++z) {
    Zone& Z = o.zones[z];
    for (int id : Z.edges) {
      Edge& f = o.ed[id];
      switch (Z.bc.type) {
        case OR_BC_EULERWALL: euler_wall_update(o, f); break;
        case OR_BC_DIRICHLET: if (o.cas.navier_stokes) dirichlet_viscous_update(o, Z, f); break;
        case OR_BC_FARFIELD: farfield_update(o, Z, f); break;
        case OR_BC_PRESSUREOUTLET: pressure_outlet_update(o, Z, f); break;
        case OR_BC_VISCOUSWALL: viscous_wall_update(o, Z, f); break;
        case OR_BC_NEWDIRICHLET: newdirichlet_update(o, Z, f); break;
        default: break;
      }
    }
  }
  (void)t;
}

// ---------------------------------------------------------------- traces
static void interpolate_to_boundaries(Oracle& o, bool gradient) {
  // each element writes only its own storage slots: element-parallel
#pragma omp parallel for schedule(static)
  for (size_t ei = 0; ei < o.el.size(); ++ei) {
    Element& e = o.el[ei];
    const int P = e.P;
    const Spectral& s = *e.sp;
    const double* Q = gradient ? &o.dQ[2 * e.offset] : &o.Q[e.offset];
    const int nd = gradient ? 2 : 1;
    for (int side = 1; side <= 4; ++side) {
      Edge& f = o.ed[e.edges[side - 1]];
      EdgeStorage& st = f.storage[e.quadPosition[side - 1]];
      std::vector<double>& out = gradient ? st.dQ : st.Q;
      std::fill(out.begin(), out.end(), 0.0);
      const std::vector<double>& lb = (side == EBOTTOM || side == ELEFT) ? s.lb[0] : s.lb[1];
      for (int d = 0; d < nd; ++d) {
        const double* Qd = Q + size_t(d) * 4 * P * P;   // dQ layout [d][j][i][v]
        for (int i = 0; i < P; ++i)
          for (int l = 0; l < P; ++l) {
            const int node = (side == EBOTTOM || side == ETOP) ? (l * P + i) : (i * P + l);
            for (int k = 0; k < 4; ++k) out[(d * P + i) * 4 + k] += Qd[node * 4 + k] * lb[l];
          }
      }
    }
  }
}

// ---------------------------------------------------------------- weak integrals
// Scalar_StdFace: QDot -= lift of F (element-local order)
static void std_face_sub(Oracle& o, int eIdx, int loc, const double* F) {
  Element& e = o.el[eIdx];
  const int P = e.P;
  const Spectral& s = *e.sp;
  double* QD = &o.QDot[e.offset];
  for (int j = 0; j < P; ++j)
    for (int i = 0; i < P; ++i)
      for (int k = 0; k < 4; ++k) {
        double v = 0.0;
        switch (loc) {
          case EBOTTOM: v = F[4 * i + k] * s.lbw[0][j]; break;
          case ERIGHT:  v = F[4 * j + k] * s.lbw[1][i]; break;
          case ETOP:    v = F[4 * i + k] * s.lbw[1][j]; break;
          case ELEFT:   v = F[4 * j + k] * s.lbw[0][i]; break;
        }
        QD[(j * P + i) * 4 + k] = QD[(j * P + i) * 4 + k] - v;
      }
}

static int solver_for(const Oracle& o, const Edge& f) {
  return (f.is_bdry() && f.riemannOverride != OR_RIEMANN_INTERIOR) ? f.riemannOverride : o.cas.riemann;
}

// ---------------------------------------------------------------- face loops
static void face_interior(Oracle& o, Edge& f, ViscousWork& vw) {
  const Physics& ph = o.ph;
  const int P = f.P();
  const EdgeStorage& sL = f.storage[SLOT_LEFT];
  const EdgeStorage& sR = f.storage[SLOT_RIGHT];
  const int PL = sL.sp->P, PR = sR.sp->P;
  std::vector<double> QL(4 * P, 0.0), QR(4 * P, 0.0);
  // ProjectSolution types 1..6
  if (f.transform[SLOT_LEFT]) {
    for (int l = 0; l <= f.NLow; ++l) for (int i = 0; i < P; ++i) for (int k = 0; k < 4; ++k)
      QL[4 * i + k] = QL[4 * i + k] + f.T_forward[i * PL + l] * sL.Q[4 * l + k];
  } else QL = sL.Q;
  if (f.transform[SLOT_RIGHT]) {
    for (int l = 0; l <= f.NLow; ++l) for (int i = 0; i < P; ++i) for (int k = 0; k < 4; ++k) {
      const int dst = f.inverse ? (P - 1 - i) : i;
      QR[4 * dst + k] = QR[4 * dst + k] + f.T_forward[i * PR + l] * sR.Q[4 * l + k];
    }
  } else if (f.inverse) {
    for (int i = 0; i < P; ++i) for (int k = 0; k < 4; ++k) QR[4 * i + k] = sR.Q[4 * (P - 1 - i) + k];
  } else QR = sR.Q;
  std::vector<double> Fs(4 * P);
  const int rs = o.cas.riemann;
  for (int i = 0; i < P; ++i) {
    double F[4];
    riemann(ph, rs, &QL[4 * i], &QR[4 * i], f.nx(i), f.ny(i), F);
    for (int k = 0; k < 4; ++k) Fs[4 * i + k] = F[k];
  }
  if (o.cas.navier_stokes) viscous_interior_flux(o, f, QL, QR, Fs, vw);
  for (int i = 0; i < P; ++i) {
    const double dS = f.straight_like() ? f.dS[0] : f.dS[i];
    for (int k = 0; k < 4; ++k) Fs[4 * i + k] = Fs[4 * i + k] * dS;
  }
  // ProjectFluxes
  std::vector<double> FL(4 * PL, 0.0), FR(4 * PR, 0.0);
  if (f.transform[SLOT_LEFT]) {
    for (int l = 0; l < P; ++l) for (int i = 0; i <= f.NLow; ++i) for (int k = 0; k < 4; ++k)
      FL[4 * i + k] = FL[4 * i + k] + f.T_backward[i * P + l] * Fs[4 * l + k];
  } else FL = Fs;
  if (f.transform[SLOT_RIGHT]) {
    for (int l = 0; l < P; ++l) for (int i = 0; i <= f.NLow; ++i) for (int k = 0; k < 4; ++k) {
      const int dst = f.inverse ? (f.NLow - i) : i;
      FR[4 * dst + k] = FR[4 * dst + k] - f.T_backward[i * P + l] * Fs[4 * l + k];
    }
  } else if (f.inverse) {
    for (int i = 0; i < P; ++i) for (int k = 0; k < 4; ++k) FR[4 * (P - 1 - i) + k] = -Fs[4 * i + k];
  } else {
    for (int i = 0; i < P; ++i) for (int k = 0; k < 4; ++k) FR[4 * i + k] = -Fs[4 * i + k];
  }
  std_face_sub(o, f.quads[SLOT_LEFT], f.edgeLocation[SLOT_LEFT], FL.data());
  std_face_sub(o, f.quads[SLOT_RIGHT], f.edgeLocation[SLOT_RIGHT], FR.data());
  if (o.cas.navier_stokes) viscous_interior_gradient_faces(o, f, QL, QR, vw);
}

static void face_subdivided(Oracle& o, Edge& f, ViscousWork& vw) {
  const Physics& ph = o.ph;
  const EdgeStorage& sL = f.storage[SLOT_LEFT];
  const EdgeStorage& sRN = f.storage[SLOT_RN];
  const EdgeStorage& sRS = f.storage[SLOT_RS];
  const int PL = sL.sp->P, PRN = sRN.sp->P, PRS = sRS.sp->P, PN = f.spN->P, PS = f.spS->P;
  auto project = [](const std::vector<double>& T, int rows, int cols, const std::vector<double>& Q) {
    std::vector<double> out(4 * rows, 0.0);
    for (int l = 0; l < cols; ++l) for (int i = 0; i < rows; ++i) for (int k = 0; k < 4; ++k)
      out[4 * i + k] = out[4 * i + k] + T[i * cols + l] * Q[4 * l + k];
    return out;
  };
  std::vector<double> QLN = project(f.T_LN_FWD, PN, PL, sL.Q);
  std::vector<double> QLS = project(f.T_LS_FWD, PS, PL, sL.Q);
  std::vector<double> QRN = project(f.T_RN_FWD, PN, PRN, sRN.Q);
  std::vector<double> QRS = project(f.T_RS_FWD, PS, PRS, sRS.Q);
  const bool curved = f.kind == E_CURVED_SUBDIV;
  std::vector<double> FN(4 * PN), FS(4 * PS);
  for (int i = 0; i < PN; ++i) {
    const double nx = curved ? f.normal_N[i] : f.normal_N[0], ny = curved ? f.normal_N[PN + i] : f.normal_N[1];
    riemann(ph, o.cas.riemann, &QLN[4 * i], &QRN[4 * i], nx, ny, &FN[4 * i]);
  }
  for (int i = 0; i < PS; ++i) {
    const double nx = curved ? f.normal_S[i] : f.normal_S[0], ny = curved ? f.normal_S[PS + i] : f.normal_S[1];
    riemann(ph, o.cas.riemann, &QLS[4 * i], &QRS[4 * i], nx, ny, &FS[4 * i]);
  }
  if (o.cas.navier_stokes) viscous_mortar_fluxes(o, f, QLN, QRN, QLS, QRS, FN, FS, vw);
  for (int i = 0; i < PN; ++i) { const double d = curved ? f.dS_N[i] : f.dS_N[0]; for (int k = 0; k < 4; ++k) FN[4 * i + k] *= d; }
  for (int i = 0; i < PS; ++i) { const double d = curved ? f.dS_S[i] : f.dS_S[0]; for (int k = 0; k < 4; ++k) FS[4 * i + k] *= d; }
  std::vector<double> FL(4 * PL, 0.0), FRN(4 * PRN, 0.0), FRS(4 * PRS, 0.0);
  for (int l = 0; l < PN; ++l) for (int i = 0; i < PL; ++i) for (int k = 0; k < 4; ++k)
    FL[4 * i + k] = FL[4 * i + k] + f.T_LN_BKW[i * PN + l] * FN[4 * l + k];
  for (int l = 0; l < PS; ++l) for (int i = 0; i < PL; ++i) for (int k = 0; k < 4; ++k)
    FL[4 * i + k] = FL[4 * i + k] + f.T_LS_BKW[i * PS + l] * FS[4 * l + k];
  for (int l = 0; l < PN; ++l) for (int i = 0; i < PRN; ++i) for (int k = 0; k < 4; ++k)
    FRN[4 * i + k] = FRN[4 * i + k] - f.T_RN_BKW[i * PN + l] * FN[4 * l + k];
  for (int l = 0; l < PS; ++l) for (int i = 0; i < PRS; ++i) for (int k = 0; k < 4; ++k)
    FRS[4 * i + k] = FRS[4 * i + k] - f.T_RS_BKW[i * PS + l] * FS[4 * l + k];
  std_face_sub(o, f.quads[SLOT_LEFT], f.edgeLocation[SLOT_LEFT], FL.data());
  std_face_sub(o, f.quads[SLOT_RN], f.edgeLocation[SLOT_RN], FRN.data());
  std_face_sub(o, f.quads[SLOT_RS], f.edgeLocation[SLOT_RS], FRS.data());
  if (o.cas.navier_stokes) viscous_mortar_gradient_faces(o, f, QLN, QRN, QLS, QRS, vw);
}

static void face_boundary(Oracle& o, Edge& f, ViscousWork& vw) {
  const Physics& ph = o.ph;
  const int P = f.P();
  std::vector<double> Fi(4 * P, 0.0);
  const std::vector<double>& Q = f.storage[0].Q;
  std::vector<double> Qb(4 * P, 0.0);
  if (f.inviscidBCType == WEAK_PRESCRIBED) {
    Fi = f.FB;
  } else {
    const std::vector<double>& uB = *f.uB;
    for (int i = 0; i < P; ++i) for (int k = 0; k < 4; ++k) Qb[4 * i + k] = f.inverse ? uB[4 * (P - 1 - i) + k] : uB[4 * i + k];
    const int rs = solver_for(o, f);
    for (int i = 0; i < P; ++i) {
      riemann(ph, rs, &Q[4 * i], &Qb[4 * i], f.nx(i), f.ny(i), &Fi[4 * i]);
      const double dS = f.straight_like() ? f.dS[0] : f.dS[i];
      for (int k = 0; k < 4; ++k) Fi[4 * i + k] = Fi[4 * i + k] * dS;
    }
  }
  std::vector<double> F = Fi;
  if (o.cas.navier_stokes) viscous_boundary_flux(o, f, F, vw);
  std_face_sub(o, f.quads[0], f.edgeLocation[0], F.data());
  if (o.cas.navier_stokes) viscous_boundary_gradient_face(o, f, vw);
}

// ---------------------------------------------------------------- volume
static void volume_loop(Oracle& o, Element& e, ViscousWork& vw) {
  const Physics& ph = o.ph;
  const int P = e.P;
  const Spectral& s = *e.sp;
  const double* Q = &o.Q[e.offset];
  std::vector<double> F(size_t(P) * P * 8);   // [(node)*8 + dim*4 + k]
  for (int q = 0; q < P * P; ++q) inviscid_flux(ph, &Q[4 * q], &F[q * 8], &F[q * 8 + 4]);
  if (o.cas.navier_stokes) viscous_volume_flux(o, e, F, vw);
  if (o.cas.navier_stokes) av_volume_flux(o, e, F);
  std::vector<double> Fc(4 * P * P, 0.0), Gc(4 * P * P, 0.0);
  for (int d = 0; d < 2; ++d)
    for (int q = 0; q < P * P; ++q)
      for (int k = 0; k < 4; ++k) Fc[4 * q + k] = Fc[4 * q + k] + F[q * 8 + d * 4 + k] * e.Ja[q * 4 + d * 2 + 0];
  for (int d = 0; d < 2; ++d)
    for (int q = 0; q < P * P; ++q)
      for (int k = 0; k < 4; ++k) Gc[4 * q + k] = Gc[4 * q + k] + F[q * 8 + d * 4 + k] * e.Ja[q * 4 + d * 2 + 1];
  double* QD = &o.QDot[e.offset];
  for (int q = 0; q < 4 * P * P; ++q) QD[q] = 0.0;
  for (int l = 0; l < P; ++l)
    for (int j = 0; j < P; ++j)
      for (int i = 0; i < P; ++i)
        for (int k = 0; k < 4; ++k) {
          const int q = j * P + i;
          QD[4 * q + k] = QD[4 * q + k] + s.hatD[i * P + l] * Fc[4 * (j * P + l) + k] + s.hatD[j * P + l] * Gc[4 * (l * P + i) + k];
        }
}

void time_derivative(Oracle& o, double t) {
  ViscousWork vw;
  interpolate_to_boundaries(o, false);
  update_zones(o, t);
  if (o.cas.navier_stokes) {
    compute_av_viscosity(o);
    set_physical_av(o);
    compute_gradient(o, vw);
    interpolate_to_boundaries(o, true);
  }
#pragma omp parallel for schedule(static)
  for (size_t ei = 0; ei < o.el.size(); ++ei) {
    ViscousWork w;
    volume_loop(o, o.el[ei], w);
  }
  for (auto& f : o.ed) {
    switch (f.kind) {
      case E_STRAIGHT: case E_CURVED: face_interior(o, f, vw); break;
      case E_SUBDIV: case E_CURVED_SUBDIV: face_subdivided(o, f, vw); break;
      default: face_boundary(o, f, vw); break;
    }
  }
#pragma omp parallel for schedule(static)
  for (size_t ei = 0; ei < o.el.size(); ++ei) {
    Element& e = o.el[ei];
    double* QD = &o.QDot[e.offset];
    for (int q = 0; q < e.P * e.P; ++q)
      for (int k = 0; k < 4; ++k) QD[4 * q + k] = QD[4 * q + k] / e.jac[q];
  }
}

}  // namespace orc
