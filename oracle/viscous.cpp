/*
 * viscous.cpp -- Navier-Stokes terms of the oracle (TEST INFRASTRUCTURE).
 *
 * Restates (artificial dissipation switched off: element and edge mu_a = 0, Fa = 0,
 * ArtificialDissipation_t base class, DGArtificialDissipation.f90:100-206):
 *   viscousFlux / AdiabaticViscousFlux     Physics/ViscousFluxes.f90:39-330
 *   BR1_ComputeGradient, dQ face loops,
 *   BR1 Riemann solvers                    Approximation/DGViscous_BR1.f90:48-441
 *   ComputeSolutionRiemann_* (u* lifting)  Approximation/DGViscousMethods.f90:538-917
 *   IP_ComputeGradient (ComputeInteriorGradient, Mesh/QuadElement_QuadProcedures.incf:42-88),
 *   IP Riemann / gradient Riemann solvers  Approximation/DGViscous_IP.f90:45-313
 *   Vector_StdVolumeGreen / Vector_StdFace / Scalar_StdGradientFace
 *                                          Approximation/DGWeakIntegrals.f90:268-622
 *   viscous parts of ComputeRiemannSolver_{Interior,CurvedInterior,Subdivided,
 *   CurvedSubdivided,StraightBdry,CurvedBdry}Edge
 *                                          Approximation/DGSpatialDiscretizationMethods.f90:545-1511
 *   ViscousWall / Dirichlet / Farfield / PressureOutlet UpdateSolution
 *                                          BoundaryConditions/{ViscousWall,Dirichlet,Farfield,PressureOutlet}.incf
 * Deviations from the reference, where its behaviour is undefined:
 *   - Farfield zones never set viscousBCType (Farfield.incf Associate/UpdateSolution),
 *     so the reference reads an unassigned viscous flux on far-field edges; here the
 *     far-field viscous condition is Neumann (zero viscous and gradient-face flux).
 *   - The straight-edge supersonic-outflow branch of FarfieldBC_UpdateSolution writes
 *     uB with swapped indices (Farfield.incf:246); here uB = interior trace, as in the
 *     curved-edge branch.
 */
#include "viscous.h"
#include <stdexcept>
#include <algorithm>

namespace orc {

// ------------------------------------------------------------------ fluxes
// viscousFlux0D/1D/2D: F[k][d] from q and dq (dq[d][k])
static void vflux(const Physics& ph, const double* q, const double* dqx, const double* dqy, double* Fx, double* Fy) {
  const double invRho = 1.0 / q[0];
  const double u = q[1] * invRho, v = q[2] * invRho;
  const double uDivRho = u * invRho, vDivRho = v * invRho;
  const double lambda = ph.lambda, gm1 = ph.gm1;
  const double divV = -uDivRho * dqx[0] + invRho * dqx[1] - vDivRho * dqy[0] + invRho * dqy[2];
  const double dxT = gm1 * invRho * (-q[3] * invRho * dqx[0] + dqx[3] + u * (u * dqx[0] - dqx[1]) + v * (v * dqx[0] - dqx[2]));
  const double dyT = gm1 * invRho * (-q[3] * invRho * dqy[0] + dqy[3] + u * (u * dqy[0] - dqy[1]) + v * (v * dqy[0] - dqy[2]));
  const double cpPr = ph.cp / ph.Pr;
  Fx[0] = 0.0;
  Fx[1] = 2.0 * (-uDivRho * dqx[0] + invRho * dqx[1]) + lambda * divV;
  Fx[2] = -vDivRho * dqx[0] - uDivRho * dqy[0] + invRho * dqy[1] + invRho * dqx[2];
  Fx[3] = u * Fx[1] + v * Fx[2] + cpPr * dxT;
  Fy[0] = 0.0;
  Fy[1] = Fx[2];
  Fy[2] = 2.0 * (-vDivRho * dqy[0] + invRho * dqy[2]) + lambda * divV;
  Fy[3] = u * Fy[1] + v * Fy[2] + cpPr * dyT;
}

// AdiabaticViscousFlux1D/2D (qB = the state whose velocity carries the work term)
static void vflux_adiabatic(const Physics& ph, const double* q, const double* qB, const double* dqx, const double* dqy,
                            double* Fx, double* Fy) {
  const double invRho = 1.0 / q[0];
  const double u = q[1] * invRho, v = q[2] * invRho;
  const double uDivRho = u * invRho, vDivRho = v * invRho;
  const double lambda = ph.lambda;
  const double divV = -uDivRho * dqx[0] + invRho * dqx[1] - vDivRho * dqy[0] + invRho * dqy[2];
  Fx[0] = 0.0;
  Fx[1] = 2.0 * (-uDivRho * dqx[0] + invRho * dqx[1]) + lambda * divV;
  Fx[2] = -vDivRho * dqx[0] - uDivRho * dqy[0] + invRho * dqy[1] + invRho * dqx[2];
  Fx[3] = (qB[1] * Fx[1] + qB[2] * Fx[2]) / qB[0];
  Fy[0] = 0.0;
  Fy[1] = Fx[2];
  Fy[2] = 2.0 * (-vDivRho * dqy[0] + invRho * dqy[2]) + lambda * divV;
  Fy[3] = (qB[1] * Fy[1] + qB[2] * Fy[2]) / qB[0];
}

static bool is_ip(const Oracle& o) { return o.cas.viscous == OR_VISC_IP; }
static double ip_epsilon(const Oracle& o) {
  return o.cas.ip_method == OR_IP_SIPG ? -1.0 : (o.cas.ip_method == OR_IP_NIPG ? 1.0 : 0.0);
}
static bool gradient_faces(const Oracle& o) { return is_ip(o) && o.cas.ip_method != OR_IP_IIPG; }

// ------------------------------------------------------------------ helpers
// edge-local arrays: [i*4+k] values, gradients [(d*P+i)*4+k]
struct EdgeArrays {
  int P = 0;
  std::vector<double> Q, dQ;
};

// viscous Riemann flux at one point (BR1 / IP interior form), including mu: Fstar[k]
static void visc_riemann(const Oracle& o, double mu_a, int N, double invh, const double* qL, const double* qR,
                         const double* dqLx, const double* dqLy, const double* dqRx, const double* dqRy, double nx,
                         double ny, double* Fs) {
  const Physics& ph = o.ph;
  const double mu = ph.mu + mu_a;
  double FLx[4], FLy[4], FRx[4], FRy[4];
  vflux(ph, qL, dqLx, dqLy, FLx, FLy);
  vflux(ph, qR, dqRx, dqRy, FRx, FRy);
  for (int k = 0; k < 4; ++k) {
    FLx[k] *= mu; FLy[k] *= mu; FRx[k] *= mu; FRy[k] *= mu;
    double s = 0.0;
    s = s + 0.5 * (FLx[k] + FRx[k]) * nx;
    s = s + 0.5 * (FLy[k] + FRy[k]) * ny;
    Fs[k] = s;
  }
  if (is_ip(o)) {
    const double penalty = o.cas.sigma0_ip * mu * N * N * invh;
    for (int k = 0; k < 4; ++k) Fs[k] = Fs[k] - penalty * (qL[k] - qR[k]);
  }
}

// IP_GradientRiemannSolver at one point: GL[d][k], GR[d][k]
static void visc_gradient_riemann(const Oracle& o, double mu_a, const double* qL, const double* qR, double nx, double ny,
                                  double* GLx, double* GLy, double* GRx, double* GRy) {
  const Physics& ph = o.ph;
  double fgx[4], fgy[4];
  for (int k = 0; k < 4; ++k) { fgx[k] = (qL[k] - qR[k]) * nx; fgy[k] = (qL[k] - qR[k]) * ny; }
  const double eps = ip_epsilon(o);
  const double cL = 0.5 * eps * (ph.mu + mu_a), cR = -0.5 * eps * (ph.mu + mu_a);
  vflux(ph, qL, fgx, fgy, GLx, GLy);
  vflux(ph, qR, fgx, fgy, GRx, GRy);
  for (int k = 0; k < 4; ++k) { GLx[k] *= cL; GLy[k] *= cL; GRx[k] *= cR; GRy[k] *= cR; }
}

// Vector_StdFace: dQ(element) += lift of Fu (element-local order), Fu[(d*P+i)*4+k]
static void vector_face_add(Oracle& o, int eIdx, int loc, const double* Fu) {
  Element& e = o.el[eIdx];
  const int P = e.P;
  const Spectral& s = *e.sp;
  double* dQ = &o.dQ[2 * e.offset];
  for (int d = 0; d < 2; ++d)
    for (int j = 0; j < P; ++j)
      for (int i = 0; i < P; ++i)
        for (int k = 0; k < 4; ++k) {
          double v = 0.0;
          switch (loc) {
            case EBOTTOM: v = Fu[(d * P + i) * 4 + k] * s.lbw[0][j]; break;
            case ERIGHT:  v = Fu[(d * P + j) * 4 + k] * s.lbw[1][i]; break;
            case ETOP:    v = Fu[(d * P + i) * 4 + k] * s.lbw[1][j]; break;
            case ELEFT:   v = Fu[(d * P + j) * 4 + k] * s.lbw[0][i]; break;
          }
          double& t = dQ[(size_t(d) * P * P + j * P + i) * 4 + k];
          t = t + v;
        }
}

// Scalar_StdGradientFace: QDot(element) -= lift of G (element-local order), G[(d*P+i)*4+k]
static void gradient_face_sub(Oracle& o, int eIdx, int loc, const double* G) {
  Element& e = o.el[eIdx];
  const int P = e.P;
  const Spectral& s = *e.sp;
  const bool alongXi = (loc == EBOTTOM || loc == ETOP);
  const int side = (loc == EBOTTOM || loc == ELEFT) ? 0 : 1;
  const std::vector<double>& lb = s.lb[side];
  // metrics interpolated to the face: Ja(:, dim, c), jac as functions of the face coordinate
  std::vector<double> Jxi(2 * P), Jeta(2 * P), jf(P);
  for (int a = 0; a < P; ++a) {
    double sxi[2] = {0, 0}, seta[2] = {0, 0}, sj = 0;
    for (int b = 0; b < P; ++b) {
      const int q = alongXi ? (b * P + a) : (a * P + b);   // interpolate along the other direction
      for (int d = 0; d < 2; ++d) {
        sxi[d] += e.Ja[q * 4 + d * 2 + 0] * lb[b];
        seta[d] += e.Ja[q * 4 + d * 2 + 1] * lb[b];
      }
      sj += e.jac[q] * lb[b];
    }
    for (int d = 0; d < 2; ++d) { Jxi[d * P + a] = sxi[d]; Jeta[d * P + a] = seta[d]; }
    jf[a] = sj;
  }
  std::vector<double> Fc(4 * P, 0.0), Gc(4 * P, 0.0);
  for (int d = 0; d < 2; ++d)
    for (int i = 0; i < P; ++i)
      for (int k = 0; k < 4; ++k) Fc[4 * i + k] = Fc[4 * i + k] + G[(d * P + i) * 4 + k] * Jxi[d * P + i];
  for (int i = 0; i < P; ++i) for (int k = 0; k < 4; ++k) Fc[4 * i + k] = Fc[4 * i + k] / jf[i];
  for (int d = 0; d < 2; ++d)
    for (int i = 0; i < P; ++i)
      for (int k = 0; k < 4; ++k) Gc[4 * i + k] = Gc[4 * i + k] + G[(d * P + i) * 4 + k] * Jeta[d * P + i];
  for (int i = 0; i < P; ++i) for (int k = 0; k < 4; ++k) Gc[4 * i + k] = Gc[4 * i + k] / jf[i];
  std::vector<double> dd(4 * P, 0.0);
  const std::vector<double>& src = alongXi ? Fc : Gc;
  for (int l = 0; l < P; ++l)
    for (int i = 0; i < P; ++i)
      for (int k = 0; k < 4; ++k) dd[4 * i + k] = dd[4 * i + k] + s.hatD[i * P + l] * src[4 * l + k];
  double* QD = &o.QDot[e.offset];
  for (int j = 0; j < P; ++j)
    for (int i = 0; i < P; ++i)
      for (int k = 0; k < 4; ++k) {
        double v;
        if (alongXi) v = dd[4 * i + k] * s.lbw[side][j] + Gc[4 * i + k] * s.dlbw[side][j];
        else v = Fc[4 * j + k] * s.dlbw[side][i] + dd[4 * j + k] * s.lbw[side][i];
        QD[(j * P + i) * 4 + k] = QD[(j * P + i) * 4 + k] - v;
      }
}

// project element-ordered traces to the edge (types 1..6); nb = number of [P][4] blocks
static std::vector<double> project_to_edge(const Edge& f, int slot, const std::vector<double>& src, int nb) {
  const int P = f.P();
  const int Ps = f.storage[slot].sp->P;
  std::vector<double> out(size_t(nb) * 4 * P, 0.0);
  const bool tr = f.transform[slot];
  const bool rev = (slot == SLOT_RIGHT) && f.inverse;
  for (int b = 0; b < nb; ++b) {
    if (tr) {
      for (int l = 0; l <= f.NLow; ++l)
        for (int i = 0; i < P; ++i) {
          const int dst = rev ? (P - 1 - i) : i;
          for (int k = 0; k < 4; ++k)
            out[(b * P + dst) * 4 + k] = out[(b * P + dst) * 4 + k] + f.T_forward[i * Ps + l] * src[(b * Ps + l) * 4 + k];
        }
    } else {
      for (int i = 0; i < P; ++i) {
        const int s_ = rev ? (P - 1 - i) : i;
        for (int k = 0; k < 4; ++k) out[(b * P + i) * 4 + k] = src[(b * Ps + s_) * 4 + k];
      }
    }
  }
  return out;
}

// edge -> element projection of fluxes (ProjectFluxes when negate, ProjectGradientFluxes otherwise)
static std::vector<double> project_to_elem(const Edge& f, int slot, const std::vector<double>& F, int nb, bool negate) {
  const int P = f.P();
  const int Ps = f.storage[slot].sp->P;
  std::vector<double> out(size_t(nb) * 4 * Ps, 0.0);
  const bool tr = f.transform[slot];
  const bool rev = (slot == SLOT_RIGHT) && f.inverse;
  const double sg = negate ? -1.0 : 1.0;
  for (int b = 0; b < nb; ++b) {
    if (tr) {
      for (int l = 0; l < P; ++l)
        for (int i = 0; i <= f.NLow; ++i) {
          const int dst = rev ? (f.NLow - i) : i;
          for (int k = 0; k < 4; ++k) {
            double& t = out[(b * Ps + dst) * 4 + k];
            if (negate) t = t - f.T_backward[i * P + l] * F[(b * P + l) * 4 + k];
            else t = t + f.T_backward[i * P + l] * F[(b * P + l) * 4 + k];
          }
        }
    } else {
      for (int i = 0; i < P; ++i) {
        const int dst = rev ? (P - 1 - i) : i;
        for (int k = 0; k < 4; ++k) out[(b * Ps + dst) * 4 + k] = sg * F[(b * P + i) * 4 + k];
      }
    }
  }
  return out;
}

// ------------------------------------------------------------------ BCs
void viscous_wall_associate(Oracle& o, Zone& Z, Edge& f) {
  const int P = f.P();
  f.inviscidBCType = WEAK_RIEMANN;
  f.uB_own.assign(4 * P, 0.0); f.uB = &f.uB_own;
  f.uSB_own.assign(4 * P, 0.0); f.uSB = &f.uSB_own;
  f.viscousBCType.assign(P, Z.bc.wall_type == 1 ? VBC_DIRICHLET : VBC_ADIABATIC);
  (void)o;
}

void viscous_wall_update(Oracle& o, Zone& Z, Edge& f) {
  const Physics& ph = o.ph;
  const int P = f.P();
  const std::vector<double>& Q = f.storage[0].Q;
  // wall velocity: sqrt(gamma) * Mach_wall * direction (ViscousWall_Construct); Tw / T_ref
  const double vx = Z.bc.wall_v[0], vy = Z.bc.wall_v[1];
  const double Tw = Z.bc.wall_T / o.cas.temperature_ref;
  const bool iso = Z.bc.wall_type == 1;
  for (int i = 0; i < P; ++i) {
    const double* q = &Q[4 * i];
    double* uB = &f.uB_own[4 * i];
    uB[0] = q[0];
    uB[1] = 2.0 * uB[0] * vx - q[1];
    uB[2] = 2.0 * uB[0] * vy - q[2];
    const double Ek = 0.5 * (uB[1] * uB[1] + uB[2] * uB[2]) / uB[0];
    uB[3] = iso ? ph.cv * uB[0] * 1.0 * Tw + Ek : q[3];
    double* uS = &f.uSB_own[4 * i];
    uS[0] = q[0];
    uS[1] = uS[0] * vx;
    uS[2] = uS[0] * vy;
    if (iso) uS[3] = ph.cv * uS[0] * 1.0 * Tw + 0.5 * (uS[1] * uS[1] + uS[2] * uS[2]) / uS[0];
    else uS[3] = q[3] - Ek + 0.5 * uS[0] * (vx * vx + vy * vy);
  }
}

void dirichlet_viscous_update(Oracle& o, Zone& Z, Edge& f) {
  const Physics& ph = o.ph;
  const int P = f.P();
  const std::vector<double>& Q = f.storage[0].Q;
  for (int i = 0; i < P; ++i) {
    const double* q = &Q[4 * i];
    const double* uB = &f.uB_own[4 * i];
    double* uS = &f.uSB_own[4 * i];
    const double rhoL = q[0], uL = q[1] / rhoL, vL = q[2] / rhoL;
    const double vnL = uL * f.nx(i) + vL * f.ny(i);
    const double pL = ph.gm1 * (q[3] - 0.5 * (q[1] * uL + q[2] * vL));
    const double aL = std::sqrt(ph.gamma * pL / rhoL);
    const double ML = std::sqrt(uL * uL + vL * vL) / aL;
    if (vnL <= 0.0) {
      if (ML > 1.0) { for (int k = 0; k < 4; ++k) uS[k] = uB[k]; }
      else {
        const double pR = pL;
        uS[0] = uB[0]; uS[1] = uB[1]; uS[2] = uB[2];
        uS[3] = ph.cv * pR + 0.5 * (uS[1] * uS[1] + uS[2] * uS[2]) / uS[0];
      }
      f.viscousBCType[i] = VBC_DIRICHLET;
    } else {
      if (ML > 1.0) { for (int k = 0; k < 4; ++k) uS[k] = q[k]; f.viscousBCType[i] = VBC_NEUMANN; }
      else {
        uS[0] = q[0]; uS[1] = q[1]; uS[2] = q[2];
        uS[3] = ph.cv * pressure(ph, uB) + 0.5 * (uS[1] * uL + uS[2] * vL);
        f.viscousBCType[i] = VBC_DIRICHLET;
      }
    }
  }
  (void)Z;
}

void farfield_update(Oracle& o, Zone& Z, Edge& f) {
  const Physics& ph = o.ph;
  const int P = f.P();
  const std::vector<double>& Q = f.storage[0].Q;
  const double* q = Z.q.data();
  const double rhoI = q[0], uI = q[1] / rhoI, vI = q[2] / rhoI;
  const double pI = ph.gm1 * (q[3] - 0.5 * q[1] * uI - 0.5 * q[2] * vI);
  for (int i = 0; i < P; ++i) {
    const double* qL = &Q[4 * i];
    double* uB = &f.uB_own[4 * i];
    const double nx = f.nx(i), ny = f.ny(i);
    const double rhoL = qL[0], uL = qL[1] / rhoL, vL = qL[2] / rhoL;
    const double vnL = uL * nx + vL * ny;
    const double pL = ph.gm1 * (qL[3] - 0.5 * qL[1] * uL - 0.5 * qL[2] * vL);
    const double aL = std::sqrt(ph.gamma * pL / rhoL);
    const double ML = std::sqrt(uL * uL + vL * vL) / aL;
    if (vnL < 0.0) {
      if (ML > 1.0) { for (int k = 0; k < 4; ++k) uB[k] = q[k]; }
      else {
        const double pR = 0.5 * (pL + pI - rhoL * aL * (nx * (uL - uI) + ny * (vL - vI)));
        const double rhoR = rhoI + (pR - pI) / (aL * aL);
        const double uR = uI + nx * (pR - pI) / (aL * rhoL);
        const double vR = vI + ny * (pR - pI) / (aL * rhoL);
        uB[0] = rhoR; uB[1] = rhoR * uR; uB[2] = rhoR * vR;
        uB[3] = ph.cv * pR + 0.5 * (uB[1] * uR + uB[2] * vR);
      }
    } else {
      if (ML > 1.0) { for (int k = 0; k < 4; ++k) uB[k] = qL[k]; }
      else {
        const double pR = pI;
        const double rhoR = rhoL + (pI - pL) / (aL * aL);
        const double uR = uL - nx * (pI - pL) / (rhoL * aL);
        const double vR = vL - ny * (pI - pL) / (rhoL * aL);
        uB[0] = rhoR; uB[1] = rhoR * uR; uB[2] = rhoR * vR;
        uB[3] = ph.cv * pR + 0.5 * (uB[1] * uR + uB[2] * vR);
      }
    }
    if (o.cas.navier_stokes) {
      for (int k = 0; k < 4; ++k) f.uSB_own[4 * i + k] = uB[k];
      f.viscousBCType[i] = VBC_NEUMANN;
    }
  }
}

void pressure_outlet_update(Oracle& o, Zone& Z, Edge& f) {
  const Physics& ph = o.ph;
  const int P = f.P();
  const std::vector<double>& Q = f.storage[0].Q;
  const double* q = Z.q.data();
  const double rhoI = q[0], uI = q[1] / rhoI, vI = q[2] / rhoI;
  const double pI = ph.gm1 * (q[3] - 0.5 * q[1] * uI - 0.5 * q[2] * vI);
  const double nrm = std::sqrt(uI * uI + vI * vI);
  const double nIx = uI / nrm, nIy = vI / nrm;
  const bool reflective = Z.bc.outflow_type != 2;
  for (int i = 0; i < P; ++i) {
    const double* qL = &Q[4 * i];
    double* uB = &f.uB_own[4 * i];
    double* uS = &f.uSB_own[4 * i];
    const double nx = f.nx(i), ny = f.ny(i);
    const double rhoL = qL[0], uL = qL[1] / rhoL, vL = qL[2] / rhoL;
    const double vnL = uL * nx + vL * ny;
    const double pL = ph.gm1 * (qL[3] - 0.5 * qL[1] * uL - 0.5 * qL[2] * vL);
    const double aL = std::sqrt(ph.gamma * pL / rhoL);
    const double ML = std::sqrt(uL * uL + vL * vL) / aL;
    int vbc;
    if (vnL < 0.0 && ML > 1.0) {
      for (int k = 0; k < 4; ++k) { uB[k] = q[k]; uS[k] = q[k]; }
      vbc = VBC_DIRICHLET;
    } else if (vnL >= 0.0 && ML > 1.0) {
      for (int k = 0; k < 4; ++k) { uB[k] = qL[k]; uS[k] = qL[k]; }
      vbc = VBC_NEUMANN;
    } else {
      double rhoR, uR, vR, pR;
      if (reflective) {
        const double R0 = pL - aL * aL * rhoL;
        const double Rplus = vnL + 2.0 * ph.cv * aL;
        rhoR = -(R0 - pI) / (aL * aL);
        const double aR = std::sqrt(ph.gamma * pI / rhoR);
        const double vnR = Rplus - 2.0 * aR * ph.cv;
        uR = uL + (vnR - vnL) * nx;
        vR = vL + (vnR - vnL) * ny;
        pR = pI;
      } else if (vnL < 0.0) {
        pR = 2.0 * pI - pL; uR = std::fabs(vnL) * nIx; vR = std::fabs(vnL) * nIy; rhoR = rhoL;
      } else {
        pR = 2.0 * pI - pL; uR = uL; vR = vL; rhoR = rhoL;
      }
      uB[0] = rhoR; uB[1] = rhoR * uR; uB[2] = rhoR * vR;
      uB[3] = ph.cv * pR + 0.5 * (uB[1] * uR + uB[2] * vR);
      if (vnL < 0.0) { for (int k = 0; k < 4; ++k) uS[k] = uB[k]; }
      else {
        uS[0] = rhoL; uS[1] = rhoL * uL; uS[2] = rhoL * vL; uS[3] = ph.cv * pR + 0.5 * rhoL * (uL * uL + vL * vL);
      }
      vbc = VBC_DIRICHLET;
    }
    if (o.cas.navier_stokes) f.viscousBCType[i] = vbc;
  }
}

// ------------------------------------------------------------------ gradient
static void vector_volume_green(Oracle& o, Element& e, double* dQ) {
  const int P = e.P;
  const Spectral& s = *e.sp;
  const double* Q = &o.Q[e.offset];
  std::vector<double> vol(size_t(2) * P * P * 4, 0.0);
  for (int d = 0; d < 2; ++d)
    for (int j = 0; j < P; ++j)
      for (int l = 0; l < P; ++l)
        for (int i = 0; i < P; ++i)
          for (int k = 0; k < 4; ++k) {
            double& t = vol[(size_t(d) * P * P + j * P + i) * 4 + k];
            t = t + Q[(j * P + l) * 4 + k] * e.Ja[(j * P + l) * 4 + d * 2 + 0] * s.hatD[i * P + l];
          }
  for (int d = 0; d < 2; ++d)
    for (int l = 0; l < P; ++l)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i)
          for (int k = 0; k < 4; ++k) {
            double& t = vol[(size_t(d) * P * P + j * P + i) * 4 + k];
            t = t + Q[(l * P + i) * 4 + k] * e.Ja[(l * P + i) * 4 + d * 2 + 1] * s.hatD[j * P + l];
          }
  for (size_t n = 0; n < vol.size(); ++n) dQ[n] = -vol[n];
}

void interior_gradient(Oracle& o, Element& e, double* dQ) {
  const int P = e.P;
  const Spectral& s = *e.sp;
  const double* Q = &o.Q[e.offset];
  std::vector<double> dxi(4 * P * P, 0.0), deta(4 * P * P, 0.0);
  for (int j = 0; j < P; ++j) for (int l = 0; l < P; ++l) for (int i = 0; i < P; ++i) for (int k = 0; k < 4; ++k)
    dxi[(j * P + i) * 4 + k] = dxi[(j * P + i) * 4 + k] + s.D[i * P + l] * Q[(j * P + l) * 4 + k];
  for (int j = 0; j < P; ++j) for (int l = 0; l < P; ++l) for (int i = 0; i < P; ++i) for (int k = 0; k < 4; ++k)
    deta[(j * P + i) * 4 + k] = deta[(j * P + i) * 4 + k] + s.D[j * P + l] * Q[(l * P + i) * 4 + k];
  for (int i = 0; i < P; ++i)
    for (int j = 0; j < P; ++j) {
      const int q = j * P + i;
      for (int k = 0; k < 4; ++k) {
        dQ[(0 * P * P + q) * 4 + k] = (dxi[q * 4 + k] * e.Ja[q * 4 + 0] + deta[q * 4 + k] * e.Ja[q * 4 + 1]) / e.jac[q];
        dQ[(size_t(1) * P * P + q) * 4 + k] = (dxi[q * 4 + k] * e.Ja[q * 4 + 2] + deta[q * 4 + k] * e.Ja[q * 4 + 3]) / e.jac[q];
      }
    }
}

static void br1_face(Oracle& o, Edge& f) {
  const int P = f.P();
  if (f.is_bdry()) {
    std::vector<double> us(4 * P);
    if (f.associated) {
      const std::vector<double>& uB = *f.uB;
      for (int i = 0; i < P; ++i)
        for (int k = 0; k < 4; ++k) {
          const double qR = f.inverse ? uB[4 * (P - 1 - i) + k] : uB[4 * i + k];
          us[4 * i + k] = 0.5 * (f.storage[0].Q[4 * i + k] + qR);
        }
    } else {
      us = *f.uSB;
    }
    std::vector<double> Fu(8 * P);
    for (int d = 0; d < 2; ++d)
      for (int i = 0; i < P; ++i) {
        const double dS = f.straight_like() ? f.dS[0] : f.dS[i];
        const double n = d == 0 ? f.nx(i) : f.ny(i);
        for (int k = 0; k < 4; ++k) Fu[(d * P + i) * 4 + k] = us[4 * i + k] * dS * n;
      }
    vector_face_add(o, f.quads[0], f.edgeLocation[0], Fu.data());
    return;
  }
  if (f.is_subdiv()) {
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
    std::vector<double> QLN = project(f.T_LN_FWD, PN, PL, sL.Q), QLS = project(f.T_LS_FWD, PS, PL, sL.Q);
    std::vector<double> QRN = project(f.T_RN_FWD, PN, PRN, sRN.Q), QRS = project(f.T_RS_FWD, PS, PRS, sRS.Q);
    std::vector<double> uN(4 * PN), uS(4 * PS);
    for (int n = 0; n < 4 * PN; ++n) uN[n] = 0.5 * (QLN[n] + QRN[n]);
    for (int n = 0; n < 4 * PS; ++n) uS[n] = 0.5 * (QLS[n] + QRS[n]);
    std::vector<double> FL(8 * PL, 0.0), FRN(8 * PRN, 0.0), FRS(8 * PRS, 0.0);
    if (f.kind == E_SUBDIV) {
      std::vector<double> uL(4 * PL, 0.0), uRN(4 * PRN, 0.0), uRS(4 * PRS, 0.0);
      for (int l = 0; l < PN; ++l) for (int i = 0; i < PL; ++i) for (int k = 0; k < 4; ++k)
        uL[4 * i + k] = uL[4 * i + k] + 0.5 * f.T_LN_BKW[i * PN + l] * uN[4 * l + k];
      for (int l = 0; l < PS; ++l) for (int i = 0; i < PL; ++i) for (int k = 0; k < 4; ++k)
        uL[4 * i + k] = uL[4 * i + k] + 0.5 * f.T_LS_BKW[i * PS + l] * uS[4 * l + k];
      for (int l = 0; l < PN; ++l) for (int i = 0; i < PRN; ++i) for (int k = 0; k < 4; ++k)
        uRN[4 * i + k] = uRN[4 * i + k] + f.T_RN_BKW[i * PN + l] * uN[4 * l + k];
      for (int l = 0; l < PS; ++l) for (int i = 0; i < PRS; ++i) for (int k = 0; k < 4; ++k)
        uRS[4 * i + k] = uRS[4 * i + k] + f.T_RS_BKW[i * PS + l] * uS[4 * l + k];
      for (int d = 0; d < 2; ++d) {
        for (int i = 0; i < PL; ++i) for (int k = 0; k < 4; ++k)
          FL[(d * PL + i) * 4 + k] = uL[4 * i + k] * f.dS[0] * f.n[d];
        for (int i = 0; i < PRN; ++i) for (int k = 0; k < 4; ++k)
          FRN[(d * PRN + i) * 4 + k] = -uRN[4 * i + k] * f.dS_N[0] * f.normal_N[d];
        for (int i = 0; i < PRS; ++i) for (int k = 0; k < 4; ++k)
          FRS[(d * PRS + i) * 4 + k] = -uRS[4 * i + k] * f.dS_S[0] * f.normal_S[d];
      }
    } else {
      std::vector<double> FN(8 * PN), FS(8 * PS);
      for (int d = 0; d < 2; ++d) {
        for (int i = 0; i < PN; ++i) for (int k = 0; k < 4; ++k)
          FN[(d * PN + i) * 4 + k] = uN[4 * i + k] * f.dS_N[i] * f.normal_N[d * PN + i];
        for (int i = 0; i < PS; ++i) for (int k = 0; k < 4; ++k)
          FS[(d * PS + i) * 4 + k] = uS[4 * i + k] * f.dS_S[i] * f.normal_S[d * PS + i];
      }
      for (int d = 0; d < 2; ++d) {
        for (int l = 0; l < PN; ++l) for (int i = 0; i < PL; ++i) for (int k = 0; k < 4; ++k)
          FL[(d * PL + i) * 4 + k] = FL[(d * PL + i) * 4 + k] + f.T_LN_BKW[i * PN + l] * FN[(d * PN + l) * 4 + k];
        for (int l = 0; l < PS; ++l) for (int i = 0; i < PL; ++i) for (int k = 0; k < 4; ++k)
          FL[(d * PL + i) * 4 + k] = FL[(d * PL + i) * 4 + k] + f.T_LS_BKW[i * PS + l] * FS[(d * PS + l) * 4 + k];
        for (int l = 0; l < PN; ++l) for (int i = 0; i < PRN; ++i) for (int k = 0; k < 4; ++k)
          FRN[(d * PRN + i) * 4 + k] = FRN[(d * PRN + i) * 4 + k] - f.T_RN_BKW[i * PN + l] * FN[(d * PN + l) * 4 + k];
        for (int l = 0; l < PS; ++l) for (int i = 0; i < PRS; ++i) for (int k = 0; k < 4; ++k)
          FRS[(d * PRS + i) * 4 + k] = FRS[(d * PRS + i) * 4 + k] - f.T_RS_BKW[i * PS + l] * FS[(d * PS + l) * 4 + k];
      }
    }
    vector_face_add(o, f.quads[SLOT_LEFT], f.edgeLocation[SLOT_LEFT], FL.data());
    vector_face_add(o, f.quads[SLOT_RN], f.edgeLocation[SLOT_RN], FRN.data());
    vector_face_add(o, f.quads[SLOT_RS], f.edgeLocation[SLOT_RS], FRS.data());
    return;
  }
  // interior conforming edge
  std::vector<double> QL = project_to_edge(f, SLOT_LEFT, f.storage[SLOT_LEFT].Q, 1);
  std::vector<double> QR = project_to_edge(f, SLOT_RIGHT, f.storage[SLOT_RIGHT].Q, 1);
  std::vector<double> us(4 * P);
  for (int n = 0; n < 4 * P; ++n) us[n] = 0.5 * (QL[n] + QR[n]);
  const int PL = f.storage[SLOT_LEFT].sp->P, PR = f.storage[SLOT_RIGHT].sp->P;
  std::vector<double> FL(8 * PL), FR(8 * PR);
  if (f.kind == E_STRAIGHT) {
    std::vector<double> uL = project_to_elem(f, SLOT_LEFT, us, 1, false);
    std::vector<double> uR = project_to_elem(f, SLOT_RIGHT, us, 1, true);
    for (int d = 0; d < 2; ++d) {
      for (int i = 0; i < PL; ++i) for (int k = 0; k < 4; ++k) FL[(d * PL + i) * 4 + k] = uL[4 * i + k] * f.dS[0] * f.n[d];
      for (int i = 0; i < PR; ++i) for (int k = 0; k < 4; ++k) FR[(d * PR + i) * 4 + k] = uR[4 * i + k] * f.dS[0] * f.n[d];
    }
  } else {
    std::vector<double> Fu(8 * P);
    for (int d = 0; d < 2; ++d)
      for (int i = 0; i < P; ++i)
        for (int k = 0; k < 4; ++k) Fu[(d * P + i) * 4 + k] = us[4 * i + k] * f.dS[i] * (d == 0 ? f.nx(i) : f.ny(i));
    FL = project_to_elem(f, SLOT_LEFT, Fu, 2, false);
    FR = project_to_elem(f, SLOT_RIGHT, Fu, 2, true);
  }
  vector_face_add(o, f.quads[SLOT_LEFT], f.edgeLocation[SLOT_LEFT], FL.data());
  vector_face_add(o, f.quads[SLOT_RIGHT], f.edgeLocation[SLOT_RIGHT], FR.data());
}

void compute_gradient(Oracle& o, ViscousWork& vw) {
  (void)vw;
  if (is_ip(o)) {
#pragma omp parallel for schedule(static)
    for (size_t ei = 0; ei < o.el.size(); ++ei) interior_gradient(o, o.el[ei], &o.dQ[2 * o.el[ei].offset]);
    return;
  }
#pragma omp parallel for schedule(static)
  for (size_t ei = 0; ei < o.el.size(); ++ei) vector_volume_green(o, o.el[ei], &o.dQ[2 * o.el[ei].offset]);
  for (auto& f : o.ed) br1_face(o, f);
#pragma omp parallel for schedule(static)
  for (size_t ei = 0; ei < o.el.size(); ++ei) {
    Element& e = o.el[ei];
    double* dQ = &o.dQ[2 * e.offset];
    const int NP = e.P * e.P;
    for (int d = 0; d < 2; ++d)
      for (int q = 0; q < NP; ++q)
        for (int k = 0; k < 4; ++k) dQ[(size_t(d) * NP + q) * 4 + k] = dQ[(size_t(d) * NP + q) * 4 + k] / e.jac[q];
  }
}

// ------------------------------------------------------------------ residual contributions
void viscous_volume_flux(Oracle& o, Element& e, std::vector<double>& F, ViscousWork& vw) {
  (void)vw;
  const Physics& ph = o.ph;
  const int NP = e.P * e.P;
  const double* Q = &o.Q[e.offset];
  const double* dQ = &o.dQ[2 * e.offset];
  const double mu = ph.mu + e.mu_a;
  for (int q = 0; q < NP; ++q) {
    double Fx[4], Fy[4];
    vflux(ph, &Q[4 * q], &dQ[4 * q], &dQ[(size_t(NP) + q) * 4], Fx, Fy);
    for (int k = 0; k < 4; ++k) {
      F[q * 8 + k] = F[q * 8 + k] - mu * Fx[k];
      F[q * 8 + 4 + k] = F[q * 8 + 4 + k] - mu * Fy[k];
    }
  }
}

void viscous_interior_flux(Oracle& o, Edge& f, const std::vector<double>& QL, const std::vector<double>& QR,
                           std::vector<double>& Fs, ViscousWork& vw) {
  (void)vw;
  const int P = f.P();
  std::vector<double> dQL = project_to_edge(f, SLOT_LEFT, f.storage[SLOT_LEFT].dQ, 2);
  std::vector<double> dQR = project_to_edge(f, SLOT_RIGHT, f.storage[SLOT_RIGHT].dQ, 2);
  for (int i = 0; i < P; ++i) {
    double Fv[4];
    visc_riemann(o, f.mu_a, f.N, f.invh, &QL[4 * i], &QR[4 * i], &dQL[4 * i], &dQL[(P + i) * 4], &dQR[4 * i],
                 &dQR[(P + i) * 4], f.nx(i), f.ny(i), Fv);
    double Fa[4];
    av_face_flux(o, f, &QL[4 * i], &QR[4 * i], Fa);
    for (int k = 0; k < 4; ++k) Fs[4 * i + k] = Fs[4 * i + k] - Fv[k] - Fa[k];
  }
}

void viscous_interior_gradient_faces(Oracle& o, Edge& f, const std::vector<double>& QL, const std::vector<double>& QR,
                                     ViscousWork& vw) {
  (void)vw;
  if (!gradient_faces(o)) return;
  const int P = f.P();
  std::vector<double> GL(8 * P), GR(8 * P);
  for (int i = 0; i < P; ++i) {
    double a[4], b[4], c[4], d[4];
    visc_gradient_riemann(o, f.mu_a, &QL[4 * i], &QR[4 * i], f.nx(i), f.ny(i), a, b, c, d);
    for (int k = 0; k < 4; ++k) {
      GL[(0 * P + i) * 4 + k] = a[k]; GL[(P + i) * 4 + k] = b[k];
      GR[(0 * P + i) * 4 + k] = c[k]; GR[(P + i) * 4 + k] = d[k];
    }
  }
  if (f.kind == E_STRAIGHT) {
    std::vector<double> gl = project_to_elem(f, SLOT_LEFT, GL, 2, false);
    std::vector<double> gr = project_to_elem(f, SLOT_RIGHT, GR, 2, false);
    for (auto& v : gl) v = v * f.dS[0];
    for (auto& v : gr) v = v * f.dS[0];
    gradient_face_sub(o, f.quads[SLOT_LEFT], f.edgeLocation[SLOT_LEFT], gl.data());
    gradient_face_sub(o, f.quads[SLOT_RIGHT], f.edgeLocation[SLOT_RIGHT], gr.data());
  } else {
    for (int d = 0; d < 2; ++d)
      for (int i = 0; i < P; ++i)
        for (int k = 0; k < 4; ++k) {
          GL[(d * P + i) * 4 + k] = GL[(d * P + i) * 4 + k] * f.dS[i];
          GR[(d * P + i) * 4 + k] = GR[(d * P + i) * 4 + k] * f.dS[i];
        }
    std::vector<double> gl = project_to_elem(f, SLOT_LEFT, GL, 2, false);
    std::vector<double> gr = project_to_elem(f, SLOT_RIGHT, GR, 2, false);
    gradient_face_sub(o, f.quads[SLOT_LEFT], f.edgeLocation[SLOT_LEFT], gl.data());
    gradient_face_sub(o, f.quads[SLOT_RIGHT], f.edgeLocation[SLOT_RIGHT], gr.data());
  }
}

static std::vector<double> mortar_grad(const std::vector<double>& T, int rows, int cols, const std::vector<double>& dQ) {
  std::vector<double> out(8 * rows, 0.0);
  for (int d = 0; d < 2; ++d)
    for (int l = 0; l < cols; ++l) for (int i = 0; i < rows; ++i) for (int k = 0; k < 4; ++k)
      out[(d * rows + i) * 4 + k] = out[(d * rows + i) * 4 + k] + T[i * cols + l] * dQ[(d * cols + l) * 4 + k];
  return out;
}

void viscous_mortar_fluxes(Oracle& o, Edge& f, const std::vector<double>& QLN, const std::vector<double>& QRN,
                           const std::vector<double>& QLS, const std::vector<double>& QRS,
                           std::vector<double>& FN, std::vector<double>& FS, ViscousWork& vw) {
  (void)vw;
  const int PL = f.storage[SLOT_LEFT].sp->P, PRN = f.storage[SLOT_RN].sp->P, PRS = f.storage[SLOT_RS].sp->P;
  const int PN = f.spN->P, PS = f.spS->P;
  const bool curved = f.kind == E_CURVED_SUBDIV;
  std::vector<double> dLN = mortar_grad(f.T_LN_FWD, PN, PL, f.storage[SLOT_LEFT].dQ);
  std::vector<double> dLS = mortar_grad(f.T_LS_FWD, PS, PL, f.storage[SLOT_LEFT].dQ);
  std::vector<double> dRN = mortar_grad(f.T_RN_FWD, PN, PRN, f.storage[SLOT_RN].dQ);
  std::vector<double> dRS = mortar_grad(f.T_RS_FWD, PS, PRS, f.storage[SLOT_RS].dQ);
  for (int i = 0; i < PN; ++i) {
    const double nx = curved ? f.normal_N[i] : f.normal_N[0], ny = curved ? f.normal_N[PN + i] : f.normal_N[1];
    double Fv[4];
    visc_riemann(o, f.mu_a, f.N_N, f.invh, &QLN[4 * i], &QRN[4 * i], &dLN[4 * i], &dLN[(PN + i) * 4], &dRN[4 * i],
                 &dRN[(PN + i) * 4], nx, ny, Fv);
    double Fa[4];
    av_face_flux(o, f, &QLN[4 * i], &QRN[4 * i], Fa);
    for (int k = 0; k < 4; ++k) FN[4 * i + k] = FN[4 * i + k] - Fv[k] - Fa[k];
  }
  for (int i = 0; i < PS; ++i) {
    const double nx = curved ? f.normal_S[i] : f.normal_S[0], ny = curved ? f.normal_S[PS + i] : f.normal_S[1];
    double Fv[4];
    visc_riemann(o, f.mu_a, f.N_S, f.invh, &QLS[4 * i], &QRS[4 * i], &dLS[4 * i], &dLS[(PS + i) * 4], &dRS[4 * i],
                 &dRS[(PS + i) * 4], nx, ny, Fv);
    double Fa[4];
    av_face_flux(o, f, &QLS[4 * i], &QRS[4 * i], Fa);
    for (int k = 0; k < 4; ++k) FS[4 * i + k] = FS[4 * i + k] - Fv[k] - Fa[k];
  }
}

void viscous_mortar_gradient_faces(Oracle& o, Edge& f, const std::vector<double>& QLN, const std::vector<double>& QRN,
                                   const std::vector<double>& QLS, const std::vector<double>& QRS, ViscousWork& vw) {
  (void)vw;
  if (!gradient_faces(o)) return;
  const int PL = f.storage[SLOT_LEFT].sp->P, PRN = f.storage[SLOT_RN].sp->P, PRS = f.storage[SLOT_RS].sp->P;
  const int PN = f.spN->P, PS = f.spS->P;
  const bool curved = f.kind == E_CURVED_SUBDIV;
  auto grads = [&](const std::vector<double>& QL, const std::vector<double>& QR, int Pm, const std::vector<double>& nrm,
                   const std::vector<double>& dSm, std::vector<double>& GL, std::vector<double>& GR) {
    GL.assign(8 * Pm, 0.0); GR.assign(8 * Pm, 0.0);
    for (int i = 0; i < Pm; ++i) {
      const double nx = curved ? nrm[i] : nrm[0], ny = curved ? nrm[Pm + i] : nrm[1];
      const double dS = curved ? dSm[i] : dSm[0];
      double a[4], b[4], c[4], d[4];
      visc_gradient_riemann(o, f.mu_a, &QL[4 * i], &QR[4 * i], nx, ny, a, b, c, d);
      for (int k = 0; k < 4; ++k) {
        GL[(0 * Pm + i) * 4 + k] = a[k] * dS; GL[(Pm + i) * 4 + k] = b[k] * dS;
        GR[(0 * Pm + i) * 4 + k] = c[k] * dS; GR[(Pm + i) * 4 + k] = d[k] * dS;
      }
    }
  };
  std::vector<double> GLN, GRN, GLS, GRS;
  grads(QLN, QRN, PN, f.normal_N, f.dS_N, GLN, GRN);
  grads(QLS, QRS, PS, f.normal_S, f.dS_S, GLS, GRS);
  std::vector<double> GL(8 * PL, 0.0), GN(8 * PRN, 0.0), GS(8 * PRS, 0.0);
  for (int d = 0; d < 2; ++d) {
    for (int l = 0; l < PN; ++l) for (int i = 0; i < PL; ++i) for (int k = 0; k < 4; ++k)
      GL[(d * PL + i) * 4 + k] = GL[(d * PL + i) * 4 + k] + f.T_LN_BKW[i * PN + l] * GLN[(d * PN + l) * 4 + k];
    for (int l = 0; l < PS; ++l) for (int i = 0; i < PL; ++i) for (int k = 0; k < 4; ++k)
      GL[(d * PL + i) * 4 + k] = GL[(d * PL + i) * 4 + k] + f.T_LS_BKW[i * PS + l] * GLS[(d * PS + l) * 4 + k];
    for (int l = 0; l < PN; ++l) for (int i = 0; i < PRN; ++i) for (int k = 0; k < 4; ++k)
      GN[(d * PRN + i) * 4 + k] = GN[(d * PRN + i) * 4 + k] + f.T_RN_BKW[i * PN + l] * GRN[(d * PN + l) * 4 + k];
    for (int l = 0; l < PS; ++l) for (int i = 0; i < PRS; ++i) for (int k = 0; k < 4; ++k)
      GS[(d * PRS + i) * 4 + k] = GS[(d * PRS + i) * 4 + k] + f.T_RS_BKW[i * PS + l] * GRS[(d * PS + l) * 4 + k];
  }
  gradient_face_sub(o, f.quads[SLOT_LEFT], f.edgeLocation[SLOT_LEFT], GL.data());
  gradient_face_sub(o, f.quads[SLOT_RN], f.edgeLocation[SLOT_RN], GN.data());
  gradient_face_sub(o, f.quads[SLOT_RS], f.edgeLocation[SLOT_RS], GS.data());
}

// boundary: F = Fi - Fv - Fa (Fi already scaled by dS), G kept for the gradient face
static thread_local std::vector<double> g_bdryG;

void viscous_boundary_flux(Oracle& o, Edge& f, std::vector<double>& F, ViscousWork& vw) {
  (void)vw;
  const Physics& ph = o.ph;
  const int P = f.P();
  const std::vector<double>& Q = f.storage[0].Q;
  const std::vector<double>& dQ = f.storage[0].dQ;
  std::vector<double> Fv(4 * P, 0.0), Fa(4 * P, 0.0);
  g_bdryG.assign(8 * P, 0.0);
  const double mu = ph.mu + f.mu_a;
  const bool ip = is_ip(o);
  const double penalty = ip ? o.cas.sigma0_ip * mu * f.N * f.N * f.invh : 0.0;
  const double eps = ip_epsilon(o);
  auto dS_at = [&](int i) { return f.straight_like() ? f.dS[0] : f.dS[i]; };
  if (!f.viscousBCType.empty() && f.viscousBCType[0] == VBC_PERIODIC && f.kind == E_STRAIGHT_BDRY) {
    const std::vector<double>& uB = *f.uB;
    const std::vector<double>& gB = *f.gB;
    for (int i = 0; i < P; ++i) {
      const int r = f.inverse ? (P - 1 - i) : i;
      double qb[4], gbx[4], gby[4];
      for (int k = 0; k < 4; ++k) { qb[k] = uB[4 * r + k]; gbx[k] = gB[4 * r + k]; gby[k] = gB[(P + r) * 4 + k]; }
      double fv[4];
      visc_riemann(o, f.mu_a, f.N, f.invh, &Q[4 * i], qb, &dQ[4 * i], &dQ[(P + i) * 4], gbx, gby, f.nx(i), f.ny(i),
                   fv);
      for (int k = 0; k < 4; ++k) Fv[4 * i + k] = fv[k] * f.dS[0];
      double fa[4];
      av_face_flux(o, f, &Q[4 * i], qb, fa);
      for (int k = 0; k < 4; ++k) Fa[4 * i + k] = fa[k] * f.dS[0];
      if (gradient_faces(o)) {
        double a[4], b[4], c[4], d[4];
        visc_gradient_riemann(o, f.mu_a, &Q[4 * i], qb, f.nx(i), f.ny(i), a, b, c, d);
        for (int k = 0; k < 4; ++k) { g_bdryG[(0 * P + i) * 4 + k] = a[k] * f.dS[0]; g_bdryG[(P + i) * 4 + k] = b[k] * f.dS[0]; }
      }
    }
  } else if (!f.viscousBCType.empty() && f.viscousBCType[0] == VBC_ADIABATIC) {
    const std::vector<double>& uS = *f.uSB;
    for (int i = 0; i < P; ++i) {
      double fa[4];
      av_face_flux(o, f, &Q[4 * i], &uS[4 * i], fa);
      for (int k = 0; k < 4; ++k) Fa[4 * i + k] = fa[k] * dS_at(i);
      double Fx[4], Fy[4];
      vflux_adiabatic(ph, &Q[4 * i], &Q[4 * i], &dQ[4 * i], &dQ[(P + i) * 4], Fx, Fy);
      for (int k = 0; k < 4; ++k) {
        double s = 0.0;
        s = s + (mu * Fx[k]) * f.nx(i);
        s = s + (mu * Fy[k]) * f.ny(i);
        if (ip) s = s - penalty * (Q[4 * i + k] - uS[4 * i + k]);
        Fv[4 * i + k] = s * dS_at(i);
      }
      if (gradient_faces(o)) {
        double fgx[4], fgy[4], Gx[4], Gy[4];
        for (int k = 0; k < 4; ++k) { fgx[k] = (Q[4 * i + k] - uS[4 * i + k]) * f.nx(i); fgy[k] = (Q[4 * i + k] - uS[4 * i + k]) * f.ny(i); }
        vflux_adiabatic(ph, &Q[4 * i], &Q[4 * i], fgx, fgy, Gx, Gy);
        for (int k = 0; k < 4; ++k) {
          g_bdryG[(0 * P + i) * 4 + k] = (eps * mu * Gx[k]) * dS_at(i);
          g_bdryG[(P + i) * 4 + k] = (eps * mu * Gy[k]) * dS_at(i);
        }
      }
    }
  } else {
    const std::vector<double>& uS = *f.uSB;
    for (int i = 0; i < P; ++i) {
      double fa[4];
      av_face_flux(o, f, &Q[4 * i], &uS[4 * i], fa);
      for (int k = 0; k < 4; ++k) Fa[4 * i + k] = fa[k] * dS_at(i);
      const int vbc = f.viscousBCType.empty() ? VBC_NEUMANN : f.viscousBCType[i];
      if (vbc == VBC_DIRICHLET) {
        double Fx[4], Fy[4];
        vflux(ph, &Q[4 * i], &dQ[4 * i], &dQ[(P + i) * 4], Fx, Fy);
        for (int k = 0; k < 4; ++k) {
          double s = (mu * Fx[k]) * f.nx(i) + (mu * Fy[k]) * f.ny(i);
          if (ip) s = s - penalty * (Q[4 * i + k] - uS[4 * i + k]);
          Fv[4 * i + k] = s * dS_at(i);
        }
        if (gradient_faces(o)) {
          double fgx[4], fgy[4], Gx[4], Gy[4];
          for (int k = 0; k < 4; ++k) { fgx[k] = (Q[4 * i + k] - uS[4 * i + k]) * f.nx(i); fgy[k] = (Q[4 * i + k] - uS[4 * i + k]) * f.ny(i); }
          vflux(ph, &Q[4 * i], fgx, fgy, Gx, Gy);
          for (int k = 0; k < 4; ++k) {
            g_bdryG[(0 * P + i) * 4 + k] = (1.0 * eps * mu * Gx[k]) * dS_at(i);
            g_bdryG[(P + i) * 4 + k] = (1.0 * eps * mu * Gy[k]) * dS_at(i);
          }
        }
      }
      // Neumann (and the far field): zero viscous and gradient-face flux
    }
  }
  for (int n = 0; n < 4 * P; ++n) F[n] = F[n] - Fv[n] - Fa[n];
}

void viscous_boundary_gradient_face(Oracle& o, Edge& f, ViscousWork& vw) {
  (void)vw;
  if (!gradient_faces(o)) return;
  gradient_face_sub(o, f.quads[0], f.edgeLocation[0], g_bdryG.data());
}

}  // namespace orc
