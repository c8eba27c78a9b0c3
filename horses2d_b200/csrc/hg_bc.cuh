// hg_bc.cuh -- boundary states of the reference's boundary-condition classes (device code).
//
// Each zone evaluates, per boundary node and from the interior trace q:
//   uB   the inviscid ghost state fed to the Riemann solver (WEAK_RIEMANN), or the
//        prescribed flux for the Euler wall (WEAK_PRESCRIBED);
//   uSB  the viscous boundary state (BR1 u* on the face, IP penalty target);
//   vbc  the viscous condition of the node: Dirichlet, Neumann or adiabatic.
// Restated from BoundaryConditions/*.incf UpdateSolution routines:
//   EulerWall       EulerWall.incf:71-158
//   ViscousWall     ViscousWall.incf:155-254 (Tw and wall velocity made dimensionless
//                   as in ViscousWall_Construct)
//   Dirichlet       Dirichlet.incf:155-300 (NAVIER_STOKES branch for uSB / vbc)
//   Farfield        Farfield.incf:138-376
//   PressureOutlet  PressureOutlet.incf:151-330
//   newDirichlet    newDirichlet.incf (UpdateSolution; uSB aliases uB in the Navier-Stokes build)
// Where the reference is undefined: far-field zones never set their viscous
// condition (Farfield.incf), so the far field is Neumann here; the straight-edge
// supersonic-outflow branch of the far field writes uB with swapped indices
// (Farfield.incf:246), so uB = q here, as on curved edges.
#pragma once
#include "hg_physics.cuh"

namespace hg {

enum { BC_PERIODIC = 1, BC_DIRICHLET = 2, BC_EULERWALL = 3, BC_VISCOUSWALL = 4, BC_FARFIELD = 5,
       BC_PRESSUREOUTLET = 6, BC_NEWDIRICHLET = 7 };
enum { VBC_DIRICHLET = 1, VBC_NEUMANN = 2, VBC_ADIABATIC = 4 };

struct Zone {
  int type, riemann;
  double q[4];          // dimensionless zone state (Dirichlet / far field / outlet)
  double Tw;            // dimensionless wall temperature (isothermal walls)
  double vw[2];         // dimensionless wall velocity
  int wall_type;        // 1 isothermal, 2 adiabatic
  int outflow_type;     // 1 reflective, 2 partially non-reflective
  int nd_mode;          // newDirichlet: 0 specify speed, 1 specify total pressure
  int nd_outflow_total; // newDirichlet: outflow pressure 0 static, 1 total
};

// NORM2 of a 2-vector with a running scale (no overflow), as Fortran's intrinsic evaluates it
template <typename real>
__device__ __forceinline__ real norm2_scaled(real a, real b) {
  real scale = real(0), ssq = real(1);
  const real xs[2] = {a, b};
#pragma unroll
  for (int n = 0; n < 2; ++n) {
    if (xs[n] != real(0)) {
      const real ax = fabs(xs[n]);
      if (scale < ax) { ssq = real(1) + ssq * (scale / ax) * (scale / ax); scale = ax; }
      else ssq = ssq + (ax / scale) * (ax / scale);
    }
  }
  return scale * sqrt_r(ssq);
}

// newDirichletBC_UpdateSolution at one node (out of line: pow would raise the register budget of
// every kernel that inlines the zone switch).
template <typename real>
__device__ __noinline__ int new_dirichlet_state(const Phys<real>& ph, const Zone& z, const real* q, real nx, real ny,
                                                real* uB, real* uSB) {
  const real gm1 = ph.gm1, gamma = ph.gamma, cv = ph.cv;
  const real cp = ph.cp;
  const real zq[4] = {real(z.q[0]), real(z.q[1]), real(z.q[2]), real(z.q[3])};
  const real uExt = zq[1] / zq[0], vExt = zq[2] / zq[0];
  const real pExt = gm1 * (zq[3] - real(0.5) * (zq[1] * uExt + zq[2] * vExt));
  const real MExtSq = (uExt * uExt + vExt * vExt) / (gamma * pExt) * zq[0];
  const real sExt = pExt / pow_r(zq[0], gamma);
  const real ptExt = pExt * pow_r(real(1) + real(0.5) * gm1 * MExtSq, cp);
  const real rhoL = q[0], uL = q[1] / rhoL, vL = q[2] / rhoL;
  const real vnL = uL * nx + vL * ny;
  const real pL = gm1 * (q[3] - real(0.5) * (q[1] * uL + q[2] * vL));
  const real aL = sqrt_r(gamma * pL / rhoL);
  const real ML = sqrt_r(uL * uL + vL * vL) / aL;
  int vbc;
  if (vnL <= real(0)) {
    if (ML > real(1)) {
#pragma unroll
      for (int k = 0; k < 4; ++k) uB[k] = zq[k];
    } else {
      const real pR = pL;
      const real rhoR = pow_r(pR / sExt, real(1) / gamma);
      const real aR = sqrt_r(gamma * pR / rhoR);
      if (z.nd_mode == 0) {
        uB[0] = zq[0]; uB[1] = zq[1]; uB[2] = zq[2];
        uB[3] = cv * pR + real(0.5) * (uB[1] * uB[1] + uB[2] * uB[2]) / uB[0];
      } else {
        const real nrm = norm2_scaled(uExt, vExt);
        const real MR = pR >= ptExt ? -sqrt_r(real(2) / gm1 * (pow_r(pR / ptExt, gm1 / gamma) - real(1)))
                                    : sqrt_r(real(2) / gm1 * (pow_r(ptExt / pR, gm1 / gamma) - real(1)));
        uB[0] = rhoR;
        uB[1] = rhoR * aR * MR * (uExt / nrm);
        uB[2] = rhoR * aR * MR * (vExt / nrm);
        uB[3] = cv * pR + real(0.5) * rhoR * aR * aR * MR * MR;
      }
    }
    vbc = VBC_DIRICHLET;
  } else if (ML > real(1)) {
#pragma unroll
    for (int k = 0; k < 4; ++k) uB[k] = q[k];
    vbc = VBC_NEUMANN;
  } else {
    uB[0] = q[0]; uB[1] = q[1]; uB[2] = q[2];
    const real pb = z.nd_outflow_total ? ptExt : pExt;
    uB[3] = cv * (real(2) * pb - pL) + real(0.5) * (uB[1] * uL + uB[2] * vL);
    vbc = VBC_DIRICHLET;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) uSB[k] = uB[k];
  return vbc;
}

// Returns the inviscid ghost uB, the viscous state uSB and the viscous condition.  qnode, when
// given, is this node's own Dirichlet state (a zone fed per node by hg_set_boundary_state: the
// reference's boundary-condition function, BoundaryConditions/BoundaryConditionFunctionDrivers.incf);
// otherwise a Dirichlet zone holds its constant state.
template <typename real>
__device__ __forceinline__ int bc_states(const Phys<real>& ph, const Zone& z, const real* q, real nx, real ny, real* uB,
                                         real* uSB, const double* qnode = nullptr) {
  const real gm1 = ph.gm1, gamma = ph.gamma, cv = ph.cv;
  switch (z.type) {
    case BC_EULERWALL: {
      const real rhovn = q[1] * nx + q[2] * ny;
      const real rhovt = -q[1] * ny + q[2] * nx;
      const real p = gm1 * (q[3] - real(0.5) * (q[1] * q[1] + q[2] * q[2]) / q[0]);
      uB[0] = q[0]; uB[1] = q[1] - real(2) * rhovn * nx; uB[2] = q[2] - real(2) * rhovn * ny; uB[3] = q[3];
      uSB[0] = q[0]; uSB[1] = q[1] - rhovn * nx; uSB[2] = q[2] - rhovn * ny;
      uSB[3] = cv * p + real(0.5) * rhovt * rhovt / q[0];
      return VBC_ADIABATIC;
    }
    case BC_VISCOUSWALL: {
      const real vx = real(z.vw[0]), vy = real(z.vw[1]), Tw = real(z.Tw);
      const bool iso = z.wall_type == 1;
      uB[0] = q[0];
      uB[1] = real(2) * uB[0] * vx - q[1];
      uB[2] = real(2) * uB[0] * vy - q[2];
      const real Ek = real(0.5) * (uB[1] * uB[1] + uB[2] * uB[2]) / uB[0];
      uB[3] = iso ? cv * uB[0] * Tw + Ek : q[3];
      uSB[0] = q[0]; uSB[1] = uSB[0] * vx; uSB[2] = uSB[0] * vy;
      uSB[3] = iso ? cv * uSB[0] * Tw + real(0.5) * (uSB[1] * uSB[1] + uSB[2] * uSB[2]) / uSB[0]
                   : q[3] - Ek + real(0.5) * uSB[0] * (vx * vx + vy * vy);
      return iso ? VBC_DIRICHLET : VBC_ADIABATIC;
    }
    case BC_DIRICHLET: {
      const double* zs = qnode ? qnode : z.q;
#pragma unroll
      for (int k = 0; k < 4; ++k) uB[k] = real(zs[k]);
      const real rhoL = q[0], uL = q[1] / rhoL, vL = q[2] / rhoL;
      const real vnL = uL * nx + vL * ny;
      const real pL = gm1 * (q[3] - real(0.5) * (q[1] * uL + q[2] * vL));
      const real aL = sqrt_r(gamma * pL / rhoL);
      const real ML = sqrt_r(uL * uL + vL * vL) / aL;
      if (vnL <= real(0)) {
        if (ML > real(1)) {
#pragma unroll
          for (int k = 0; k < 4; ++k) uSB[k] = uB[k];
        } else {
          uSB[0] = uB[0]; uSB[1] = uB[1]; uSB[2] = uB[2];
          uSB[3] = cv * pL + real(0.5) * (uSB[1] * uSB[1] + uSB[2] * uSB[2]) / uSB[0];
        }
        return VBC_DIRICHLET;
      }
      if (ML > real(1)) {
#pragma unroll
        for (int k = 0; k < 4; ++k) uSB[k] = q[k];
        return VBC_NEUMANN;
      }
      const real pB = gm1 * (uB[3] - real(0.5) * (uB[1] * uB[1] + uB[2] * uB[2]) / uB[0]);
      uSB[0] = q[0]; uSB[1] = q[1]; uSB[2] = q[2];
      uSB[3] = cv * pB + real(0.5) * (uSB[1] * uL + uSB[2] * vL);
      return VBC_DIRICHLET;
    }
    case BC_FARFIELD: {
      const real rhoI = real(z.q[0]), uI = real(z.q[1]) / rhoI, vI = real(z.q[2]) / rhoI;
      const real pI = gm1 * (real(z.q[3]) - real(0.5) * real(z.q[1]) * uI - real(0.5) * real(z.q[2]) * vI);
      const real rhoL = q[0], uL = q[1] / rhoL, vL = q[2] / rhoL;
      const real vnL = uL * nx + vL * ny;
      const real pL = gm1 * (q[3] - real(0.5) * q[1] * uL - real(0.5) * q[2] * vL);
      const real aL = sqrt_r(gamma * pL / rhoL);
      const real ML = sqrt_r(uL * uL + vL * vL) / aL;
      if (ML > real(1)) {
        if (vnL < real(0)) {
#pragma unroll
          for (int k = 0; k < 4; ++k) uB[k] = real(z.q[k]);
        } else {
#pragma unroll
          for (int k = 0; k < 4; ++k) uB[k] = q[k];
        }
      } else {
        real rhoR, uR, vR, pR;
        if (vnL < real(0)) {
          pR = real(0.5) * (pL + pI - rhoL * aL * (nx * (uL - uI) + ny * (vL - vI)));
          rhoR = rhoI + (pR - pI) / (aL * aL);
          uR = uI + nx * (pR - pI) / (aL * rhoL);
          vR = vI + ny * (pR - pI) / (aL * rhoL);
        } else {
          pR = pI;
          rhoR = rhoL + (pI - pL) / (aL * aL);
          uR = uL - nx * (pI - pL) / (rhoL * aL);
          vR = vL - ny * (pI - pL) / (rhoL * aL);
        }
        uB[0] = rhoR; uB[1] = rhoR * uR; uB[2] = rhoR * vR;
        uB[3] = cv * pR + real(0.5) * (uB[1] * uR + uB[2] * vR);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) uSB[k] = uB[k];
      return VBC_NEUMANN;
    }
    case BC_PRESSUREOUTLET: {
      const real rhoI = real(z.q[0]), uI = real(z.q[1]) / rhoI, vI = real(z.q[2]) / rhoI;
      const real pI = gm1 * (real(z.q[3]) - real(0.5) * real(z.q[1]) * uI - real(0.5) * real(z.q[2]) * vI);
      const real nrm = sqrt_r(uI * uI + vI * vI);
      const real rhoL = q[0], uL = q[1] / rhoL, vL = q[2] / rhoL;
      const real vnL = uL * nx + vL * ny;
      const real pL = gm1 * (q[3] - real(0.5) * q[1] * uL - real(0.5) * q[2] * vL);
      const real aL = sqrt_r(gamma * pL / rhoL);
      const real ML = sqrt_r(uL * uL + vL * vL) / aL;
      if (ML > real(1)) {
        const bool in = vnL < real(0);
#pragma unroll
        for (int k = 0; k < 4; ++k) { uB[k] = in ? real(z.q[k]) : q[k]; uSB[k] = uB[k]; }
        return in ? VBC_DIRICHLET : VBC_NEUMANN;
      }
      real rhoR, uR, vR, pR;
      if (z.outflow_type != 2) {
        const real R0 = pL - aL * aL * rhoL;
        const real Rplus = vnL + real(2) * cv * aL;
        rhoR = -(R0 - pI) / (aL * aL);
        const real aR = sqrt_r(gamma * pI / rhoR);
        const real vnR = Rplus - real(2) * aR * cv;
        uR = uL + (vnR - vnL) * nx;
        vR = vL + (vnR - vnL) * ny;
        pR = pI;
      } else if (vnL < real(0)) {
        pR = real(2) * pI - pL; uR = fabs(vnL) * (uI / nrm); vR = fabs(vnL) * (vI / nrm); rhoR = rhoL;
      } else {
        pR = real(2) * pI - pL; uR = uL; vR = vL; rhoR = rhoL;
      }
      uB[0] = rhoR; uB[1] = rhoR * uR; uB[2] = rhoR * vR;
      uB[3] = cv * pR + real(0.5) * (uB[1] * uR + uB[2] * vR);
      if (vnL < real(0)) {
#pragma unroll
        for (int k = 0; k < 4; ++k) uSB[k] = uB[k];
      } else {
        uSB[0] = rhoL; uSB[1] = rhoL * uL; uSB[2] = rhoL * vL; uSB[3] = cv * pR + real(0.5) * rhoL * (uL * uL + vL * vL);
      }
      return VBC_DIRICHLET;
    }
    case BC_NEWDIRICHLET:
      return new_dirichlet_state(ph, z, q, nx, ny, uB, uSB);
    default: {
#pragma unroll
      for (int k = 0; k < 4; ++k) { uB[k] = q[k]; uSB[k] = q[k]; }
      return VBC_NEUMANN;
    }
  }
}

}  // namespace hg
