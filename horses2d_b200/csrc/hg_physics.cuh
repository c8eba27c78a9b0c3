// hg_physics.cuh -- device physics of the DGSEM residual (Euler part).
//
// Each function states the reference routine it computes; arithmetic follows the
// reference's order of operations so the FP64 path agrees with the reference to
// rounding (the kernels are built with FMA contraction, which changes only the
// last bits).
//   inviscid_flux   Physics/InviscidFluxes.f90:104-147 (scaled by 1/(sqrt(gamma) M),
//                   _DIMENSIONLESS_TAU)
//   roe / hll       Physics/RiemannSolvers.f90:189-305 / 307-399
//   exact           Physics/RiemannSolvers.f90:33-187, 405-459 (Newton on the star pressure)
//   lxf             Rusanov flux, no reference counterpart; same rotation and scaling
//   euler_wall      BoundaryConditions/EulerWall.incf:71-158 (prescribed wall flux)
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace hg {

enum { RIEMANN_ROE = 0, RIEMANN_HLL = 1, RIEMANN_EXACT = 2, RIEMANN_LXF = 3 };

struct PhysConst {
  double gamma, gm1, cp, cv, invSqrtGammaMach;
  double mu, cpPr, lambda;   // dimensionless viscosity, cp/Pr, second viscosity (-2/3)
};

template <typename real>
struct Phys {
  real gamma, gm1, cp, cv, isgm, mu, cpPr, lambda;
  __device__ __forceinline__ void load(const PhysConst& c) {
    gamma = real(c.gamma); gm1 = real(c.gm1); cp = real(c.cp); cv = real(c.cv); isgm = real(c.invSqrtGammaMach);
    mu = real(c.mu); cpPr = real(c.cpPr); lambda = real(c.lambda);
  }
};

template <typename real> __device__ __forceinline__ real sqrt_r(real x);
template <> __device__ __forceinline__ double sqrt_r(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float sqrt_r(float x) { return sqrtf(x); }
template <typename real> __device__ __forceinline__ real pow_r(real x, real y);
template <> __device__ __forceinline__ double pow_r(double x, double y) { return pow(x, y); }
template <> __device__ __forceinline__ float pow_r(float x, float y) { return powf(x, y); }

template <typename real>
__device__ __forceinline__ void inviscid_flux(const Phys<real>& ph, const real* u, real* f, real* g) {
  const real invRho = real(1) / u[0];
  const real vx = u[1] * invRho, vy = u[2] * invRho;
  const real p = ph.gm1 * (u[3] - real(0.5) * u[1] * vx - real(0.5) * u[2] * vy);
  f[0] = u[1]; f[1] = u[1] * vx + p; f[2] = u[1] * vy; f[3] = (u[3] + p) * vx;
  g[0] = u[2]; g[1] = f[2]; g[2] = u[2] * vy + p; g[3] = (u[3] + p) * vy;
#pragma unroll
  for (int k = 0; k < 4; ++k) { f[k] *= ph.isgm; g[k] *= ph.isgm; }
}

template <typename real>
__device__ __forceinline__ void flux_normal(real rho, real u, real v, real p, real H, real* F) {
  F[0] = rho * u; F[1] = F[0] * u + p; F[2] = F[0] * v; F[3] = H * F[0];
}

template <typename real>
__device__ __forceinline__ void rotate_back_scale(const Phys<real>& ph, real* F, real nx, real ny) {
  const real Ft = F[1] * nx - F[2] * ny;
  F[2] = F[1] * ny + F[2] * nx;
  F[1] = Ft;
#pragma unroll
  for (int k = 0; k < 4; ++k) F[k] *= ph.isgm;
}

template <typename real>
__device__ __forceinline__ void roe(const Phys<real>& ph, const real* qL, const real* qR, real nx, real ny, real* F) {
  const real rhoL = qL[0], invRhoL = real(1) / rhoL, sqrtRhoL = sqrt_r(rhoL);
  const real uL = (qL[1] * nx + qL[2] * ny) * invRhoL, vL = (-qL[1] * ny + qL[2] * nx) * invRhoL;
  const real pL = ph.gm1 * (qL[3] - real(0.5) * rhoL * (uL * uL + vL * vL));
  const real HL = ph.cp * pL * invRhoL + real(0.5) * (uL * uL + vL * vL);
  const real rhoR = qR[0], invRhoR = real(1) / rhoR, sqrtRhoR = sqrt_r(rhoR);
  const real uR = (qR[1] * nx + qR[2] * ny) * invRhoR, vR = (-qR[1] * ny + qR[2] * nx) * invRhoR;
  const real pR = ph.gm1 * (qR[3] - real(0.5) * rhoR * (uR * uR + vR * vR));
  const real HR = ph.cp * pR * invRhoR + real(0.5) * (uR * uR + vR * vR);
  const real invrho = real(1) / (sqrtRhoL + sqrtRhoR);
  const real u = (sqrtRhoL * uL + sqrtRhoR * uR) * invrho;
  const real v = (sqrtRhoL * vL + sqrtRhoR * vR) * invrho;
  const real H = (sqrtRhoL * HL + sqrtRhoR * HR) * invrho;
  const real a = sqrt_r(ph.gm1 * (H - real(0.5) * (u * u + v * v)));
  const real dq0 = rhoR - rhoL, dq1 = rhoR * uR - rhoL * uL, dq2 = rhoR * vR - rhoL * vL, dq3 = qR[3] - qL[3];
  const real al2 = dq2 - v * dq0;
  const real al1 = ph.gm1 * (dq0 * (H - u * u) + u * dq1 - dq3 + (dq2 - v * dq0) * v) / (a * a);
  const real al0 = (dq0 * (u + a) - dq1 - a * al1) / (real(2) * a);
  const real al3 = dq0 - (al0 + al1);
  flux_normal(rhoL, uL, vL, pL, HL, F);
  // waves with negative speed, added in the reference's order (u-a, u, u, u+a)
  if (!(u - a > real(0))) {
    const real s = al0 * (u - a);
    F[0] += s; F[1] += s * (u - a); F[2] += s * v; F[3] += s * (H - u * a);
    if (!(u > real(0))) {
      const real s1 = al1 * u;
      F[0] += s1; F[1] += s1 * u; F[2] += s1 * v; F[3] += s1 * (real(0.5) * (u * u + v * v));
      const real s2 = al2 * u;
      F[2] += s2; F[3] += s2 * v;
      if (!(u + a > real(0))) {
        const real s3 = al3 * (u + a);
        F[0] += s3; F[1] += s3 * (u + a); F[2] += s3 * v; F[3] += s3 * (H + u * a);
      }
    }
  }
  rotate_back_scale(ph, F, nx, ny);
}

template <typename real>
__device__ __forceinline__ void hll(const Phys<real>& ph, const real* qL, const real* qR, real nx, real ny, real* F) {
  const real rhoL = qL[0], invRhoL = real(1) / rhoL;
  const real uL = (qL[1] * nx + qL[2] * ny) * invRhoL, vL = (-qL[1] * ny + qL[2] * nx) * invRhoL;
  const real pL = ph.gm1 * (qL[3] - real(0.5) * rhoL * (uL * uL + vL * vL));
  const real HL = ph.cp * pL * invRhoL + real(0.5) * (uL * uL + vL * vL);
  const real aL = sqrt_r(ph.gamma * pL * invRhoL), rhoeL = qL[3];
  const real rhoR = qR[0], invRhoR = real(1) / rhoR;
  const real uR = (qR[1] * nx + qR[2] * ny) * invRhoR, vR = (-qR[1] * ny + qR[2] * nx) * invRhoR;
  const real pR = ph.gm1 * (qR[3] - real(0.5) * rhoR * (uR * uR + vR * vR));
  const real HR = ph.cp * pR * invRhoR + real(0.5) * (uR * uR + vR * vR);
  const real aR = sqrt_r(ph.gamma * pR * invRhoR), rhoeR = qR[3];
  const real sqrtRhoL = sqrt_r(rhoL), sqrtRhoR = sqrt_r(rhoR);
  const real invrho = real(1) / (sqrtRhoL + sqrtRhoR);
  const real u = (sqrtRhoL * uL + sqrtRhoR * uR) * invrho;
  const real v = (sqrtRhoL * vL + sqrtRhoR * vR) * invrho;
  const real H = (sqrtRhoL * HL + sqrtRhoR * HR) * invrho;
  const real a = sqrt_r(ph.gm1 * (H - real(0.5) * (u * u + v * v)));
  const real SL = fmin(uL - aL, u - a), SR = fmax(uR + aR, u + a);
  if (SL >= real(0)) flux_normal(rhoL, uL, vL, pL, HL, F);
  else if (SR <= real(0)) flux_normal(rhoR, uR, vR, pR, HR, F);
  else {
    const real invdS = real(1) / (SR - SL);
    F[0] = (SR * rhoL * uL - SL * rhoR * uR + SL * SR * (rhoR - rhoL)) * invdS;
    F[1] = (SR * (rhoL * uL * uL + pL) - SL * (rhoR * uR * uR + pR) + SL * SR * (rhoR * uR - rhoL * uL)) * invdS;
    F[2] = (SR * rhoL * uL * vL - SL * rhoR * uR * vR + SR * SL * (rhoR * vR - rhoL * vL)) * invdS;
    F[3] = (SR * uL * rhoL * HL - SL * uR * rhoR * HR + SR * SL * (rhoeR - rhoeL)) * invdS;
  }
  rotate_back_scale(ph, F, nx, ny);
}

template <typename real>
__device__ __forceinline__ void lxf(const Phys<real>& ph, const real* qL, const real* qR, real nx, real ny, real* F) {
  const real rhoL = qL[0], invRhoL = real(1) / rhoL;
  const real uL = (qL[1] * nx + qL[2] * ny) * invRhoL, vL = (-qL[1] * ny + qL[2] * nx) * invRhoL;
  const real pL = ph.gm1 * (qL[3] - real(0.5) * rhoL * (uL * uL + vL * vL));
  const real HL = ph.cp * pL * invRhoL + real(0.5) * (uL * uL + vL * vL);
  const real aL = sqrt_r(ph.gamma * pL * invRhoL);
  const real rhoR = qR[0], invRhoR = real(1) / rhoR;
  const real uR = (qR[1] * nx + qR[2] * ny) * invRhoR, vR = (-qR[1] * ny + qR[2] * nx) * invRhoR;
  const real pR = ph.gm1 * (qR[3] - real(0.5) * rhoR * (uR * uR + vR * vR));
  const real HR = ph.cp * pR * invRhoR + real(0.5) * (uR * uR + vR * vR);
  const real aR = sqrt_r(ph.gamma * pR * invRhoR);
  const real lam = fmax(fabs(uL) + aL, fabs(uR) + aR);
  real FL[4], FR[4];
  flux_normal(rhoL, uL, vL, pL, HL, FL);
  flux_normal(rhoR, uR, vR, pR, HR, FR);
  const real dq[4] = {rhoR - rhoL, rhoR * uR - rhoL * uL, rhoR * vR - rhoL * vL, qR[3] - qL[3]};
#pragma unroll
  for (int k = 0; k < 4; ++k) F[k] = real(0.5) * (FL[k] + FR[k]) - real(0.5) * lam * dq[k];
  rotate_back_scale(ph, F, nx, ny);
}

// Exact Riemann solver (Physics/RiemannSolvers.f90:33-187 with the star-pressure iteration of
// :405-459), in the face-normal frame.  It runs in its own kernel (exact_flux_kernel, hg_exact.cu)
// ahead of the stage kernels, which read its face fluxes: the iteration and its many pow calls
// would otherwise widen the register budget of every fused kernel.
template <typename real>
struct ExactFace {
  real qn[2][4];   // left / right conserved state, momentum rotated to (normal, tangential)
  real w[2][5];    // left / right {rho, u_n, u_t, p, a}
  real gamma, gm1, cp, cv;
};

// Wave curve f(p) of one side and its derivative (shock branch above the side's pressure,
// rarefaction branch below).
template <typename real>
__device__ __forceinline__ void exact_wave(const ExactFace<real>& X, real p, const real* W, real& F, real& dF) {
  if (p > W[3]) {
    const real A = real(2) / (W[0] * (X.gamma + real(1)));
    const real B = X.gm1 * W[3] / (X.gamma + real(1));
    const real s = sqrt_r(A / (p + B));
    F = (p - W[3]) * s;
    dF = s * (real(1) - real(0.5) * (p - W[3]) / (B + p));
  } else {
    F = real(2) * X.cv * W[4] * (pow_r(p / W[3], real(0.5) / X.cp) - real(1));
    dF = real(1) / (W[0] * W[4]) * pow_r(p / W[3], real(-0.5) * (X.gamma + real(1)) / X.gamma);
  }
}

// Star pressure: two-rarefaction guess, then Newton (at most 50 steps, stop at relative change
// 1e-6); returns u* through ustar.
template <typename real>
__device__ __forceinline__ real exact_star(const ExactFace<real>& X, real& ustar) {
  const real* wL = X.w[0];
  const real* wR = X.w[1];
  real pstar = pow_r((wL[4] + wR[4] - real(0.5) * X.gm1 * (wR[1] - wL[1])) /
                         (wL[4] / pow_r(wL[3], real(0.5) / X.cp) + wR[4] / pow_r(wR[3], real(0.5) / X.cp)),
                     real(2) * X.cp);
  real FL = real(0), dFL = real(0), FR = real(0), dFR = real(0);
#pragma unroll 1
  for (int it = 1; it <= 50; ++it) {
    exact_wave(X, pstar, wL, FL, dFL);
    exact_wave(X, pstar, wR, FR, dFR);
    const real Fn = FL + FR + wR[1] - wL[1], dF = dFL + dFR;
    const real pold = pstar;
    pstar = pold - Fn / dF;
    if (fabs(real(0.5) * fabs(pstar - pold) / (pstar + pold)) < real(1.0e-6)) {
      exact_wave(X, pstar, wL, FL, dFL);
      exact_wave(X, pstar, wR, FR, dFR);
      break;
    }
  }
  ustar = real(0.5) * (wL[1] + wR[1] + FR - FL);
  return pstar;
}

// Godunov flux at x/t = 0 (normal frame, unscaled) with the reference's branch conditions; a state
// that meets none of them gives a zero flux, as in the reference.
template <typename real>
__device__ __forceinline__ void exact_sample(const ExactFace<real>& X, real pstar, real ustar, real* F) {
  const real gamma = X.gamma, cp = X.cp, cv = X.cv;
  const real g1 = gamma + real(1), gq = (gamma - real(1)) / (gamma + real(1));
  const int side = ustar >= real(0) ? 0 : 1;
  const real* w = X.w[side];
  real rs = real(0), us = real(0), vs = real(0), ps = real(0);
  bool star = false, upw = false;
  const real sr = pow_r(pstar / w[3], real(0.5) / cp);
  if (side == 0) {
    const real ss = sqrt_r(g1 / (real(2) * gamma) * pstar / w[3] + real(0.5) / cp);
    if (pstar <= w[3] && w[1] >= w[4]) upw = true;
    else if (pstar <= w[3] && w[1] < w[4] && ustar < w[4] * sr) { rs = w[0] * pow_r(pstar / w[3], real(1) / gamma); star = true; }
    else if (pstar <= w[3] && w[1] < w[4] && ustar >= w[4] * sr) {
      us = real(2) * w[4] / g1 + (gamma - real(1)) / g1 * w[1];
      rs = w[0] * pow_r(us / w[4], real(2) * cv);
      ps = w[3] * pow_r(rs / w[0], gamma); vs = w[2];
    } else if (pstar > w[3] && w[1] >= w[4] * ss) upw = true;
    else if (pstar > w[3] && w[1] < w[4] * ss) {
      rs = w[0] * ((pstar / w[3] + gq) / (pstar / w[3] * (gamma - real(1)) / g1 + real(1))); star = true;
    }
  } else {
    if (pstar <= w[3] && w[1] + w[4] <= real(0)) upw = true;
    else if (pstar <= w[3] && w[1] + w[4] >= real(0) && ustar + w[4] * sr >= real(0)) {
      rs = w[0] * pow_r(pstar / w[3], real(1) / gamma); star = true;
    } else if (pstar <= w[3] && w[1] + w[4] > real(0) && ustar + w[4] * sr < real(0)) {
      us = real(-2) * w[4] / g1 + (gamma - real(1)) / g1 * w[1];
      rs = w[0] * pow_r(-us / w[4], real(2) * cv);
      ps = w[3] * pow_r(rs / w[0], gamma); vs = w[2];
    } else if (pstar > w[3] && w[1] + w[4] * (real(0.5) * g1 / gamma * pstar / w[3] + real(0.5) / cp) <= real(0)) upw = true;
    else if (pstar > w[3] && w[1] + w[4] * (g1 / (real(2) * gamma) * pstar / w[3] + real(0.5) / cp) > real(0)) {
      rs = w[0] * ((pstar / w[3] + gq) / (pstar / w[3] * (gamma - real(1)) / g1 + real(1))); star = true;
    }
  }
  if (star) { us = ustar; vs = w[2]; ps = pstar; }
  if (upw) {
    const real* qn = X.qn[side];
    F[0] = qn[1]; F[1] = qn[1] * w[1] + w[3]; F[2] = qn[2] * w[1];
    F[3] = w[1] * (cp * w[3] + real(0.5) * (qn[1] * w[1] + qn[2] * w[2]));
  } else {
    F[0] = rs * us; F[1] = rs * us * us + ps; F[2] = rs * us * vs;
    F[3] = us * (cp * ps + real(0.5) * rs * (us * us + vs * vs));
  }
}

template <typename real>
__device__ __forceinline__ void exact(const Phys<real>& ph, const real* qL, const real* qR, real nx, real ny, real* F) {
  ExactFace<real> X;
  X.gamma = ph.gamma; X.gm1 = ph.gm1; X.cp = ph.cp; X.cv = ph.cv;
  const real* q[2] = {qL, qR};
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    real* qn = X.qn[s];
    real* w = X.w[s];
    qn[0] = q[s][0]; qn[1] = q[s][1] * nx + q[s][2] * ny; qn[2] = -q[s][1] * ny + q[s][2] * nx; qn[3] = q[s][3];
    w[0] = qn[0]; w[1] = qn[1] / qn[0]; w[2] = qn[2] / qn[0];
    w[3] = ph.gm1 * (qn[3] - real(0.5) * (qn[1] * w[1] + qn[2] * w[2])); w[4] = sqrt_r(ph.gamma * w[3] / w[0]);
  }
  real ustar;
  const real pstar = exact_star(X, ustar);
  exact_sample(X, pstar, ustar, F);
  rotate_back_scale(ph, F, nx, ny);
}

template <typename real>
__device__ __forceinline__ void riemann(int which, const Phys<real>& ph, const real* qL, const real* qR, real nx, real ny,
                                        real* F) {
  if (which == RIEMANN_HLL) hll(ph, qL, qR, nx, ny, F);
  else if (which == RIEMANN_LXF) lxf(ph, qL, qR, nx, ny, F);
  else roe(ph, qL, qR, nx, ny, F);
}

// Riemann flux of one face node in a stage kernel: the exact solver's value is read from the face
// flux buffer [n_el*4][P][4] that exact_flux_kernel filled for this stage (same arguments).
template <typename real>
__device__ __forceinline__ void face_riemann(int which, const Phys<real>& ph, const real* qL, const real* qR, real nx,
                                             real ny, const real* FX, size_t slot, real* F) {
  if (which == RIEMANN_EXACT) {
#pragma unroll
    for (int k = 0; k < 4; ++k) F[k] = FX[slot * 4 + k];
  } else {
    riemann(which, ph, qL, qR, nx, ny, F);
  }
}

// Prescribed Euler-wall flux F(q_wall) . n dS, q_wall = interior state with the normal momentum removed.
template <typename real>
__device__ __forceinline__ void euler_wall_flux(const Phys<real>& ph, const real* q0, real nx, real ny, real dS, real* F) {
  const real rhovn = q0[1] * nx + q0[2] * ny;
  const real rhovt = -q0[1] * ny + q0[2] * nx;   // enters squared: the sign convention of curved walls is immaterial
  const real p = ph.gm1 * (q0[3] - real(0.5) * (q0[1] * q0[1] + q0[2] * q0[2]) / q0[0]);
  real q[4] = {q0[0], q0[1] - rhovn * nx, q0[2] - rhovn * ny, ph.cv * p + real(0.5) * rhovt * rhovt / q0[0]};
  real f[4], g[4];
  inviscid_flux(ph, q, f, g);
#pragma unroll
  for (int k = 0; k < 4; ++k) F[k] = f[k] * nx * dS + g[k] * ny * dS;
}

// viscousFlux (Physics/ViscousFluxes.f90:39-164): Fx, Fy from q and its gradient (dqx, dqy)
template <typename real>
__device__ __forceinline__ void viscous_flux(const Phys<real>& ph, const real* q, const real* dqx, const real* dqy,
                                             real* Fx, real* Fy) {
  const real invRho = real(1) / q[0];
  const real u = q[1] * invRho, v = q[2] * invRho;
  const real uDivRho = u * invRho, vDivRho = v * invRho;
  const real divV = -uDivRho * dqx[0] + invRho * dqx[1] - vDivRho * dqy[0] + invRho * dqy[2];
  const real dxT = ph.gm1 * invRho * (-q[3] * invRho * dqx[0] + dqx[3] + u * (u * dqx[0] - dqx[1]) + v * (v * dqx[0] - dqx[2]));
  const real dyT = ph.gm1 * invRho * (-q[3] * invRho * dqy[0] + dqy[3] + u * (u * dqy[0] - dqy[1]) + v * (v * dqy[0] - dqy[2]));
  Fx[0] = real(0);
  Fx[1] = real(2) * (-uDivRho * dqx[0] + invRho * dqx[1]) + ph.lambda * divV;
  Fx[2] = -vDivRho * dqx[0] - uDivRho * dqy[0] + invRho * dqy[1] + invRho * dqx[2];
  Fx[3] = u * Fx[1] + v * Fx[2] + ph.cpPr * dxT;
  Fy[0] = real(0);
  Fy[1] = Fx[2];
  Fy[2] = real(2) * (-vDivRho * dqy[0] + invRho * dqy[2]) + ph.lambda * divV;
  Fy[3] = u * Fy[1] + v * Fy[2] + ph.cpPr * dyT;
}

// AdiabaticViscousFlux1D/2D (ViscousFluxes.f90:230-330): no heat flux, work term with qB's velocity
template <typename real>
__device__ __forceinline__ void viscous_flux_adiabatic(const Phys<real>& ph, const real* q, const real* qB,
                                                       const real* dqx, const real* dqy, real* Fx, real* Fy) {
  const real invRho = real(1) / q[0];
  const real u = q[1] * invRho, v = q[2] * invRho;
  const real uDivRho = u * invRho, vDivRho = v * invRho;
  const real divV = -uDivRho * dqx[0] + invRho * dqx[1] - vDivRho * dqy[0] + invRho * dqy[2];
  Fx[0] = real(0);
  Fx[1] = real(2) * (-uDivRho * dqx[0] + invRho * dqx[1]) + ph.lambda * divV;
  Fx[2] = -vDivRho * dqx[0] - uDivRho * dqy[0] + invRho * dqy[1] + invRho * dqx[2];
  Fx[3] = (qB[1] * Fx[1] + qB[2] * Fx[2]) / qB[0];
  Fy[0] = real(0);
  Fy[1] = Fx[2];
  Fy[2] = real(2) * (-vDivRho * dqy[0] + invRho * dqy[2]) + ph.lambda * divV;
  Fy[3] = (qB[1] * Fy[1] + qB[2] * Fy[2]) / qB[0];
}

}  // namespace hg
