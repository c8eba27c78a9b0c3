// hg_ns.cuh -- Navier-Stokes stage kernels (BR1 and interior penalty) for sm_100a.
//
// Per Runge-Kutta stage two launches:
//   ns_gradient_kernel  the element gradient dQ -- BR1 lifting
//        dQ = [ -VolGreen(Q Ja) + sum_faces lift(u* dS n) ] / J,  u* = (QL + QR)/2 or the
//        boundary's viscous state (BR1_ComputeGradient, Approximation/DGViscous_BR1.f90:48-111;
//        ComputeSolutionRiemann_*, DGViscousMethods.f90:538-917), or the interior-penalty local
//        gradient (ComputeInteriorGradient, Mesh/QuadElement_QuadProcedures.incf:42-88) -- and
//        writes only its traces on the four sides (interpolateGradientsToBoundaries,
//        DGSpatialDiscretizationMethods.f90:1577-1631);
//   ns_gradient_kernel also stores the BR1 gradient dQ ([n_el][2][4][NP], coalesced per node); the
//        interior-penalty gradient is element-local and the stage kernel recomputes it, so with IP the
//        gradient kernel runs only when something else needs it (gradient traces for viscous fluxes,
//        the artificial-viscosity indicator);
//   interior penalty with an element-local indicator (none, modal, learned): no gradient kernel per
//        stage.  The stage kernel ends with the gradient traces of the state it wrote (GT_out, the
//        other half of a ping-pong pair, as for the Q traces) and, on the last stage of a time step,
//        the indicator of that state (mu_next): everything the next stage reads from its neighbours.
//        The gradient kernel then runs only once after the state is replaced (hg_set_state);
//   ns_stage_kernel     reads the BR1 dQ back (written once, read once per stage),
//        F = Fi - Fv at the nodes (QDotVolumeLoop :243-268), face fluxes
//        F* = (Fi* - Fv*) dS with the neighbours' Q and dQ traces (BR1: (FvL+FvR)/2 . n; IP adds
//        sigma0 mu N^2 invh (uL - uR), DGViscous_IP.f90:45-130), boundary viscous fluxes by
//        condition (Dirichlet / adiabatic / Neumann, :1142-1511), the interior-penalty gradient-face
//        terms lifted by Scalar_StdGradientFace (DGWeakIntegrals.f90:268-495), 1/J, the RK update
//        and the new Q traces.
#pragma once
#include "hg_stage.cuh"
#include "hg_sensor.cuh"

namespace hg {

template <typename real>
struct NSArgs {
  int n_el;
  const int4* side;         // [n_el*4] {neighbour trace slot, flags, zone, per-node state row or -1}
  const real* side_geo;     // normals / dS (per node, or per side when AFFINE)
  const double* side_invh;  // [n_el*4] invh of the side's edge
  const real* vol_geo;      // Ja00 Ja01 Ja10 Ja11 1/J (per node, or per element when AFFINE)
  const real* jac;          // [n_el][NP] J per node (curved meshes)
  const double* mats;       // hatD[NP] lb0 lb1 lbw0 lbw1 [P each] D[NP] dlbw0 dlbw1 [P each]
  const Zone* zones;
  const double* bq;         // per-node Dirichlet states [rows][P][4] (sides whose side.w >= 0)
  const real* FX;           // exact-solver face fluxes [n_el*4][P][4] of this stage (RIEMANN_EXACT faces)
  const real* NF;           // mortar face fluxes [slots][P][4] of the SIDE_FLUX sides (stage kernel)
  const real* NFG;          // mortar BR1 gradient face terms [slots][P][2][4] of the SIDE_FLUX sides
  const real* NJ;           // mortar jump sums [slots][2] of the SIDE_FLUX sides (dissipation indicator)
  double* Q;
  real* G;
  const real* T_in;         // Q traces of the current state  [n_el*4][P][4]
  real* T_out;
  real* GT;                 // dQ traces of the current state [n_el*4][P][2][4]
  real* GT_out;             // dQ traces of the updated state (fused interior-penalty stages)
  real* dQ;                 // element gradients              [n_el][2][4][NP]
  int viscous;              // viscous fluxes present: mu != 0 or the Physical artificial viscosity
  int run_gradient;         // host side: whether this stage needs the gradient kernel
  int run_stage;            // host side: whether to launch the stage kernel (a composite runs the
                            // mortar fluxes between the parts' gradient and stage kernels)
  double* QDot;
  double* resid;
  double a, b, c;
  int first, update, riemann;
  int ip, grad_faces;       // interior penalty (else BR1); gradient-face terms (SIPG/NIPG)
  double sigma0, epsilon;
  PhysConst pc;
  // artificial dissipation (jumps-based indicator)
  int av;                   // 0 none, 1 Laplacian, 2 Physical
  const double* av_el;      // [n_el][2] Ceps sqrt(Volume)/(N+1), sum of the 4 edge areas
  const double* side_area;  // [n_el*4] Area of each side's edge
  double* mu_av;            // [n_el] element viscosity of the current state (written by the gradient kernel)
  SensorArgs sensor;        // which indicator sets it (jumps, modal, learned)
  int fuse;                 // interior penalty, element-local indicator: the stage kernel writes GT_out and,
  int last;                 //   on the last stage of a step (last), the indicator of its new state into
  double* mu_next;          //   mu_next
  int* health;              // device health word {bits, first element} (check_state)
  int* health_host;         // mapped host flag set beside it
};

__host__ __device__ constexpr int epb_ns(int P) {
  return P == 2 ? 16 : P == 3 ? 7 : P == 4 ? 8 : P == 5 ? 5 : P == 6 ? 4 : P == 7 ? 3 : P <= 9 ? 2 : 1;
}
__host__ __device__ constexpr int epb_ns_small(int P) {
  return P == 2 ? 4 : P <= 6 ? 2 : 1;
}
__host__ __device__ constexpr int epb_ns_of(int P, int variant) { return variant ? epb_ns_small(P) : epb_ns(P); }
__host__ __device__ constexpr int block_ns(int P) { return ((P * P * epb_ns(P) + 31) / 32) * 32; }

// Shared tiles of one CTA.
// ST: the stage kernel's tiles; the gradient kernel has no contravariant fluxes (Fc, Gc) and leaves
// that shared memory to the shock sensor.
template <int P, int EPB, typename real, bool AFFINE, bool ST = true>
struct NSTiles {
  static constexpr int NP = P * P, FT = 4 * P;
  real mat[3 * NP + 7 * P];   // hatD lb0 lb1 lbw0 lbw1 D dlbw0 dlbw1 w Vinv
  real Q[4][EPB][NP];
  real Ja[AFFINE ? 1 : 5][AFFINE ? 1 : EPB][AFFINE ? 1 : NP];   // Ja00 Ja01 Ja10 Ja11 J
  real dQ[2][4][EPB][NP];
  real Fc[ST ? 4 : 1][ST ? EPB : 1][ST ? NP : 1];
  real Gc[ST ? 4 : 1][ST ? EPB : 1][ST ? NP : 1];
  real face[12][EPB][FT];   // BR1 u* dS n (8) / F* (4) + gradient-face contravariant fluxes (8)
  real gfd[ST ? 4 : 1][ST ? EPB : 1][ST ? FT : 1];   // gradient-face terms contracted along their side
  real dl[ST && AFFINE ? 2 : 1][ST && AFFINE ? P : 1];   // (lb0^T D)(l), (lb1^T D)(l): normal derivatives at the sides
  double red[32][4];
};

template <int P, int EPB, typename real, bool AFFINE, bool ST>
__device__ __forceinline__ real trace_of(const NSTiles<P, EPB, real, AFFINE, ST>& s, const real (*src)[EPB][P * P], int k,
                                         int le, int side, int kk, const real* lbv) {
  real t = real(0);
#pragma unroll
  for (int m = 0; m < P; ++m) {
    const int l = trace_step<real>(P, m, kk);
    t += src[k][le][face_node(P, side, l, kk)] * lbv[l];
  }
  return t;
}

// The four variables' traces at face node kk of side `side` (the interpolant weights loaded once).
template <int P, int EPB, typename real>
__device__ __forceinline__ void trace4(const real (*src)[EPB][P * P], int le, int side, int kk, const real* lbv,
                                       real* out) {
#pragma unroll
  for (int k = 0; k < 4; ++k) out[k] = real(0);
#pragma unroll
  for (int m = 0; m < P; ++m) {
    const int l = trace_step<real>(P, m, kk);
    const int node = face_node(P, side, l, kk);
    const real w = lbv[l];
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] += src[k][le][node] * w;
  }
}

// Element gradient into s.dQ (both kernels).  Requires s.Q (and s.Ja) filled and synchronized.
template <int P, int EPB, typename real, bool AFFINE, bool IP, bool ST>
__device__ __forceinline__ void element_gradient(const NSArgs<real>& a, NSTiles<P, EPB, real, AFFINE, ST>& s,
                                                 const Phys<real>& ph, int le, int tid, int e, bool active,
                                                 const real* geoE) {
  constexpr int NP = P * P, FT = 4 * P;
  const real* hatDT = s.mat;   // transposed: hatDT[l * P + i] = hatD(i, l)
  const real* lb0 = s.mat + NP;
  const real* lb1 = lb0 + P;
  const real* lbw0 = lb1 + P;
  const real* lbw1 = lbw0 + P;
  const real* DT = lbw1 + P;   // transposed D
  const int i = tid % P, j = tid / P;
  if (!IP) {
    // BR1 face terms u* dS n (outward normal of this element)
    if (active) {
      for (int t = tid; t < FT; t += NP) {
        const int sd_ = t / P, kk = t % P;
        const int4 sd = a.side[size_t(e) * 4 + sd_];
        const int kind = sd.y & 15;
        if (kind == SIDE_FLUX) {   // p-nonconforming or subdivided edge: terms from the mortar kernel
          const real* gp = a.NFG + (size_t(sd.x) * P + kk) * 8;
#pragma unroll
          for (int k = 0; k < 8; ++k) s.face[k][le][t] = gp[k];
          continue;
        }
        const real* lbv = (sd_ == 0 || sd_ == 3) ? lb0 : lb1;
        real qo[4];
        trace4<P, EPB, real>(s.Q, le, sd_, kk, lbv, qo);
        const real* g3 = AFFINE ? a.side_geo + (size_t(e) * 4 + sd_) * 3 : a.side_geo + ((size_t(e) * 4 + sd_) * P + kk) * 3;
        const real nx = real(g3[0]), ny = real(g3[1]), dS = real(g3[2]);
        real us[4];
        if (kind == SIDE_LEFT || kind == SIDE_RIGHT) {
          const int kn = (sd.y & SIDE_REVERSED) ? (P - 1 - kk) : kk;
          real tp[4];
          ld4(a.T_in + (size_t(sd.x) * P + kn) * 4, tp);
#pragma unroll
          for (int k = 0; k < 4; ++k) us[k] = kind == SIDE_RIGHT ? real(0.5) * (tp[k] + qo[k]) : real(0.5) * (qo[k] + tp[k]);
        } else {
          real uB[4];
          bc_states(ph, a.zones[sd.z], qo, nx, ny, uB, us, sd.w >= 0 ? a.bq + (size_t(sd.w) * P + kk) * 4 : nullptr);
        }
        const real sg = kind == SIDE_RIGHT ? real(-1) : real(1);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          s.face[k][le][t] = (sg * us[k]) * dS * nx;
          s.face[4 + k][le][t] = (sg * us[k]) * dS * ny;
        }
      }
    }
    __syncthreads();
  }
  if (active) {
    real Ja00, Ja01, Ja10, Ja11, iJ;
    if constexpr (AFFINE) { Ja00 = geoE[0]; Ja01 = geoE[1]; Ja10 = geoE[2]; Ja11 = geoE[3]; iJ = geoE[4]; }
    else { Ja00 = s.Ja[0][le][tid]; Ja01 = s.Ja[1][le][tid]; Ja10 = s.Ja[2][le][tid]; Ja11 = s.Ja[3][le][tid];
           iJ = real(1) / s.Ja[4][le][tid]; }
    // the operator rows and metrics of a node are loaded once per l and reused for the 4 variables
    if (IP) {
      real dxi[4] = {real(0), real(0), real(0), real(0)}, deta[4] = {real(0), real(0), real(0), real(0)};
#pragma unroll
      for (int l = 0; l < P; ++l) {
        const real di = DT[l * P + i], dj = DT[l * P + j];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          dxi[k] += di * s.Q[k][le][j * P + l];
          deta[k] += dj * s.Q[k][le][l * P + i];
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        s.dQ[0][k][le][tid] = (dxi[k] * Ja00 + deta[k] * Ja01) * iJ;
        s.dQ[1][k][le][tid] = (dxi[k] * Ja10 + deta[k] * Ja11) * iJ;
      }
    } else {
      real v0[4] = {real(0), real(0), real(0), real(0)}, v1[4] = {real(0), real(0), real(0), real(0)};
      if constexpr (AFFINE) {
        real axi[4] = {real(0), real(0), real(0), real(0)}, aeta[4] = {real(0), real(0), real(0), real(0)};
#pragma unroll
        for (int l = 0; l < P; ++l) {
          const real hi = hatDT[l * P + i], hj = hatDT[l * P + j];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            axi[k] += hi * s.Q[k][le][j * P + l];
            aeta[k] += hj * s.Q[k][le][l * P + i];
          }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          v0[k] = axi[k] * Ja00 + aeta[k] * Ja01;
          v1[k] = axi[k] * Ja10 + aeta[k] * Ja11;
        }
      } else {
#pragma unroll
        for (int l = 0; l < P; ++l) {
          const int nx_ = j * P + l, ny_ = l * P + i;
          const real hi = hatDT[l * P + i], hj = hatDT[l * P + j];
          const real j0 = s.Ja[0][le][nx_], j1 = s.Ja[1][le][ny_], j2 = s.Ja[2][le][nx_], j3 = s.Ja[3][le][ny_];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const real qx = s.Q[k][le][nx_] * hi, qy = s.Q[k][le][ny_] * hj;
            v0[k] += qx * j0 + qy * j1;
            v1[k] += qx * j2 + qy * j3;
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const real l0 = s.face[k][le][0 * P + i] * lbw0[j] + s.face[k][le][1 * P + j] * lbw1[i] +
                        s.face[k][le][2 * P + i] * lbw1[j] + s.face[k][le][3 * P + j] * lbw0[i];
        const real l1 = s.face[4 + k][le][0 * P + i] * lbw0[j] + s.face[4 + k][le][1 * P + j] * lbw1[i] +
                        s.face[4 + k][le][2 * P + i] * lbw1[j] + s.face[4 + k][le][3 * P + j] * lbw0[i];
        s.dQ[0][k][le][tid] = (-v0[k] + l0) * iJ;
        s.dQ[1][k][le][tid] = (-v1[k] + l1) * iJ;
      }
    }
  }
}

template <int P, int EPB, typename real, bool AFFINE, bool ST>
__device__ __forceinline__ void load_tiles(const NSArgs<real>& a, NSTiles<P, EPB, real, AFFINE, ST>& s, int flat, int le,
                                           int tid, int e, bool active, real* geoE) {
  constexpr int NP = P * P;
  // hatD and D are held transposed (column l contiguous): a warp then reads hatD(i, l) over its nodes'
  // i from consecutive words instead of a stride of P (bank conflicts)
  for (int k = flat; k < 3 * NP + 7 * P; k += blockDim.x) {
    int src = k;
    if (k < NP) src = (k % P) * P + k / P;
    else if (k >= NP + 4 * P && k < 2 * NP + 4 * P) { const int m = k - NP - 4 * P; src = NP + 4 * P + (m % P) * P + m / P; }
    s.mat[k] = real(a.mats[src]);
  }
  if (active) {
    const double2* qp = reinterpret_cast<const double2*>(a.Q + (size_t(e) * NP + tid) * 4);
    const double2 q01 = qp[0], q23 = qp[1];
    s.Q[0][le][tid] = real(q01.x); s.Q[1][le][tid] = real(q01.y);
    s.Q[2][le][tid] = real(q23.x); s.Q[3][le][tid] = real(q23.y);
    if constexpr (AFFINE) {
#pragma unroll
      for (int k = 0; k < 5; ++k) geoE[k] = real(a.vol_geo[size_t(e) * 5 + k]);
    } else {
      const real* gp = a.vol_geo + (size_t(e) * NP + tid) * 5;
#pragma unroll
      for (int k = 0; k < 4; ++k) s.Ja[k][le][tid] = real(gp[k]);
      s.Ja[4][le][tid] = real(a.jac[size_t(e) * NP + tid]);
      geoE[4] = real(gp[4]);
    }
  }
}

// JumpsBasedElementViscosity (Approximation/DGArtificialDissipation.f90:277-338) of each element of the
// CTA into a.mu_av.  Edge jumps (Edge_ComputeJumps and the boundary/curved variants,
// Mesh/QuadElement_EdgeProcedures.incf:1348-1619): sum over the edge nodes, in the edge's order, of
// w (2 (QL-QR)/(QL+QR))^2 dS for rho and rhoE; boundary and periodic edges use the viscous boundary
// state (uSB) and dS at their first node.  Uses s.face[0..1] as scratch; ends with a barrier.
template <int P, int EPB, typename real, bool AFFINE, bool ST>
__device__ __forceinline__ void element_viscosity(const NSArgs<real>& a, NSTiles<P, EPB, real, AFFINE, ST>& s,
                                                  const Phys<real>& ph, int le, int tid, int e, bool active) {
  constexpr int NP = P * P, FT = 4 * P;
  if (a.sensor.kind != SENSOR_JUMPS) {   // modal-decay or learned indicator (hg_sensor.cuh)
    // evaluated on the first stage of a time step (and for a bare time derivative); the later stages
    // of the step keep that viscosity.  The reference's jumps indicator is re-evaluated every stage.
    if (!a.first) return;
    const int n_active = a.n_el - int(blockIdx.x) * EPB < EPB ? a.n_el - int(blockIdx.x) * EPB : EPB;
    const SensorOut so = element_sensor<P, EPB, real>(a.sensor, ph, s.Q, n_active, s.mat + 2 * NP + 7 * P, le,
                                                      tid, active, nullptr);
    if (active && tid == 0) a.mu_av[e] = a.av_el[2 * size_t(e)] * so.g;
    __syncthreads();
    return;
  }
  const real* lb0 = s.mat + NP;
  const real* lb1 = lb0 + P;
  const real* wq = s.mat + 2 * NP + 6 * P;
  if (active) {
    for (int t = tid; t < FT; t += NP) {
      const int sd_ = t / P, kk = t % P;
      const int4 sd = a.side[size_t(e) * 4 + sd_];
      const int kind = sd.y & 15;
      if (kind == SIDE_FLUX) {   // edge between orders or subdivided edge: the mortar kernel's jump sums
        s.face[0][le][t] = kk == 0 ? a.NJ[size_t(sd.x) * 2] : real(0);
        s.face[1][le][t] = kk == 0 ? a.NJ[size_t(sd.x) * 2 + 1] : real(0);
        continue;
      }
      const real* lbv = (sd_ == 0 || sd_ == 3) ? lb0 : lb1;
      real qo[4];
      trace4<P, EPB, real>(s.Q, le, sd_, kk, lbv, qo);
      const size_t sbase = size_t(e) * 4 + sd_;
      real qn0, qn3;
      bool node0 = true;
      if (kind == SIDE_LEFT || kind == SIDE_RIGHT) {
        const int kn = (sd.y & SIDE_REVERSED) ? (P - 1 - kk) : kk;
        const real* tp = a.T_in + (size_t(sd.x) * P + kn) * 4;
        qn0 = tp[0];
        qn3 = tp[3];
        node0 = sd.z >= 0;   // periodic edges are boundary edges of the reference
      } else {
        const real* g3 = AFFINE ? a.side_geo + sbase * 3 : a.side_geo + (sbase * P + kk) * 3;
        real uB[4], uS[4];
        bc_states(ph, a.zones[sd.z], qo, real(g3[0]), real(g3[1]), uB, uS,
                  sd.w >= 0 ? a.bq + (size_t(sd.w) * P + kk) * 4 : nullptr);
        qn0 = uS[0];
        qn3 = uS[3];
      }
      const real dSn = real(AFFINE ? a.side_geo[sbase * 3 + 2] : a.side_geo[(sbase * P + (node0 ? 0 : kk)) * 3 + 2]);
      const real jr = real(2) * (qo[0] - qn0) / (qo[0] + qn0);
      const real je = real(2) * (qo[3] - qn3) / (qo[3] + qn3);
      s.face[0][le][t] = wq[kk] * jr * jr * dSn;
      s.face[1][le][t] = wq[kk] * je * je * dSn;
    }
  }
  __syncthreads();
  if (active && tid == 0) {
    real gr = real(0), ge = real(0);
#pragma unroll
    for (int sd_ = 0; sd_ < 4; ++sd_) {
      const int fl = a.side[size_t(e) * 4 + sd_].y;
      const bool rev = (fl & 15) == SIDE_RIGHT && (fl & SIDE_REVERSED);
      real sr = real(0), se = real(0);
      for (int n = 0; n < P; ++n) {
        const int kk = rev ? (P - 1 - n) : n;
        sr = sr + s.face[0][le][sd_ * P + kk];
        se = se + s.face[1][le][sd_ * P + kk];
      }
      gr = gr + sr;
      ge = ge + se;
    }
    double gk = double(gr > ge ? gr : ge) / a.av_el[2 * size_t(e) + 1];
    gk = gk > 1.0e-8 ? log10(gk) : -1.7976931348623157e308;
    const double k = 5.0;
    const double s0 = log10(1.0 / ((P * P) * double(P * P))) + 1.0;
    double G;
    if (gk < s0 - k) G = 0.0;
    else if (gk < s0 + k) G = 0.5 * sin(0.5 * 3.141592653589793238462643 * (gk - s0) / k) + 0.5;
    else G = 1.0;
    a.mu_av[e] = a.av_el[2 * size_t(e)] * G;
  }
}

template <int P, int EPB, typename real, bool AFFINE, bool IP, bool AV>
__global__ void __launch_bounds__(block_of(P, EPB)) ns_gradient_kernel(NSArgs<real> a) {
  constexpr int NP = P * P, FT = 4 * P;
  __shared__ NSTiles<P, EPB, real, AFFINE, false> s;
  const int flat = threadIdx.x, le = flat / NP, tid = flat - le * NP;
  const int e = blockIdx.x * EPB + le;
  const bool active = le < EPB && e < a.n_el;
  Phys<real> ph;
  ph.load(a.pc);
  real geoE[5];
  load_tiles(a, s, flat, le, tid, e, active, geoE);
  __syncthreads();
  // the interior-penalty gradient is element-local: without viscous fluxes nothing here uses it (the
  // launch then only evaluates the indicator); a.viscous is uniform over the launch
  if (!IP || a.viscous) {
    element_gradient<P, EPB, real, AFFINE, IP>(a, s, ph, le, tid, e, active, geoE);
    __syncthreads();
  }
  if (AV) element_viscosity<P, EPB, real, AFFINE>(a, s, ph, le, tid, e, active);
  if (!active) return;
  if (!IP) {   // the lifted gradient is not local: store it for the stage kernel
    real* g = a.dQ + size_t(e) * 8 * NP + tid;
#pragma unroll
    for (int d = 0; d < 2; ++d)
#pragma unroll
      for (int k = 0; k < 4; ++k) g[(d * 4 + k) * NP] = s.dQ[d][k][le][tid];
  }
  if (!a.viscous) return;   // gradient traces only feed viscous face fluxes
  const real* lb0 = s.mat + NP;
  const real* lb1 = lb0 + P;
  for (int t = tid; t < FT; t += NP) {
    const int sd_ = t / P, kk = t % P;
    const real* lbv = (sd_ == 0 || sd_ == 3) ? lb0 : lb1;
    real* gp = a.GT + ((size_t(e) * 4 + sd_) * P + kk) * 8;
    real tx[4], ty[4];
    trace4<P, EPB, real>(s.dQ[0], le, sd_, kk, lbv, tx);
    trace4<P, EPB, real>(s.dQ[1], le, sd_, kk, lbv, ty);
    st4(gp, tx);
    st4(gp + 4, ty);
  }
}

// Volume flux of node n of element le: F = Fi - (mu + mu_a) Fv (- mu_a grad Q for the Laplacian
// dissipation), contravariant, into s.Fc and s.Gc (QDotVolumeLoop, DGSpatialDiscretizationMethods.f90:
// 243-268).  Reads the node's Q and gradient from the tiles.
template <int P, int EPB, typename real, bool AFFINE, bool IP, bool AV>
__device__ __forceinline__ void ns_volume_flux(const NSArgs<real>& a, NSTiles<P, EPB, real, AFFINE>& s,
                                               const Phys<real>& ph, int le, int n, real mu_e, bool need_grad,
                                               bool visc, const real* geoE) {
  constexpr int NP = P * P;
  const int i = n % P, j = n / P;
  const real mu = ph.mu;
  real Ja00, Ja01, Ja10, Ja11;
  if constexpr (AFFINE) { Ja00 = geoE[0]; Ja01 = geoE[1]; Ja10 = geoE[2]; Ja11 = geoE[3]; }
  else { Ja00 = s.Ja[0][le][n]; Ja01 = s.Ja[1][le][n]; Ja10 = s.Ja[2][le][n]; Ja11 = s.Ja[3][le][n]; }
  real q[4], gx[4], gy[4], fi[4], gi[4], fv[4], gv[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) { q[k] = s.Q[k][le][n]; gx[k] = s.dQ[0][k][le][n]; gy[k] = s.dQ[1][k][le][n]; }
  inviscid_flux(ph, q, fi, gi);
  if (visc) viscous_flux(ph, q, gx, gy, fv, gv);
  else {
#pragma unroll
    for (int k = 0; k < 4; ++k) { fv[k] = real(0); gv[k] = real(0); }
  }
  const real mu_v = (AV && a.av == 2) ? mu + mu_e : mu;
  real ax[4] = {real(0), real(0), real(0), real(0)}, ay[4] = {real(0), real(0), real(0), real(0)};
  if (AV && a.av == 1 && need_grad) {   // Laplacian: mu_e times the element-local gradient (ComputeInteriorGradient)
    if (IP) {
#pragma unroll
      for (int k = 0; k < 4; ++k) { ax[k] = gx[k]; ay[k] = gy[k]; }
    } else {
      const real* DT = s.mat + NP + 4 * P;   // D (transposed) follows hatD, lb0, lb1, lbw0, lbw1
      const real iJl = AFFINE ? geoE[4] : real(1) / s.Ja[4][le][n];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        real dxi = real(0), deta = real(0);
#pragma unroll
        for (int l = 0; l < P; ++l) {
          dxi += DT[l * P + i] * s.Q[k][le][j * P + l];
          deta += DT[l * P + j] * s.Q[k][le][l * P + i];
        }
        ax[k] = (dxi * Ja00 + deta * Ja01) * iJl;
        ay[k] = (dxi * Ja10 + deta * Ja11) * iJl;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    real f = fi[k] - mu_v * fv[k], g = gi[k] - mu_v * gv[k];
    if (AV && a.av == 1) { f = f - mu_e * ax[k]; g = g - mu_e * ay[k]; }
    s.Fc[k][le][n] = f * Ja00 + g * Ja10;
    s.Gc[k][le][n] = f * Ja01 + g * Ja11;
  }
}

// Face node t (= side * P + kk) of element le: the side's flux F* dS (signed for a RIGHT side) into
// s.face[0..3] and, with SIPG / NIPG, the contravariant gradient-face terms into s.face[4..11]
// (ComputeRiemannSolver_* and the viscous face loops, DGSpatialDiscretizationMethods.f90:545-1511;
// DGViscous_BR1.f90:311-371, DGViscous_IP.f90:120-134, 240-247; DGArtificialDissipation.f90:208-249).
template <int P, int EPB, typename real, bool AFFINE, bool IP, bool AV>
__device__ __forceinline__ void ns_face_task(const NSArgs<real>& a, NSTiles<P, EPB, real, AFFINE>& s,
                                             const Phys<real>& ph, int le, int e, int t, real mu_e, bool visc,
                                             const real* geoE, const real (*own)[EPB][4 * P], bool own_g) {
  constexpr int NP = P * P;
  const real mu = ph.mu;
  const real* lb0 = s.mat + NP;
  const real* lb1 = lb0 + P;
  const int sd_ = t / P, kk = t % P;
  const int4 sd = a.side[size_t(e) * 4 + sd_];
  const int kind = sd.y & 15;
  if (kind == SIDE_FLUX) {   // inviscid and viscous flux of the mortar kernel, and its gradient-face terms
    real fp[4];
    ld4(a.NF + (size_t(sd.x) * P + kk) * 4, fp);
#pragma unroll
    for (int k = 0; k < 4; ++k) s.face[k][le][t] = fp[k];
    if (IP && a.grad_faces && visc) {
      const real* gp = a.NFG + (size_t(sd.x) * P + kk) * 8;
      const real* lbv = (sd_ == 0 || sd_ == 3) ? lb0 : lb1;
      real fJa00, fJa01, fJa10, fJa11, fiJ;   // metrics and 1/J at the face node
      if constexpr (AFFINE) { fJa00 = geoE[0]; fJa01 = geoE[1]; fJa10 = geoE[2]; fJa11 = geoE[3]; fiJ = geoE[4]; }
      else {
        fJa00 = trace_of(s, s.Ja, 0, le, sd_, kk, lbv);
        fJa01 = trace_of(s, s.Ja, 1, le, sd_, kk, lbv);
        fJa10 = trace_of(s, s.Ja, 2, le, sd_, kk, lbv);
        fJa11 = trace_of(s, s.Ja, 3, le, sd_, kk, lbv);
        fiJ = real(1) / trace_of(s, s.Ja, 4, le, sd_, kk, lbv);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        s.face[4 + k][le][t] = (gp[k] * fJa00 + gp[4 + k] * fJa10) * fiJ;
        s.face[8 + k][le][t] = (gp[k] * fJa01 + gp[4 + k] * fJa11) * fiJ;
      }
    }
    return;
  }
  const real* lbv = (sd_ == 0 || sd_ == 3) ? lb0 : lb1;
  real qo[4], gox[4] = {real(0), real(0), real(0), real(0)}, goy[4] = {real(0), real(0), real(0), real(0)};
  // this element's own traces of the current state (Q, and the gradient when viscous): what the previous
  // stage (or the prologue, or this stage's gradient kernel) wrote for the neighbours, prefetched
  cp_async_wait_all();
#pragma unroll
  for (int k = 0; k < 4; ++k) qo[k] = own[k][le][t];
  if (visc) {
    if (own_g) {
#pragma unroll
      for (int k = 0; k < 4; ++k) { gox[k] = own[4 + k][le][t]; goy[k] = own[8 + k][le][t]; }
    } else {   // no shared memory left for them: formed here
      trace4<P, EPB, real>(s.dQ[0], le, sd_, kk, lbv, gox);
      trace4<P, EPB, real>(s.dQ[1], le, sd_, kk, lbv, goy);
    }
  }
  const real* g3 = AFFINE ? a.side_geo + (size_t(e) * 4 + sd_) * 3 : a.side_geo + ((size_t(e) * 4 + sd_) * P + kk) * 3;
  const real nx = real(g3[0]), ny = real(g3[1]), dS = real(g3[2]);
  const real invh = real(a.side_invh[size_t(e) * 4 + sd_]);
  // edge viscosity (JumpsBasedEdgeViscosity): mean over the edge's elements; boundary and
  // periodic edges have one element
  real mu_ed = mu_e;
  if (AV && (kind == SIDE_LEFT || kind == SIDE_RIGHT) && sd.z < 0)
    mu_ed = (real(a.mu_av[sd.x >> 2]) + mu_e) / real(2);
  const real mu_f = (AV && a.av == 2) ? mu + mu_ed : mu;
  const real lap = (AV && a.av == 1) ? mu_ed * real(a.side_area[size_t(e) * 4 + sd_]) : real(0);
  const real penalty = IP ? real(a.sigma0) * mu_f * real(P - 1) * real(P - 1) * invh : real(0);
  real F[4], Gx[4] = {real(0), real(0), real(0), real(0)}, Gy[4] = {real(0), real(0), real(0), real(0)};
  if (kind == SIDE_LEFT || kind == SIDE_RIGHT) {
    real qn[4], gnx[4] = {real(0), real(0), real(0), real(0)}, gny[4] = {real(0), real(0), real(0), real(0)};
    // the neighbour's traces, prefetched into this task's own face slots (prefetch_neighbour_traces)
    cp_async_wait_all();
#pragma unroll
    for (int k = 0; k < 4; ++k) qn[k] = s.face[k][le][t];
    if (visc) {
#pragma unroll
      for (int k = 0; k < 4; ++k) { gnx[k] = s.face[4 + k][le][t]; gny[k] = s.face[8 + k][le][t]; }
    }
    const bool right = kind == SIDE_RIGHT;
    const real* QL = right ? qn : qo;
    const real* QR = right ? qo : qn;
    int solver = a.riemann;
    if (sd.z >= 0) { const int zr = a.zones[sd.z].riemann; if (zr >= 0) solver = zr; }
    real Fi[4], FLx[4] = {real(0), real(0), real(0), real(0)}, FLy[4] = {real(0), real(0), real(0), real(0)};
    real FRx[4] = {real(0), real(0), real(0), real(0)}, FRy[4] = {real(0), real(0), real(0), real(0)};
    face_riemann(solver, ph, QL, QR, nx, ny, a.FX, (size_t(e) * 4 + sd_) * P + kk, Fi);
    if (visc) {
      viscous_flux(ph, QL, right ? gnx : gox, right ? gny : goy, FLx, FLy);
      viscous_flux(ph, QR, right ? gox : gnx, right ? goy : gny, FRx, FRy);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      real fv = real(0.5) * (mu_f * FLx[k] + mu_f * FRx[k]) * nx + real(0.5) * (mu_f * FLy[k] + mu_f * FRy[k]) * ny;
      if (IP) fv = fv - penalty * (QL[k] - QR[k]);
      if (AV) {
        const real fa = -(lap * (QL[k] - QR[k]));
        F[k] = (Fi[k] - fv - fa) * dS;
      } else {
        F[k] = (Fi[k] - fv) * dS;
      }
      if (right) F[k] = -F[k];
    }
    if (IP && a.grad_faces && visc) {
      real fgx[4], fgy[4], Ax[4], Ay[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) { fgx[k] = (QL[k] - QR[k]) * nx; fgy[k] = (QL[k] - QR[k]) * ny; }
      viscous_flux(ph, right ? QR : QL, fgx, fgy, Ax, Ay);
      const real cf = (right ? real(-0.5) : real(0.5)) * real(a.epsilon) * mu_f;
#pragma unroll
      for (int k = 0; k < 4; ++k) { Gx[k] = cf * Ax[k] * dS; Gy[k] = cf * Ay[k] * dS; }
    }
  } else {
    const Zone& z = a.zones[sd.z];
    real uB[4], uSB[4];
    const int vbc = bc_states(ph, z, qo, nx, ny, uB, uSB, sd.w >= 0 ? a.bq + (size_t(sd.w) * P + kk) * 4 : nullptr);
    real Fi[4];
    if (kind == SIDE_WALL) {
      euler_wall_flux(ph, qo, nx, ny, dS, Fi);
    } else {
      const int solver = z.riemann >= 0 ? z.riemann : a.riemann;
      face_riemann(solver, ph, qo, uB, nx, ny, a.FX, (size_t(e) * 4 + sd_) * P + kk, Fi);
#pragma unroll
      for (int k = 0; k < 4; ++k) Fi[k] = Fi[k] * dS;
    }
    real fv[4] = {real(0), real(0), real(0), real(0)};
    if (vbc != VBC_NEUMANN && visc) {
      real Fx[4], Fy[4];
      if (vbc == VBC_ADIABATIC) viscous_flux_adiabatic(ph, qo, qo, gox, goy, Fx, Fy);
      else viscous_flux(ph, qo, gox, goy, Fx, Fy);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        fv[k] = (mu_f * Fx[k]) * nx + (mu_f * Fy[k]) * ny;
        if (IP) fv[k] = fv[k] - penalty * (qo[k] - uSB[k]);
        fv[k] = fv[k] * dS;
      }
      if (IP && a.grad_faces) {
        real fgx[4], fgy[4], Ax[4], Ay[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) { fgx[k] = (qo[k] - uSB[k]) * nx; fgy[k] = (qo[k] - uSB[k]) * ny; }
        if (vbc == VBC_ADIABATIC) viscous_flux_adiabatic(ph, qo, qo, fgx, fgy, Ax, Ay);
        else viscous_flux(ph, qo, fgx, fgy, Ax, Ay);
        const real cf = real(a.epsilon) * mu_f;
#pragma unroll
        for (int k = 0; k < 4; ++k) { Gx[k] = (cf * Ax[k]) * dS; Gy[k] = (cf * Ay[k]) * dS; }
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) F[k] = AV ? Fi[k] - fv[k] - (-(lap * (qo[k] - uSB[k]))) * dS : Fi[k] - fv[k];
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) s.face[k][le][t] = F[k];
  if (IP && a.grad_faces && visc) {
    // metrics at the face node (interpolated along the other direction) and contravariant G
    real fJa00, fJa01, fJa10, fJa11, fiJ;   // metrics and 1/J at the face node (one division, or none)
    if constexpr (AFFINE) { fJa00 = geoE[0]; fJa01 = geoE[1]; fJa10 = geoE[2]; fJa11 = geoE[3]; fiJ = geoE[4]; }
    else {
      fJa00 = trace_of(s, s.Ja, 0, le, sd_, kk, lbv);
      fJa01 = trace_of(s, s.Ja, 1, le, sd_, kk, lbv);
      fJa10 = trace_of(s, s.Ja, 2, le, sd_, kk, lbv);
      fJa11 = trace_of(s, s.Ja, 3, le, sd_, kk, lbv);
      fiJ = real(1) / trace_of(s, s.Ja, 4, le, sd_, kk, lbv);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      s.face[4 + k][le][t] = (Gx[k] * fJa00 + Gy[k] * fJa10) * fiJ;
      s.face[8 + k][le][t] = (Gx[k] * fJa01 + Gy[k] * fJa11) * fiJ;
    }
  }
}

// The traces that the face tasks of this thread read (Q traces, and the gradient traces when viscous),
// copied asynchronously at the start of the launch: the neighbour's into the task's own face slots
// (face[0..3][le][t] and face[4..11][le][t] belong to face task t alone, which reads them before it
// writes its fluxes there), this element's own into s.own (the trace buffers hold them: the previous
// stage's output, the prologue's, or this stage's gradient kernel's), so the copies need no barrier
// and their latency overlaps the volume phase.  The thread-to-task map is that of the face phase
// (t = tid, tid + NP, ...).
template <int P, int EPB, typename real, bool AFFINE>
__device__ __forceinline__ void prefetch_neighbour_traces(const NSArgs<real>& a, NSTiles<P, EPB, real, AFFINE>& s,
                                                          real (*own)[EPB][4 * P], bool own_g, int le, int e,
                                                          int tid, bool active, bool visc) {
  constexpr int NP = P * P, FT = 4 * P;
  if (active)
    for (int t = tid; t < FT; t += NP) {
      const int sd_ = t / P, kk = t % P;
      const int4 sd = a.side[size_t(e) * 4 + sd_];
      const int kind = sd.y & 15;
      if (kind != SIDE_FLUX) {
        const size_t slot = (size_t(e) * 4 + sd_) * P + kk;
#pragma unroll
        for (int k = 0; k < 4; ++k) cp_async_real(&own[k][le][t], a.T_in + slot * 4 + k);
        if (visc && own_g) {
#pragma unroll
          for (int k = 0; k < 8; ++k) cp_async_real(&own[4 + k][le][t], a.GT + slot * 8 + k);
        }
      }
      if (kind == SIDE_LEFT || kind == SIDE_RIGHT) {
        const int kn = (sd.y & SIDE_REVERSED) ? (P - 1 - kk) : kk;
        const real* qp = a.T_in + (size_t(sd.x) * P + kn) * 4;
#pragma unroll
        for (int k = 0; k < 4; ++k) cp_async_real(&s.face[k][le][t], qp + k);
        if (visc) {
          const real* gp = a.GT + (size_t(sd.x) * P + kn) * 8;
#pragma unroll
          for (int k = 0; k < 8; ++k) cp_async_real(&s.face[4 + k][le][t], gp + k);
        }
      }
    }
  cp_async_commit();
}

template <int P, int EPB, typename real, bool AFFINE, bool IP, bool AV>
__global__ void __launch_bounds__(block_of(P, EPB)) ns_stage_kernel(NSArgs<real> a) {
  constexpr int NP = P * P, FT = 4 * P;
  constexpr int NW = block_of(P, EPB) / 32;
  __shared__ NSTiles<P, EPB, real, AFFINE> s;
  const int flat = threadIdx.x, le = flat / NP, tid = flat - le * NP;
  const int e = blockIdx.x * EPB + le;
  const bool active = le < EPB && e < a.n_el;
  Phys<real> ph;
  ph.load(a.pc);
  const real mu = ph.mu;
  real geoE[5];
  const bool visc = a.viscous != 0;
  // the own traces of the face tasks: Q and gradient where the static shared memory allows (48 KB),
  // else Q alone (the gradient traces are then formed in the face task)
  constexpr bool OWN_G = sizeof(s) + size_t(12) * EPB * FT * sizeof(real) <= 48 * 1024;
  __shared__ real s_own[OWN_G ? 12 : 4][EPB][FT];
  prefetch_neighbour_traces<P, EPB, real, AFFINE>(a, s, s_own, OWN_G, le, e, tid, active, visc);
  load_tiles(a, s, flat, le, tid, e, active, geoE);
  const real mu_e = (AV && active) ? real(a.mu_av[e]) : real(0);
  // the element gradient feeds the viscous fluxes and the Laplacian dissipation's volume term; an
  // element without either (mu_e = 0: that term is exactly zero) skips it
  const bool need_grad = visc || (AV && a.av == 1 && mu_e != real(0));
  if (IP) {   // the interior-penalty gradient is element-local: recompute it here
    __syncthreads();
    element_gradient<P, EPB, real, AFFINE, IP>(a, s, ph, le, tid, e, active && need_grad, geoE);
  } else if (active) {
    const real* g = a.dQ + size_t(e) * 8 * NP + tid;
#pragma unroll
    for (int d = 0; d < 2; ++d)
#pragma unroll
      for (int k = 0; k < 4; ++k) s.dQ[d][k][le][tid] = g[(d * 4 + k) * NP];
  }
  __syncthreads();
  const int i = tid % P, j = tid / P;
  const real* hatDT = s.mat;   // transposed: hatDT[l * P + i] = hatD(i, l)
  const real* lb0 = s.mat + NP;
  const real* lb1 = lb0 + P;
  const real* lbw0 = lb1 + P;
  const real* lbw1 = lbw0 + P;
  const real* dlbw0 = lbw1 + P + NP;
  const real* dlbw1 = dlbw0 + P;
  real iJ;
  if (active) iJ = geoE[4];
  // Volume fluxes and face fluxes are independent: where an element has at least a quarter of its
  // threads beyond its 4(N+1) face nodes (N >= 5), those threads form the volume fluxes of all its nodes
  // while the first 4(N+1) threads form the face fluxes (one barrier fewer, and no thread idles through
  // the face phase); otherwise each thread forms its own node's volume flux, then the face fluxes.
  constexpr bool OVERLAP = 4 * (NP - FT) >= NP;
  if constexpr (OVERLAP) {
    if (active) {
      if (tid < FT) ns_face_task<P, EPB, real, AFFINE, IP, AV>(a, s, ph, le, e, tid, mu_e, visc, geoE, s_own, OWN_G);
      else
        for (int n = tid - FT; n < NP; n += NP - FT)
          ns_volume_flux<P, EPB, real, AFFINE, IP, AV>(a, s, ph, le, n, mu_e, need_grad, visc, geoE);
    }
  } else {
    if (active) ns_volume_flux<P, EPB, real, AFFINE, IP, AV>(a, s, ph, le, tid, mu_e, need_grad, visc, geoE);
    __syncthreads();
    if (active)
      for (int t = tid; t < FT; t += NP)
        ns_face_task<P, EPB, real, AFFINE, IP, AV>(a, s, ph, le, e, t, mu_e, visc, geoE, s_own, OWN_G);
  }
  __syncthreads();
  // The gradient-face terms enter the lift as hatD-contractions along their side, which depend on the
  // node's index along that side only (Scalar_StdGradientFace): formed once per side node here (P
  // multiply-adds each) instead of at every node of the element.
  const bool gf = IP && a.grad_faces && visc;   // uniform over the launch
  if (gf && active) {
    for (int t = tid; t < FT; t += NP) {
      const int sd_ = t / P, kk = t % P;
      const int row = (sd_ & 1) ? 8 : 4;   // bottom / top: the xi component; right / left: the eta one
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        real d = real(0);
#pragma unroll
        for (int l = 0; l < P; ++l) d += hatDT[l * P + kk] * s.face[row + k][le][sd_ * P + l];
        s.gfd[k][le][t] = d;
      }
    }
  }
  real qd[4] = {real(0), real(0), real(0), real(0)};
  if (active) {
#pragma unroll
    for (int l = 0; l < P; ++l) {
      const real hi = hatDT[l * P + i], hj = hatDT[l * P + j];
#pragma unroll
      for (int k = 0; k < 4; ++k) qd[k] = qd[k] + hi * s.Fc[k][le][j * P + l] + hj * s.Gc[k][le][l * P + i];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      qd[k] = qd[k] - s.face[k][le][0 * P + i] * lbw0[j];
      qd[k] = qd[k] - s.face[k][le][1 * P + j] * lbw1[i];
      qd[k] = qd[k] - s.face[k][le][2 * P + i] * lbw1[j];
      qd[k] = qd[k] - s.face[k][le][3 * P + j] * lbw0[i];
    }
  }
  if (gf) __syncthreads();
  if (active) {
    if (gf) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        qd[k] = qd[k] - (s.gfd[k][le][0 * P + i] * lbw0[j] + s.face[8 + k][le][0 * P + i] * dlbw0[j]);
        qd[k] = qd[k] - (s.face[4 + k][le][1 * P + j] * dlbw1[i] + s.gfd[k][le][1 * P + j] * lbw1[i]);
        qd[k] = qd[k] - (s.gfd[k][le][2 * P + i] * lbw1[j] + s.face[8 + k][le][2 * P + i] * dlbw1[j]);
        qd[k] = qd[k] - (s.face[4 + k][le][3 * P + j] * dlbw0[i] + s.gfd[k][le][3 * P + j] * lbw0[i]);
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) qd[k] = qd[k] * iJ;
    const size_t off = (size_t(e) * NP + tid) * 4;
    if (a.QDot) {
      double2* dp = reinterpret_cast<double2*>(a.QDot + off);
      dp[0] = make_double2(double(qd[0]), double(qd[1]));
      dp[1] = make_double2(double(qd[2]), double(qd[3]));
    }
    if (a.update) {
      real gn[4];
      if (a.first) {
#pragma unroll
        for (int k = 0; k < 4; ++k) gn[k] = real(a.b) * qd[k];
      } else {
        real go[4];
        ld4(a.G + off, go);
#pragma unroll
        for (int k = 0; k < 4; ++k) gn[k] = real(a.a) * go[k] + real(a.b) * qd[k];
      }
      st4(a.G + off, gn);
      double2* qp = reinterpret_cast<double2*>(a.Q + off);
      double2 q01 = qp[0], q23 = qp[1];
      q01.x = q01.x + a.c * double(gn[0]);
      q01.y = q01.y + a.c * double(gn[1]);
      q23.x = q23.x + a.c * double(gn[2]);
      q23.y = q23.y + a.c * double(gn[3]);
      qp[0] = q01; qp[1] = q23;
      check_state(a.health, a.health_host, q01.x, q01.y, q23.x, q23.y, e);
      s.Q[0][le][tid] = real(q01.x); s.Q[1][le][tid] = real(q01.y);
      s.Q[2][le][tid] = real(q23.x); s.Q[3][le][tid] = real(q23.y);
    }
  }
  if (a.resid) {
    double m[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) m[k] = active ? fabs(double(qd[k])) : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
      for (int k = 0; k < 4; ++k) m[k] = nanmax(m[k], __shfl_xor_sync(0xffffffffu, m[k], off));
    if ((flat & 31) == 0)
#pragma unroll
      for (int k = 0; k < 4; ++k) s.red[flat >> 5][k] = m[k];
  }
  __syncthreads();
  if (a.resid && flat < 4) {
    double mx = 0.0;
    for (int w = 0; w < NW; ++w) mx = nanmax(mx, s.red[w][flat]);
    a.resid[size_t(blockIdx.x) * 4 + flat] = mx;
  }
  if (active && a.update) {
    for (int t = tid; t < FT; t += NP) {
      const int sd_ = t / P, kk = t % P;
      const real* lbv = (sd_ == 0 || sd_ == 3) ? lb0 : lb1;
      real tr[4];
      trace4<P, EPB, real>(s.Q, le, sd_, kk, lbv, tr);
      st4(a.T_out + ((size_t(e) * 4 + sd_) * P + kk) * 4, tr);
      if (IP && AFFINE && a.fuse && visc) {   // the face tiles are dead since the lift
#pragma unroll
        for (int k = 0; k < 4; ++k) s.face[k][le][t] = tr[k];
      }
    }
  }
  if (IP && AFFINE && a.fuse && a.update && visc && flat < 2 * P) {
    const int sdt = flat / P, l = flat % P;
    const real* lbv = sdt == 0 ? lb0 : lb1;
    const real* DT = lbw1 + P;   // transposed D: DT[l * P + i] = D(i, l)
    real d = real(0);
#pragma unroll
    for (int m = 0; m < P; ++m) d += lbv[m] * DT[l * P + m];
    s.dl[sdt][l] = d;
  }
  if constexpr (IP) {
    // Fused interior penalty: what the next stage's neighbours read of this element's new state --
    // its gradient traces (the local gradient, ComputeInteriorGradient, interpolated to the sides) and,
    // after the last stage of a step, its element-local indicator.  a.fuse, a.update, a.viscous and
    // a.last are uniform over the launch.
    if (a.fuse && a.update) {
      __syncthreads();   // every node's new state is in s.Q (and, affine, its traces in s.face[0..3])
      if (visc && AFFINE) {
        // Affine element: the traces of the gradient straight from the new state.  Along the side, the
        // derivative of the side's Q traces (D applied to them); across it, each normal line of nodes
        // contracted with lb^T D.  The same as the nodal gradient interpolated to the side, without
        // forming the gradient at every node.
        if (active) {
          const real* DT = lbw1 + P;   // transposed D
          for (int t = tid; t < FT; t += NP) {
            const int sd_ = t / P, kk = t % P;
            const real* dlv = s.dl[(sd_ == 0 || sd_ == 3) ? 0 : 1];
            real dt_[4] = {real(0), real(0), real(0), real(0)}, dn[4] = {real(0), real(0), real(0), real(0)};
#pragma unroll
            for (int l = 0; l < P; ++l) {
              const real dk = DT[l * P + kk];
#pragma unroll
              for (int k = 0; k < 4; ++k) dt_[k] += dk * s.face[k][le][sd_ * P + l];
            }
#pragma unroll
            for (int m = 0; m < P; ++m) {
              const int l = trace_step<real>(P, m, kk);
              const int node = face_node(P, sd_, l, kk);
              const real w = dlv[l];
#pragma unroll
              for (int k = 0; k < 4; ++k) dn[k] += w * s.Q[k][le][node];
            }
            // bottom / top: along the side is xi; right / left: along the side is eta
            const bool alongXi = sd_ == 0 || sd_ == 2;
            const real Ja00 = geoE[0], Ja01 = geoE[1], Ja10 = geoE[2], Ja11 = geoE[3], iJ = geoE[4];
            real tx[4], ty[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const real dxi = alongXi ? dt_[k] : dn[k], deta = alongXi ? dn[k] : dt_[k];
              tx[k] = (dxi * Ja00 + deta * Ja01) * iJ;
              ty[k] = (dxi * Ja10 + deta * Ja11) * iJ;
            }
            real* gp = a.GT_out + ((size_t(e) * 4 + sd_) * P + kk) * 8;
            st4(gp, tx);
            st4(gp + 4, ty);
          }
        }
      } else if (visc) {
        element_gradient<P, EPB, real, AFFINE, IP>(a, s, ph, le, tid, e, active, geoE);
        __syncthreads();
        if (active) {
          for (int t = tid; t < FT; t += NP) {
            const int sd_ = t / P, kk = t % P;
            const real* lbv = (sd_ == 0 || sd_ == 3) ? lb0 : lb1;
            real* gp = a.GT_out + ((size_t(e) * 4 + sd_) * P + kk) * 8;
            real tx[4], ty[4];
            trace4<P, EPB, real>(s.dQ[0], le, sd_, kk, lbv, tx);
            trace4<P, EPB, real>(s.dQ[1], le, sd_, kk, lbv, ty);
            st4(gp, tx);
            st4(gp + 4, ty);
          }
        }
      }
      if (AV && a.last && a.sensor.kind != SENSOR_JUMPS) {
        const int n_active = a.n_el - int(blockIdx.x) * EPB < EPB ? a.n_el - int(blockIdx.x) * EPB : EPB;
        // the gradient, contravariant-flux and face tiles (contiguous) are dead here: where they are
        // large enough they hold the indicator's scratch, which keeps the kernel's static shared memory
        // within 48 KB (FP64 at high and low orders); otherwise the indicator declares its own
        constexpr size_t dead = sizeof(s.dQ) + sizeof(s.Fc) + sizeof(s.Gc) + sizeof(s.face) + sizeof(s.gfd);
        constexpr bool lend = dead >= sensor_ext_bytes<P, EPB, real>();
        __syncthreads();   // the gradient traces above have read s.dQ (affine: s.face)
        const SensorOut so = element_sensor<P, EPB, real, lend>(a.sensor, ph, s.Q, n_active, s.mat + 2 * NP + 7 * P,
                                                                le, tid, active, nullptr, &s.dQ[0][0][0][0]);
        if (active && tid == 0) a.mu_next[e] = a.av_el[2 * size_t(e)] * so.g;
      }
    }
  }
}

}  // namespace hg
