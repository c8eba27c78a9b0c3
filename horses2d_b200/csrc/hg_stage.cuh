// hg_stage.cuh -- the fused DGSEM stage kernel (Euler) for sm_100a.
//
// One launch = one Runge-Kutta stage (or one bare time derivative) over all
// elements.  Per element (one thread per node, EPB elements per CTA):
//   1. load Q (reference layout, 32 B per node: coalesced) and the metrics;
//   2. Euler flux -> contravariant fluxes into shared memory
//        (Scalar_StdVolumeGreen, Approximation/DGWeakIntegrals.f90:111-181);
//   3. 4(N+1) face-node tasks: own trace (from shared memory) and the neighbour's
//      trace of the previous stage (global, written by that element's previous
//      launch), Riemann solver / boundary state, x dS
//        (ComputeRiemannSolver_*, DGSpatialDiscretizationMethods.f90:545-1511;
//         projections types 1-2, Mesh/QuadElement_EdgeProcedures.incf:749-1206);
//   4. volume contraction with hatD, surface lift with lbw (Scalar_StdFace,
//      DGWeakIntegrals.f90:183-266), division by J (computeQDot :226-233);
//   5. low-storage RK update G = a G + b QDot, Q += c G
//        (DGTimeIntegrator.f90:282-365), in place;
//   6. traces of the new Q on the 4 sides for the next launch (ping-pong buffer)
//        (interpolateSolutionToBoundaries, :1520-1574).
// The Riemann flux of an interior face is evaluated by both of its elements with
// identical arguments (LEFT trace, RIGHT trace, LEFT's normal), so both see the
// same value and the face needs no separate launch or flux buffer.
//
// CTAs are one-dimensional, padded to whole warps (threads past EPB*(N+1)^2 only
// take part in barriers and reductions).  Shared tiles are variable-major
// ([var][element][node]) so that a warp reading one row or column of a tile
// touches consecutive words.
#pragma once
#include "hg_physics.cuh"
#include "hg_bc.cuh"

namespace hg {

// side kinds; SIDE_FLUX: a p-nonconforming or subdivided edge, whose lifted flux (projected to this
// element's side nodes, dS and sign applied) the mortar kernel has written to the NF buffer
enum { SIDE_LEFT = 0, SIDE_RIGHT = 1, SIDE_STATE = 2, SIDE_WALL = 3, SIDE_FLUX = 4 };
constexpr int SIDE_REVERSED = 16;

template <typename real>
struct StageArgs {
  int n_el;
  const int4* side;        // [n_el*4] {neighbour trace slot, flags, zone, per-node state row or -1}
  const real* side_geo;    // [n_el*4][P][3] (or [n_el*4][3] affine)  nx, ny, dS in this element's side order
  const real* vol_geo;     // [n_el][P*P][5] (or [n_el][5] affine)  Ja00 Ja01 Ja10 Ja11 1/J
  const double* mats;      // hatD[P*P], lb0[P], lb1[P], lbw0[P], lbw1[P]
  const Zone* zones;
  const double* bq;        // per-node Dirichlet states [rows][P][4] (sides whose side.w >= 0)
  const real* FX;          // exact-solver face fluxes [n_el*4][P][4] of this stage (RIEMANN_EXACT faces)
  const real* NF;          // mortar fluxes [slots][P][4] of SIDE_FLUX sides (slot = side.x)
  double* Q;               // [n_el][P*P][4]
  real* G;                 // [n_el][P*P][4]
  const real* T_in;        // [n_el*4][P][4]
  real* T_out;
  double* QDot;            // optional output (time derivative only)
  double* resid;           // optional per-CTA max |QDot| per variable: [gridDim.x][4]
  int* health;             // device health word {bits, element} (check_state), may be null
  int* health_host;        // mapped host flag set beside it, may be null
  double a, b, c;          // G = a G + b QDot ; Q += c G
  int first;               // a == 0: do not read G
  int update;              // 1: RK update, 0: only QDot (and traces of the unchanged Q)
  int riemann;
  PhysConst pc;
};

// Elements per CTA: tiling variant 0 (default, large CTAs) and variant 1 (small CTAs: more CTAs in
// flight on small meshes); hg_autotune times both on the resident state and keeps the faster.
__host__ __device__ constexpr int epb_for(int P) {
  return P == 2 ? 32 : P == 3 ? 16 : P == 4 ? 16 : P == 5 ? 8 : P == 6 ? 8 : P == 7 ? 4 : P == 8 ? 4 : P <= 11 ? 3 : 2;
}
__host__ __device__ constexpr int epb_small_for(int P) {
  return P == 2 ? 8 : P == 3 ? 4 : P == 4 ? 4 : P == 5 ? 2 : P == 6 ? 2 : P == 7 ? 2 : 1;
}
__host__ __device__ constexpr int epb_stage(int P, int variant) { return variant ? epb_small_for(P) : epb_for(P); }
__host__ __device__ constexpr int block_of(int P, int EPB) { return ((P * P * EPB + 31) / 32) * 32; }
__host__ __device__ constexpr int block_for(int P) { return block_of(P, epb_for(P)); }

// Four consecutive values of a record that starts at a multiple of 4 values from a cudaMalloc'd base
// (16-byte aligned in float, 32-byte in double): one 128-bit access in float, two in double.
__device__ __forceinline__ void ld4(const float* p, float* o) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
__device__ __forceinline__ void ld4(const double* p, double* o) {
  const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void st4(float* p, const float* v) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double* p, const double* v) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

// One value from global into shared memory as an asynchronous copy (4 or 8 bytes); the issuing thread
// sees it after cp_async_wait_all.
__device__ __forceinline__ void cp_async_real(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
               "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_real(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
               "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// max that keeps NaN (a residual that is NaN must stay visible)
__device__ __forceinline__ double nanmax(double m, double v) { return (v > m || v != v) ? v : m; }

// Health of an updated node state.  The reference stops with "The simulation has crashed" when Q holds
// a NaN (DGTimeIntegrator.f90:224-233); here every RK update checks its node: bit 1 a non-finite value,
// bit 2 rho <= 0, bit 4 p <= 0 (tested as rho (rho E) - |rho u|^2 / 2 = rho p / (gamma - 1) <= 0, no
// division).  health = {bits, an offending element (the first to arrive)}; the mapped host flag tells
// the host without a synchronisation that the word is no longer clean.
enum { HEALTH_NONFINITE = 1, HEALTH_DENSITY = 2, HEALTH_PRESSURE = 4 };
__device__ __forceinline__ void check_state(int* health, int* health_host, double r, double ru, double rv,
                                            double rE, int e) {
  const bool finite = fabs(r) + fabs(ru) + fabs(rv) + fabs(rE) < 1.0e300;
  const double k = r * rE - 0.5 * (ru * ru + rv * rv);
  if (finite && r > 0.0 && k > 0.0) return;
  const int bits = !finite ? HEALTH_NONFINITE : (r > 0.0 ? HEALTH_PRESSURE : HEALTH_DENSITY);
  if (health) {
    atomicOr(health, bits);
    atomicCAS(health + 1, -1, e);
  }
  if (health_host) *reinterpret_cast<volatile int*>(health_host) = 1;
}

// AFFINE: metrics constant per element (vol_geo [n_el][5]) and normals/dS constant
// per side (side_geo [n_el*4][3]), as for parallelogram elements with straight edges.
// LGL: Gauss-Lobatto nodes, whose boundary interpolants are unit vectors (lb = e_0 / e_N): traces are
// node values and the lift touches only the boundary rows -- the same arithmetic as the dense form
// with its exact zeros left out.
__host__ __device__ constexpr int face_node(int P, int side, int l, int kk) {
  return (side == 0 || side == 2) ? (l * P + kk) : (kk * P + l);
}
// Order of the P terms of a trace at face node kk: step m takes line node l = (m + kk) mod P.  The face
// nodes of a side sit in consecutive lanes; without the rotation the lanes of a right or left side (a
// column of the tile) would read one column at a time, P words apart, into the same banks.  Every Q
// trace of a state (stage, gradient and trace kernels) sums in this order, so an element's own trace and
// the copy its neighbour reads stay equal bit for bit.
__host__ __device__ constexpr int trace_l(int P, int m, int kk) { return (m + kk) % P; }
// The rotation is used in double, where a column side's lanes collide 4 ways; in float they collide 2
// ways and the rotated (runtime) addressing costs more registers than the conflicts cost time.
template <typename real>
__host__ __device__ constexpr int trace_step(int P, int m, int kk) { return sizeof(real) == 8 ? trace_l(P, m, kk) : m; }

template <int P, int EPB, typename real, bool AFFINE, bool LGL>
__global__ void __launch_bounds__(block_of(P, EPB)) stage_kernel(StageArgs<real> a) {
  constexpr int NP = P * P;
  constexpr int FT = 4 * P;
  constexpr int NW = block_of(P, EPB) / 32;
  __shared__ real s_mat[NP + 4 * P];
  __shared__ real s_Fc[4][EPB][NP];
  __shared__ real s_Gc[4][EPB][NP];
  __shared__ real s_Q[4][EPB][NP];
  __shared__ real s_F[4][EPB][FT];
  __shared__ double s_red[NW][4];

  const int flat = threadIdx.x;
  const int le = flat / NP;               // element in block
  const int tid = flat - le * NP;         // node in element
  // hatD held transposed (column l contiguous): conflict-free reads of hatD(i, l) across a warp's nodes
  for (int k = flat; k < NP + 4 * P; k += blockDim.x) s_mat[k] = real(a.mats[k < NP ? (k % P) * P + k / P : k]);
  const int e = blockIdx.x * EPB + le;
  const bool active = le < EPB && e < a.n_el;
  Phys<real> ph;
  ph.load(a.pc);
  const int i = tid % P, j = tid / P;

  const size_t off = (size_t(e) * NP + tid) * 4;
  real geo[5];
  if (active) {
    const double2* qp = reinterpret_cast<const double2*>(a.Q + off);
    const double2 q01 = qp[0], q23 = qp[1];
    const real q[4] = {real(q01.x), real(q01.y), real(q23.x), real(q23.y)};
    const real* gp = AFFINE ? a.vol_geo + size_t(e) * 5 : a.vol_geo + (size_t(e) * NP + tid) * 5;
#pragma unroll
    for (int k = 0; k < 5; ++k) geo[k] = real(gp[k]);
    real f[4], g[4];
    inviscid_flux(ph, q, f, g);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      s_Fc[k][le][tid] = f[k] * geo[0] + g[k] * geo[2];   // F Ja(1,IX) + G Ja(2,IX)
      s_Gc[k][le][tid] = f[k] * geo[1] + g[k] * geo[3];   // F Ja(1,IY) + G Ja(2,IY)
      s_Q[k][le][tid] = q[k];
    }
  }
  __syncthreads();
  const real* hatDT = s_mat;   // transposed: hatDT[l * P + i] = hatD(i, l)
  const real* lb0 = s_mat + NP;
  const real* lb1 = lb0 + P;
  const real* lbw0 = lb1 + P;
  const real* lbw1 = lbw0 + P;

  // face-node tasks: Riemann fluxes of the 4 sides (element-local order)
  if (active) {
    for (int t = tid; t < FT; t += NP) {
      const int s = t / P, kk = t % P;
      const int4 sd = a.side[size_t(e) * 4 + s];
      const int kind = sd.y & 15;
      if (kind == SIDE_FLUX) {
        real fp[4];
        ld4(a.NF + (size_t(sd.x) * P + kk) * 4, fp);
#pragma unroll
        for (int k = 0; k < 4; ++k) s_F[k][le][t] = fp[k];
        continue;
      }
      const real* lbv = (s == 0 || s == 3) ? lb0 : lb1;
      real qo[4] = {real(0), real(0), real(0), real(0)};
      if (LGL) {
        const int node = face_node(P, s, (s == 0 || s == 3) ? 0 : P - 1, kk);
#pragma unroll
        for (int k = 0; k < 4; ++k) qo[k] = s_Q[k][le][node];
      } else {
#pragma unroll
        for (int m = 0; m < P; ++m) {
          const int l = trace_step<real>(P, m, kk);
          const int node = face_node(P, s, l, kk);
#pragma unroll
          for (int k = 0; k < 4; ++k) qo[k] += s_Q[k][le][node] * lbv[l];
        }
      }
      const real* g3 = AFFINE ? a.side_geo + (size_t(e) * 4 + s) * 3 : a.side_geo + ((size_t(e) * 4 + s) * P + kk) * 3;
      const real nx = g3[0], ny = g3[1], dS = g3[2];
      real F[4];
      if (kind == SIDE_WALL) {
        euler_wall_flux(ph, qo, nx, ny, dS, F);
      } else {
        real qn[4];
        int solver = a.riemann;
        if (kind == SIDE_STATE) {
          const Zone& z = a.zones[sd.z];
          real us[4];
          bc_states(ph, z, qo, nx, ny, qn, us, sd.w >= 0 ? a.bq + (size_t(sd.w) * P + kk) * 4 : nullptr);
          if (z.riemann >= 0) solver = z.riemann;
        } else {
          const int kn = (sd.y & SIDE_REVERSED) ? (P - 1 - kk) : kk;
          ld4(a.T_in + (size_t(sd.x) * P + kn) * 4, qn);
          if (sd.z >= 0) { const int zr = a.zones[sd.z].riemann; if (zr >= 0) solver = zr; }
        }
        if (kind == SIDE_RIGHT) {
          face_riemann(solver, ph, qn, qo, nx, ny, a.FX, (size_t(e) * 4 + s) * P + kk, F);
#pragma unroll
          for (int k = 0; k < 4; ++k) F[k] = -(F[k] * dS);
        } else {
          face_riemann(solver, ph, qo, qn, nx, ny, a.FX, (size_t(e) * 4 + s) * P + kk, F);
#pragma unroll
          for (int k = 0; k < 4; ++k) F[k] = F[k] * dS;
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) s_F[k][le][t] = F[k];
    }
  }
  __syncthreads();

  real qd[4] = {real(0), real(0), real(0), real(0)};
  if (active) {
#pragma unroll
    for (int l = 0; l < P; ++l) {
      const real hi = hatDT[l * P + i], hj = hatDT[l * P + j];
#pragma unroll
      for (int k = 0; k < 4; ++k) qd[k] = qd[k] + hi * s_Fc[k][le][j * P + l] + hj * s_Gc[k][le][l * P + i];
    }
    // lift: bottom F(i) lbw0(j), right F(j) lbw1(i), top F(i) lbw1(j), left F(j) lbw0(i)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (LGL) {
        if (j == 0) qd[k] = qd[k] - s_F[k][le][0 * P + i] * lbw0[0];
        if (i == P - 1) qd[k] = qd[k] - s_F[k][le][1 * P + j] * lbw1[P - 1];
        if (j == P - 1) qd[k] = qd[k] - s_F[k][le][2 * P + i] * lbw1[P - 1];
        if (i == 0) qd[k] = qd[k] - s_F[k][le][3 * P + j] * lbw0[0];
      } else {
        qd[k] = qd[k] - s_F[k][le][0 * P + i] * lbw0[j];
        qd[k] = qd[k] - s_F[k][le][1 * P + j] * lbw1[i];
        qd[k] = qd[k] - s_F[k][le][2 * P + i] * lbw1[j];
        qd[k] = qd[k] - s_F[k][le][3 * P + j] * lbw0[i];
      }
      qd[k] = qd[k] * geo[4];
    }
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
      s_Q[0][le][tid] = real(q01.x); s_Q[1][le][tid] = real(q01.y);
      s_Q[2][le][tid] = real(q23.x); s_Q[3][le][tid] = real(q23.y);
    }
  }
  if (a.resid) {   // uniform over the grid: every thread of the CTA takes part
    double m[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) m[k] = active ? fabs(double(qd[k])) : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
      for (int k = 0; k < 4; ++k) m[k] = nanmax(m[k], __shfl_xor_sync(0xffffffffu, m[k], off));
    if ((flat & 31) == 0)
#pragma unroll
      for (int k = 0; k < 4; ++k) s_red[flat >> 5][k] = m[k];
  }
  __syncthreads();
  if (a.resid && flat < 4) {
    double mx = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) mx = nanmax(mx, s_red[w][flat]);
    a.resid[size_t(blockIdx.x) * 4 + flat] = mx;
  }
  // traces of the updated state for the next launch
  if (active && a.update) {
    for (int t = tid; t < FT; t += NP) {
      const int s = t / P, kk = t % P;
      const real* lbv = (s == 0 || s == 3) ? lb0 : lb1;
      real tr[4] = {real(0), real(0), real(0), real(0)};
      if (LGL) {
        const int node = face_node(P, s, (s == 0 || s == 3) ? 0 : P - 1, kk);
#pragma unroll
        for (int k = 0; k < 4; ++k) tr[k] = s_Q[k][le][node];
      } else {
#pragma unroll
        for (int m = 0; m < P; ++m) {
          const int l = trace_step<real>(P, m, kk);
          const int node = face_node(P, s, l, kk);
#pragma unroll
          for (int k = 0; k < 4; ++k) tr[k] += s_Q[k][le][node] * lbv[l];
        }
      }
      st4(a.T_out + ((size_t(e) * 4 + s) * P + kk) * 4, tr);
    }
  }
}

// Traces of the resident state (after hg_set_state).
template <int P, int EPB, typename real>
__global__ void __launch_bounds__(block_for(P)) trace_kernel(int n_el, const double* Q, const double* mats, real* T) {
  constexpr int NP = P * P;
  constexpr int FT = 4 * P;
  __shared__ real s_lb[2 * P];
  __shared__ real s_Q[4][EPB][NP];
  const int flat = threadIdx.x;
  const int le = flat / NP, tid = flat - le * NP;
  for (int k = flat; k < 2 * P; k += blockDim.x) s_lb[k] = real(mats[NP + k]);
  const int e = blockIdx.x * EPB + le;
  const bool active = le < EPB && e < n_el;
  if (active)
#pragma unroll
    for (int k = 0; k < 4; ++k) s_Q[k][le][tid] = real(Q[(size_t(e) * NP + tid) * 4 + k]);
  __syncthreads();
  if (!active) return;
  for (int t = tid; t < FT; t += NP) {
    const int s = t / P, kk = t % P;
    const real* lbv = (s == 0 || s == 3) ? s_lb : s_lb + P;
    real tr[4] = {real(0), real(0), real(0), real(0)};
    for (int m = 0; m < P; ++m) {
      const int l = trace_step<real>(P, m, kk);
      const int node = face_node(P, s, l, kk);
#pragma unroll
      for (int k = 0; k < 4; ++k) tr[k] += s_Q[k][le][node] * lbv[l];
    }
    real* tp = T + ((size_t(e) * 4 + s) * P + kk) * 4;
#pragma unroll
    for (int k = 0; k < 4; ++k) tp[k] = tr[k];
  }
}

// Max over the per-CTA residual partials: out[k] = max_b part[b*4+k] (NaN kept).
static __global__ void residual_reduce_kernel(int nblocks, const double* part, double* out) {
  __shared__ double s[4][256];
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < 4; ++k) m[k] = nanmax(m[k], part[size_t(b) * 4 + k]);
#pragma unroll
  for (int k = 0; k < 4; ++k) s[k][threadIdx.x] = m[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < 4; ++k) s[k][threadIdx.x] = nanmax(s[k][threadIdx.x], s[k][threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = s[threadIdx.x][0];
}

}  // namespace hg
