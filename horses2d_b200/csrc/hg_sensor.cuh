// hg_sensor.cuh -- element shock sensors that set the artificial viscosity (device code).
//
// Three indicators feed the same viscosity law mu_e = Ceps sqrt(Volume)/(N+1) G (the law of
// JumpsBasedElementViscosity, Approximation/DGArtificialDissipation.f90:322-336):
//   jumps    the reference's interface-jumps indicator (hg_ns.cuh element_viscosity);
//   modal    modal decay (Persson-Peraire): s = max over rho, p of log10(E_N / E), E the energy of
//            the element's orthonormal-Legendre modal coefficients and E_N that of the modes whose
//            higher index is N; G = ramp(s; s0, kappa), the same sine ramp as the jumps indicator;
//   learned  an MLP 16 -> 32 -> 32 -> 1 (tanh hidden layers, sigmoid output) on 16 modal features
//            (for rho and p: log10 of the energy fraction in modal index k = 0..3 along xi and along
//            eta, higher indices folded into 3, floored at 1e-10); G = sigmoid output, or the modal G
//            when a feature lies outside the box seen in training (out-of-distribution fallback).
// No reference counterpart exists for modal and learned.
#pragma once
#include "hg_physics.cuh"

namespace hg {

enum { SENSOR_JUMPS = 0, SENSOR_MODAL = 1, SENSOR_LEARNED = 2 };
constexpr int MLP_IN = 16, MLP_H = 32;
constexpr int MLP_W1 = 0, MLP_B1 = MLP_W1 + MLP_H * MLP_IN, MLP_W2 = MLP_B1 + MLP_H, MLP_B2 = MLP_W2 + MLP_H * MLP_H,
              MLP_W3 = MLP_B2 + MLP_H, MLP_B3 = MLP_W3 + MLP_H, MLP_PARAMS = MLP_B3 + 1;

struct SensorArgs {
  int kind;            // SENSOR_*
  double s0, kappa;    // modal ramp centre and half width
  const float* mlp;    // [MLP_PARAMS] W1^T[16][32] b1 W2^T[32][32] b2 W3[32] b3 (hidden unit fastest)
  const float* lo;     // [16] feature box of the training set (with margin)
  const float* hi;     // [16]
};

__host__ __device__ constexpr int sensor_scratch(int P) { return 2 * P * P + 24 + MLP_IN + 2 * MLP_H + 4; }

__device__ __forceinline__ double sensor_ramp(double s, double s0, double k) {
  if (s < s0 - k) return 0.0;
  if (s < s0 + k) return 0.5 * sin(0.5 * 3.141592653589793238462643 * (s - s0) / k) + 0.5;
  return 1.0;
}

__device__ __forceinline__ float mlp_sigmoid(float z) { return 1.0f / (1.0f + expf(-z)); }

// smallest energy fraction a feature resolves (log10 floor -10: FP32 round-off, ~1e-14, stays below)
constexpr double SENSOR_FLOOR = 1e-10;
template <typename real> __device__ __forceinline__ real log10_r(real x);
template <> __device__ __forceinline__ double log10_r(double x) { return log10(x); }
template <> __device__ __forceinline__ float log10_r(float x) { return log10f(x); }
template <typename real> __device__ __forceinline__ real fmax_r(real a, real b) { return a > b ? a : b; }

struct SensorOut {
  double g_modal, g_learned, g;
  int ood;
};

// Modal indicator and (if asked) the learned one for element `le` of the CTA.  Q: the element tiles
// [4][EPB][NP] in shared memory; n_active: elements of this CTA that exist.  All threads of the CTA call it (it holds barriers);
// results are valid in thread tid == 0 of each element.
//
// Network inference: the weights (stored with the hidden unit fastest) are copied once per CTA into
// shared memory, and each warp evaluates one element at a time with one lane per hidden unit: the
// inputs are broadcast from the element's scratch row, the 32-input sums of the second layer run as
// four interleaved partial sums, and the output unit is a warp shuffle tree.
// Shared memory the indicator needs when the caller lends it (EXT): EPB scratch rows, then the weights.
template <int P, int EPB, typename real>
__host__ __device__ constexpr size_t sensor_ext_bytes() {
  return size_t(EPB) * sensor_scratch(P) * sizeof(real) + size_t(MLP_PARAMS) * sizeof(float);
}

template <int P, int EPB, typename real, bool EXT = false>
__device__ __forceinline__ SensorOut element_sensor(const SensorArgs& sa, const Phys<real>& ph,
                                                    const real (*Q)[EPB][P * P], int n_active,
                                                    const real* Vinv, int le, int tid, bool active,
                                                    float* feat_out, real* ext = nullptr) {
  constexpr int NP = P * P, N = P - 1, SS = sensor_scratch(P);
  // scratch rows of the CTA's elements: declared here, or lent by the caller (EXT: shared memory the
  // caller no longer needs, sensor_ext_bytes long), so that every access is a shared-memory one
  real* scr_all;
  if constexpr (EXT) {
    scr_all = ext;
  } else {
    __shared__ real s_scr[EPB * SS];
    scr_all = s_scr;
  }
  real* scr = scr_all + (le < EPB ? le : 0) * SS;
  real* uh = scr;                 // [2][NP] modal coefficients of rho, p (k_eta * P + k_xi)
  real* en = scr + 2 * NP;        // [2][12]: Ex[4], Ey[4], E, EN, -, -
  real* ft = en + 24;             // [16] features
  real* h1 = ft + MLP_IN;         // [32]
  real* h2 = h1 + MLP_H;          // [32]
  real* pn = h2 + MLP_H;          // [2] modal-decay indicators of rho and p, [2] learned G
  SensorOut out{0.0, 0.0, 0.0, 0};
  // nodal pressure into uh[NP..) as a staging area, then the transform in place per variable
  real pnode = real(0);
  if (active) {
    const real r = Q[0][le][tid], ru = Q[1][le][tid], rv = Q[2][le][tid], rE = Q[3][le][tid];
    pnode = ph.gm1 * (rE - real(0.5) * (ru * ru + rv * rv) / r);
  }
  __syncthreads();
  real c0 = real(0), c1 = real(0);
  if (active) {
    const int m = tid % P, n = tid / P;
    // u_hat(m, n) = sum_j Vinv(n, j) sum_i Vinv(m, i) u(i, j)
#pragma unroll
    for (int j = 0; j < P; ++j) {
      real a0 = real(0);
#pragma unroll
      for (int i = 0; i < P; ++i) a0 += Vinv[m * P + i] * Q[0][le][j * P + i];
      c0 += Vinv[n * P + j] * a0;
    }
  }
  // pressure needs every node's value: stage it in the second half of uh
  if (active) uh[NP + tid] = pnode;
  __syncthreads();
  if (active) {
    const int m = tid % P, n = tid / P;
#pragma unroll
    for (int j = 0; j < P; ++j) {
      real a1 = real(0);
#pragma unroll
      for (int i = 0; i < P; ++i) a1 += Vinv[m * P + i] * uh[NP + j * P + i];
      c1 += Vinv[n * P + j] * a1;
    }
  }
  __syncthreads();
  if (active) { uh[tid] = c0 * c0; uh[NP + tid] = c1 * c1; }   // modal energies
  __syncthreads();
  // features q < 16 and the two modal-decay indicators (q = 16, 17), one per thread
  if (active)
    for (int q = tid; q < MLP_IN + 2; q += NP) {
      const int v = q < MLP_IN ? q >> 3 : q - MLP_IN;
      const real* c2 = uh + v * NP;
      real E = real(0), part = real(0);
      if (q < MLP_IN) {
        const int dir = (q >> 2) & 1, k = q & 3;
        for (int n = 0; n < P; ++n)
          for (int m = 0; m < P; ++m) {
            const real x = c2[n * P + m];
            const int idx = dir == 0 ? m : n;
            E += x;
            if ((idx < 3 ? idx : 3) == k) part += x;
          }
        ft[q] = log10_r(fmax_r(E > real(0) ? part / E : real(0), real(SENSOR_FLOOR)));
      } else {
        for (int n = 0; n < P; ++n)
          for (int m = 0; m < P; ++m) {
            const real x = c2[n * P + m];
            E += x;
            if (m == N || n == N) part += x;
          }
        pn[v] = (E > real(0) && part > real(0)) ? log10_r(part / E) : real(-1e30);
      }
    }
  __syncthreads();
  if (active && tid == 0) {
    const double smax = double(pn[0] > pn[1] ? pn[0] : pn[1]);
    out.g_modal = sensor_ramp(smax, sa.s0, sa.kappa);
    int ood = 0;
    for (int q = 0; q < MLP_IN; ++q) {
      if (feat_out) feat_out[q] = float(ft[q]);
      if (sa.lo && (float(ft[q]) < sa.lo[q] || float(ft[q]) > sa.hi[q])) ood = 1;
    }
    out.ood = ood;
  }
  if (sa.kind == SENSOR_LEARNED) {
    static_assert(MLP_H == 32, "one lane per hidden unit");
    float* s_w;   // W1^T[16][32] b1 W2^T[32][32] b2 W3 b3
    if constexpr (EXT) {
      s_w = reinterpret_cast<float*>(ext + EPB * SS);
    } else {
      __shared__ float s_w_own[MLP_PARAMS];
      s_w = s_w_own;
    }
    for (int d = threadIdx.x; d < MLP_PARAMS; d += blockDim.x) s_w[d] = __ldg(sa.mlp + d);
    __syncthreads();
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int el = threadIdx.x >> 5; el < n_active; el += nw) {
      real* r = scr_all + el * SS;
      const real* f = r + 2 * NP + 24;
      real* g1 = r + 2 * NP + 24 + MLP_IN;
      float z = s_w[MLP_B1 + lane];
#pragma unroll
      for (int q = 0; q < MLP_IN; ++q) z += s_w[MLP_W1 + q * MLP_H + lane] * float(f[q]);
      g1[lane] = real(tanhf(z));
      __syncwarp();
      float zp[4] = {s_w[MLP_B2 + lane], 0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int q = 0; q < MLP_H; ++q) zp[q & 3] += s_w[MLP_W2 + q * MLP_H + lane] * float(g1[q]);
      const float h = tanhf((zp[0] + zp[1]) + (zp[2] + zp[3]));
      float y = s_w[MLP_W3 + lane] * h;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) y += __shfl_xor_sync(0xffffffffu, y, off);
      if (lane == 0) r[2 * NP + 24 + MLP_IN + 2 * MLP_H + 2] = real(mlp_sigmoid(y + s_w[MLP_B3]));
      __syncwarp();
    }
    __syncthreads();
    if (active && tid == 0) out.g_learned = double(pn[2]);
  }
  out.g = sa.kind == SENSOR_LEARNED ? (out.ood ? out.g_modal : out.g_learned) : out.g_modal;
  return out;
}

}  // namespace hg
