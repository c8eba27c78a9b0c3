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
//            eta, higher indices folded into 3, floored at 1e-10); G = the sigmoid output y mapped
//            to max(0, (y - c) / (1 - c)), c = LEARNED_CUT (an exact zero below 5 % of the maximum
//            viscosity, as the modal ramp has below s0 - kappa: elements without viscosity skip the
//            dissipation's gradient work), or the modal G when a feature lies outside the box seen in
//            training (out-of-distribution fallback).
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

// Scratch row of one element (reals): the 16 features, the first hidden layer (as floats), the two
// modal-decay indicators and the learned G, 16 out-of-box flags, the per-index energy sums of rho and p
// along xi and eta (4P), the modal energies of rho and p (2 P^2); rows are a multiple of 4 reals long so
// that the features and the hidden layer are read with 16-byte loads.
constexpr int SR_FT = 0, SR_H = SR_FT + MLP_IN, SR_PN = SR_H + MLP_H, SR_OOD = SR_PN + 4, SR_SUM = SR_OOD + MLP_IN;
__host__ __device__ constexpr int sensor_uh(int P) { return SR_SUM + 4 * P; }
__host__ __device__ constexpr int sensor_scratch(int P) { return (sensor_uh(P) + 2 * P * P + 3) / 4 * 4; }

__device__ __forceinline__ double sensor_ramp(double s, double s0, double k) {
  if (s < s0 - k) return 0.0;
  if (s < s0 + k) return 0.5 * sin(0.5 * 3.141592653589793238462643 * (s - s0) / k) + 0.5;
  return 1.0;
}

__device__ __forceinline__ float mlp_sigmoid(float z) { return 1.0f / (1.0f + expf(-z)); }
constexpr float LEARNED_CUT = 0.05f;
__device__ __forceinline__ float learned_g(float y) { return y > LEARNED_CUT ? (y - LEARNED_CUT) / (1.0f - LEARNED_CUT) : 0.0f; }

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
// shared memory by asynchronous copies issued on entry, so that they arrive during the modal
// transform; each warp evaluates one element at a time with one lane per hidden unit: the inputs and
// the first hidden layer are broadcast from the element's scratch row as 16-byte loads, the 32-input
// sums of the second layer run as four interleaved partial sums, and the output unit is a warp
// shuffle tree.  The out-of-box test runs per feature in the thread that forms it.
// Shared memory the indicator needs when the caller lends it (EXT): EPB scratch rows, then the weights.
template <int P, int EPB, typename real>
__host__ __device__ constexpr size_t sensor_ext_bytes() {
  return 16 + size_t(EPB) * sensor_scratch(P) * sizeof(real) + size_t(MLP_PARAMS) * sizeof(float);
}

// The network's weights into shared memory (16-byte aligned) as asynchronous copies: 16-byte chunks,
// the odd last float as a 4-byte copy.  Each thread waits for its own with sensor_weights_wait; a
// barrier after that makes all of them visible.
__device__ __forceinline__ void sensor_weights_async(float* s_w, const float* g, int t, int nt) {
  constexpr int C16 = MLP_PARAMS / 4;
  const unsigned base = static_cast<unsigned>(__cvta_generic_to_shared(s_w));
  for (int c = t; c < C16; c += nt)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(base + 16u * unsigned(c)), "l"(g + 4 * c)
                 : "memory");
  if (t == 0)
    for (int d = 4 * C16; d < MLP_PARAMS; ++d)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(base + 4u * unsigned(d)), "l"(g + d) : "memory");
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void sensor_weights_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// 16 consecutive reals of a 16-byte aligned shared row as floats
__device__ __forceinline__ void load16(const float* r, float* f) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float4 v = reinterpret_cast<const float4*>(r)[k];
    f[4 * k] = v.x; f[4 * k + 1] = v.y; f[4 * k + 2] = v.z; f[4 * k + 3] = v.w;
  }
}
__device__ __forceinline__ void load16(const double* r, float* f) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const double2 v = reinterpret_cast<const double2*>(r)[k];
    f[2 * k] = float(v.x); f[2 * k + 1] = float(v.y);
  }
}

template <int P, int EPB, typename real, bool EXT = false>
__device__ __forceinline__ SensorOut element_sensor(const SensorArgs& sa, const Phys<real>& ph,
                                                    const real (*Q)[EPB][P * P], int n_active,
                                                    const real* Vinv, int le, int tid, bool active,
                                                    float* feat_out, real* ext = nullptr) {
  constexpr int NP = P * P, N = P - 1, SS = sensor_scratch(P), UH = sensor_uh(P);
  // scratch rows of the CTA's elements, then the weights: declared here, or lent by the caller (EXT:
  // shared memory the caller no longer needs, sensor_ext_bytes long), so that every access is a
  // shared-memory one
  real* scr_all;
  float* s_w;   // W1^T[16][32] b1 W2^T[32][32] b2 W3 b3
  if constexpr (EXT) {
    scr_all = reinterpret_cast<real*>((reinterpret_cast<uintptr_t>(ext) + 15) & ~uintptr_t(15));
    s_w = reinterpret_cast<float*>(scr_all + EPB * SS);
  } else {
    __shared__ __align__(16) real s_scr[EPB * SS];
    __shared__ __align__(16) float s_w_own[MLP_PARAMS];
    scr_all = s_scr;
    s_w = s_w_own;
  }
  const bool learned = sa.kind == SENSOR_LEARNED;
  // the weights travel while the modal transform runs
  if (learned) sensor_weights_async(s_w, sa.mlp, threadIdx.x, blockDim.x);
  real* scr = scr_all + (le < EPB ? le : 0) * SS;
  real* uh = scr + UH;            // [2][NP] modal coefficients, then energies, of rho, p (k_eta * P + k_xi)
  real* sum = scr + SR_SUM;       // [2 variables][2 directions][P] energies per modal index
  real* pn = scr + SR_PN;         // [2] modal-decay indicators of rho and p, learned G, constant-state flag
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
  // energies per modal index: t = (v * 2 + dir) * P + k sums over the other index
  if (active)
    for (int t = tid; t < 4 * P; t += NP) {
      const int v = t / (2 * P), dir = (t / P) & 1, k = t % P;
      const real* c2 = uh + v * NP;
      real a = real(0);
#pragma unroll
      for (int j = 0; j < P; ++j) a += c2[dir == 0 ? j * P + k : k * P + j];
      sum[t] = a;
    }
  __syncthreads();
  // features q < 16 (with their out-of-box flags) and the two modal-decay indicators (q = 16, 17)
  if (active)
    for (int q = tid; q < MLP_IN + 2; q += NP) {
      const int v = q < MLP_IN ? q >> 3 : q - MLP_IN;
      const real* sv = sum + 2 * v * P;   // along xi: sv[m]; along eta: sv[P + n]
      real E = real(0);
#pragma unroll
      for (int m = 0; m < P; ++m) E += sv[m];
      if (q < MLP_IN) {
        const int dir = (q >> 2) & 1, k = q & 3;
        real part = real(0);
        if (k < 3) {
          if (k < P) part = sv[dir * P + k];
        } else {
          for (int m = 3; m < P; ++m) part += sv[dir * P + m];
        }
        // x / x is 1 exactly (also where the build's FP32 division is the approximate one)
        const real frac = E > real(0) ? (part == E ? real(1) : part / E) : real(0);
        const real f = log10_r(fmax_r(frac, real(SENSOR_FLOOR)));
        scr[SR_FT + q] = f;
        if (feat_out) feat_out[q] = float(f);
        scr[SR_OOD + q] = (sa.lo && (float(f) < __ldg(sa.lo + q) || float(f) > __ldg(sa.hi + q))) ? real(1) : real(0);
      } else {
        // the modes whose higher index is N: row N along eta plus column N below it
        const real* c2 = uh + v * NP;
        real part = real(0);
#pragma unroll
        for (int m = 0; m < P; ++m) part += c2[N * P + m];
#pragma unroll
        for (int n = 0; n < N; ++n) part += c2[n * P + N];
        pn[v] = (E > real(0) && part > real(0)) ? log10_r(part / E) : real(-1e30);
      }
    }
  __syncthreads();
  if (active && tid == 0) {
    const double smax = double(pn[0] > pn[1] ? pn[0] : pn[1]);
    out.g_modal = sensor_ramp(smax, sa.s0, sa.kappa);
    real ood = real(0);
#pragma unroll
    for (int q = 0; q < MLP_IN; ++q) ood += scr[SR_OOD + q];
    out.ood = ood > real(0);
    // constant-state element: every energy in the mean mode (fractions 1 and the floor exactly)
    bool flat = true;
#pragma unroll
    for (int q = 0; q < MLP_IN; ++q)
      flat = flat && scr[SR_FT + q] == ((q & 3) == 0 ? real(0) : log10_r(real(SENSOR_FLOOR)));
    pn[3] = flat ? real(1) : real(0);
  }
  if (learned) {
    static_assert(MLP_H == 32, "one lane per hidden unit");
    sensor_weights_wait();
    __syncthreads();
    // one warp per element, one lane per hidden unit; inputs and the first hidden layer are read back
    // as broadcast 16-byte loads, the output unit is a shuffle tree.  Constant-state elements all have
    // the same features: only the first of them in the CTA (rep) is evaluated, the others take its G
    // (the same inputs through the same code: the same bits).
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    int rep = -1;
    for (int el = 0; el < n_active && rep < 0; ++el)
      if (scr_all[el * SS + SR_PN + 3] != real(0)) rep = el;
    for (int el = threadIdx.x >> 5; el < n_active; el += nw) {
      real* r = scr_all + el * SS;
      if (r[SR_PN + 3] != real(0) && el != rep) continue;
      float f[MLP_IN];
      load16(r + SR_FT, f);
      float z = s_w[MLP_B1 + lane];
#pragma unroll
      for (int q = 0; q < MLP_IN; ++q) z += s_w[MLP_W1 + q * MLP_H + lane] * f[q];
      float* h1 = reinterpret_cast<float*>(r + SR_H);
      h1[lane] = tanhf(z);
      __syncwarp();
      float zp[4] = {s_w[MLP_B2 + lane], 0.0f, 0.0f, 0.0f};
#pragma unroll 2
      for (int q4 = 0; q4 < MLP_H / 4; ++q4) {
        const float4 h = reinterpret_cast<const float4*>(h1)[q4];
        zp[0] += s_w[MLP_W2 + (4 * q4 + 0) * MLP_H + lane] * h.x;
        zp[1] += s_w[MLP_W2 + (4 * q4 + 1) * MLP_H + lane] * h.y;
        zp[2] += s_w[MLP_W2 + (4 * q4 + 2) * MLP_H + lane] * h.z;
        zp[3] += s_w[MLP_W2 + (4 * q4 + 3) * MLP_H + lane] * h.w;
      }
      const float h = tanhf((zp[0] + zp[1]) + (zp[2] + zp[3]));
      float y = s_w[MLP_W3 + lane] * h;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) y += __shfl_xor_sync(0xffffffffu, y, off);
      if (lane == 0) r[SR_PN + 2] = real(learned_g(mlp_sigmoid(y + s_w[MLP_B3])));
    }
    __syncthreads();
    if (active && tid == 0) out.g_learned = double(pn[3] != real(0) ? scr_all[rep * SS + SR_PN + 2] : pn[2]);
  }
  out.g = learned ? (out.ood ? out.g_modal : out.g_learned) : out.g_modal;
  return out;
}

}  // namespace hg
