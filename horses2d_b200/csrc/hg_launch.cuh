// hg_launch.cuh -- definitions of the per-order launch templates declared in hg_ctx.h.
// Included only by the instantiation units hg_inst_*.cu.
#pragma once
#include "hg_ctx.h"

template <int P, typename real, int V>
void launch_stage_PV(hg_ctx* c, const StageArgs<real>& a) {
  constexpr int EPB = epb_stage(P, V);
  constexpr int BLK = block_of(P, EPB);
  const int grid = (a.n_el + EPB - 1) / EPB;
  static bool attr = false;
  if (!attr) {
    max_carveout(stage_kernel<P, EPB, real, true, false>);
    max_carveout(stage_kernel<P, EPB, real, false, false>);
    max_carveout(stage_kernel<P, EPB, real, true, true>);
    max_carveout(stage_kernel<P, EPB, real, false, true>);
    attr = true;
  }
  const bool lgl = c->node_type == HG_NODES_LGL;
  timed(c, HG_KERNEL_STAGE, [&] {
    if (c->affine) {
      if (lgl) stage_kernel<P, EPB, real, true, true><<<grid, BLK, 0, c->stream>>>(a);
      else stage_kernel<P, EPB, real, true, false><<<grid, BLK, 0, c->stream>>>(a);
    } else {
      if (lgl) stage_kernel<P, EPB, real, false, true><<<grid, BLK, 0, c->stream>>>(a);
      else stage_kernel<P, EPB, real, false, false><<<grid, BLK, 0, c->stream>>>(a);
    }
  });
  ++c->launches;
}

template <int P, typename real>
void launch_trace_P(hg_ctx* c) {
  constexpr int EPB = epb_for(P);
  const int grid = (c->n_el + EPB - 1) / EPB;
  timed(c, HG_KERNEL_TRACE, [&] {
    trace_kernel<P, EPB, real><<<grid, block_for(P), 0, c->stream>>>(c->n_el, c->d_Q, c->d_mats,
                                                                     static_cast<real*>(c->d_T[c->cur]));
  });
  ++c->launches;
}

template <int P, typename real, int V, bool AFFINE, bool IP, bool AV>
static void launch_ns_PAI(hg_ctx* c, const NSArgs<real>& a) {
  constexpr int EPB = epb_ns_of(P, V);
  constexpr int BLK = block_of(P, EPB);
  const int grid = (a.n_el + EPB - 1) / EPB;
  static bool attr = false;
  if (!attr) {
    max_carveout(ns_gradient_kernel<P, EPB, real, AFFINE, IP, AV>);
    max_carveout(ns_stage_kernel<P, EPB, real, AFFINE, IP, AV>);
    attr = true;
  }
  if (a.run_gradient) {
    timed(c, HG_KERNEL_GRADIENT,
          [&] { ns_gradient_kernel<P, EPB, real, AFFINE, IP, AV><<<grid, BLK, 0, c->stream>>>(a); });
    ++c->launches;
  }
  if (a.run_stage) {
    timed(c, HG_KERNEL_STAGE,
          [&] { ns_stage_kernel<P, EPB, real, AFFINE, IP, AV><<<grid, BLK, 0, c->stream>>>(a); });
    ++c->launches;
  }
}

template <int P, typename real, int V>
void launch_ns_PV(hg_ctx* c, const NSArgs<real>& a) {
  // artificial dissipation is a template switch so that the plain kernels keep their register budget
  if (c->av) {
    if (c->affine) {
      if (c->ip) launch_ns_PAI<P, real, V, true, true, true>(c, a); else launch_ns_PAI<P, real, V, true, false, true>(c, a);
    } else {
      if (c->ip) launch_ns_PAI<P, real, V, false, true, true>(c, a); else launch_ns_PAI<P, real, V, false, false, true>(c, a);
    }
  } else {
    if (c->affine) {
      if (c->ip) launch_ns_PAI<P, real, V, true, true, false>(c, a); else launch_ns_PAI<P, real, V, true, false, false>(c, a);
    } else {
      if (c->ip) launch_ns_PAI<P, real, V, false, true, false>(c, a); else launch_ns_PAI<P, real, V, false, false, false>(c, a);
    }
  }
}

// Sensor indicators of the resident state, per element: features [n_el][16] (optional) and
// {modal G, learned G, out-of-distribution flag, G used} [n_el][4] (optional).  The learned G is
// evaluated whenever weights are set.
template <int P, int EPB, typename real>
__global__ void __launch_bounds__(block_ns(P)) sensor_eval_kernel(int n_el, const double* Q, const double* mats,
                                                                  SensorArgs sa, PhysConst pc, float* feat,
                                                                  double* out) {
  constexpr int NP = P * P;
  __shared__ real sQ[4][EPB][NP];
  __shared__ real sV[NP];
  const int flat = threadIdx.x, le = flat / NP, tid = flat - le * NP;
  const int e = blockIdx.x * EPB + le;
  const bool active = le < EPB && e < n_el;
  for (int k = flat; k < NP; k += blockDim.x) sV[k] = real(mats[2 * NP + 7 * P + k]);
  if (active) {
    const double* q = Q + (size_t(e) * NP + tid) * 4;
#pragma unroll
    for (int k = 0; k < 4; ++k) sQ[k][le][tid] = real(q[k]);
  }
  __syncthreads();
  Phys<real> ph;
  ph.load(pc);
  SensorArgs s2 = sa;
  if (sa.mlp) s2.kind = SENSOR_LEARNED;
  const int n_active = n_el - int(blockIdx.x) * EPB < EPB ? n_el - int(blockIdx.x) * EPB : EPB;
  SensorOut so = element_sensor<P, EPB, real>(s2, ph, sQ, n_active, sV, le, tid, active,
                                             (active && feat) ? feat + size_t(e) * MLP_IN : nullptr);
  if (active && tid == 0 && out) {
    const double g = sa.kind == SENSOR_LEARNED ? so.g : (sa.kind == SENSOR_MODAL ? so.g_modal : -1.0);
    out[size_t(e) * 4 + 0] = so.g_modal;
    out[size_t(e) * 4 + 1] = sa.mlp ? so.g_learned : -1.0;
    out[size_t(e) * 4 + 2] = so.ood;
    out[size_t(e) * 4 + 3] = g;
  }
}

template <int P, typename real>
void launch_sensor_eval_P(hg_ctx* c, float* feat, double* out) {
  constexpr int EPB = epb_ns(P);
  const int grid = (c->n_el + EPB - 1) / EPB;
  sensor_eval_kernel<P, EPB, real><<<grid, block_ns(P), 0, c->stream>>>(c->n_el, c->d_Q, c->d_mats, sensor_args(c),
                                                                         c->pc, feat, out);
  ++c->launches;
}
