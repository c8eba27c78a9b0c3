// hg_launch.cuh -- definitions of the per-order launch templates declared in hg_ctx.h.
// Included only by the instantiation units hg_inst_*.cu.
#pragma once
#include "hg_ctx.h"

template <int P, typename real>
void launch_stage_P(hg_ctx* c, const StageArgs<real>& a) {
  constexpr int EPB = epb_for(P);
  const int grid = (a.n_el + EPB - 1) / EPB;
  static bool attr = false;
  if (!attr) {
    max_carveout(stage_kernel<P, EPB, real, true>);
    max_carveout(stage_kernel<P, EPB, real, false>);
    attr = true;
  }
  timed(c, HG_KERNEL_STAGE, [&] {
    if (c->affine) stage_kernel<P, EPB, real, true><<<grid, block_for(P), 0, c->stream>>>(a);
    else stage_kernel<P, EPB, real, false><<<grid, block_for(P), 0, c->stream>>>(a);
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

template <int P, typename real, bool AFFINE, bool IP, bool AV>
static void launch_ns_PAI(hg_ctx* c, const NSArgs<real>& a) {
  constexpr int EPB = epb_ns(P);
  const int grid = (a.n_el + EPB - 1) / EPB;
  static bool attr = false;
  if (!attr) {
    max_carveout(ns_gradient_kernel<P, EPB, real, AFFINE, IP, AV>);
    max_carveout(ns_stage_kernel<P, EPB, real, AFFINE, IP, AV>);
    attr = true;
  }
  timed(c, HG_KERNEL_GRADIENT,
        [&] { ns_gradient_kernel<P, EPB, real, AFFINE, IP, AV><<<grid, block_ns(P), 0, c->stream>>>(a); });
  timed(c, HG_KERNEL_STAGE,
        [&] { ns_stage_kernel<P, EPB, real, AFFINE, IP, AV><<<grid, block_ns(P), 0, c->stream>>>(a); });
  c->launches += 2;
}

template <int P, typename real>
void launch_ns_P(hg_ctx* c, const NSArgs<real>& a) {
  // artificial dissipation is a template switch so that the plain kernels keep their register budget
  if (c->av) {
    if (c->affine) {
      if (c->ip) launch_ns_PAI<P, real, true, true, true>(c, a); else launch_ns_PAI<P, real, true, false, true>(c, a);
    } else {
      if (c->ip) launch_ns_PAI<P, real, false, true, true>(c, a); else launch_ns_PAI<P, real, false, false, true>(c, a);
    }
  } else {
    if (c->affine) {
      if (c->ip) launch_ns_PAI<P, real, true, true, false>(c, a); else launch_ns_PAI<P, real, true, false, false>(c, a);
    } else {
      if (c->ip) launch_ns_PAI<P, real, false, true, false>(c, a); else launch_ns_PAI<P, real, false, false, false>(c, a);
    }
  }
}
