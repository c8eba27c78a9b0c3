// hg_api.cu -- C ABI of libhorsesgpu.so (declared in include/horses_gpu.h).
//
// Host responsibilities: validate the flattened mesh, turn the reference's
// edge-centric connectivity (mesh%edges, Mesh/QuadElement.f90:95-135 after
// Edge_LinkWithElements / Zone_LinkPeriodicZones) into per-element side tables,
// upload everything once, and sequence the stage kernels of the low-storage
// Runge-Kutta schemes (Approximation/DGTimeIntegrator.f90:263-365).
#include "hg_ctx.h"
#include "hg_spectral.h"

#include <cstring>
#include <cmath>
#include <algorithm>


static std::string g_create_err;

// A stepped state that is no longer physical (health_check): status HG_STATUS_CRASHED.
struct Crashed : std::runtime_error {
  using std::runtime_error::runtime_error;
};

static int fail(hg_ctx* c, const std::exception& ex) {
  if (c) c->err = ex.what();
  return dynamic_cast<const Crashed*>(&ex) ? HG_STATUS_CRASHED : 1;
}

template <typename T>
static T* dalloc(size_t n) {
  void* p = nullptr;
  HG_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  return static_cast<T*>(p);
}

static void drop_graph(hg_ctx* c) {
  for (auto& x : c->gexec) {
    if (x) cudaGraphExecDestroy(x);
    x = nullptr;
  }
  for (auto& x : c->gexec1) {
    if (x) cudaGraphExecDestroy(x);
    x = nullptr;
  }
  c->g_scheme = -1;
  c->g1_scheme = -1;
  c->g1_seen[0] = c->g1_seen[1] = 0;
  ++c->gen;
}

void ctx_free(hg_ctx* c) {
  if (!c) return;
  composite_free(c);
  drop_graph(c);
  for (cudaEvent_t e : c->prof_pool) cudaEventDestroy(e);
  void* ptrs[] = {c->d_side, c->d_side_geo, c->d_vol_geo, c->d_mats, c->d_zones, c->d_Q, c->d_G, c->d_T[0], c->d_T[1],
                  c->d_QDot, c->d_resid, c->d_resid_out, c->d_elmax, c->d_side_invh, c->d_jac, c->d_GT[0],
                  c->d_GT[1], c->d_av_el, c->d_side_area, c->d_mu_av[0], c->d_mu_av[1], c->d_mlp, c->d_feat_lo,
                  c->d_feat_hi, c->d_dQ,
                  c->d_FX, c->d_bq, c->d_si_out, c->d_NF, c->d_NFG, c->d_NJ, c->d_exact_sides};
  for (int* p : c->d_zone_sides) if (p) cudaFree(p);
  for (void* p : ptrs) if (p) cudaFree(p);
  if (!c->health_shared) {
    if (c->d_health) cudaFree(c->d_health);
    if (c->h_health) cudaFreeHost(c->h_health);
  }
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
}

// ------------------------------------------------------------------ health of the stepped state
// The stage kernels check every updated node (check_state, hg_stage.cuh) and set the device word
// {bits, element} and the mapped host flag; the host reads the flag without a synchronisation before
// each step call and after every synchronising call.
static void health_alloc(hg_ctx* c) {
  c->d_health = dalloc<int>(2);
  const int clean[2] = {0, -1};
  HG_CUDA(cudaMemcpy(c->d_health, clean, sizeof(clean), cudaMemcpyHostToDevice));
  void* h = nullptr;
  HG_CUDA(cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped));
  c->h_health = static_cast<int*>(h);
  *reinterpret_cast<volatile int*>(c->h_health) = 0;
  void* dptr = nullptr;
  HG_CUDA(cudaHostGetDevicePointer(&dptr, h, 0));
  c->d_health_flag = static_cast<int*>(dptr);
}

static void health_share(hg_ctx* part, const hg_ctx* owner) {
  part->d_health = owner->d_health;
  part->h_health = owner->h_health;
  part->d_health_flag = owner->d_health_flag;
  part->health_shared = true;
}

static void health_reset(hg_ctx* c) {
  const int clean[2] = {0, -1};
  HG_CUDA(cudaMemcpyAsync(c->d_health, clean, sizeof(clean), cudaMemcpyHostToDevice, c->stream));
  HG_CUDA(cudaStreamSynchronize(c->stream));
  *reinterpret_cast<volatile int*>(c->h_health) = 0;
}

// Throws the reference's crash message if a stage has flagged the state with a fatal condition (after
// synchronising, so that the word is complete); a no-op while the host flag is clean.  Conditions that
// are recorded but not fatal clear the host flag again, so that later calls do not synchronise until a
// new event.
static void health_check(hg_ctx* c) {
  if (!c->h_health || *reinterpret_cast<volatile int*>(c->h_health) == 0) return;
  HG_CUDA(cudaStreamSynchronize(c->stream));
  int w[2] = {0, -1};
  HG_CUDA(cudaMemcpy(w, c->d_health, sizeof(w), cudaMemcpyDeviceToHost));
  if ((w[0] & c->health_fatal) == 0) {
    *reinterpret_cast<volatile int*>(c->h_health) = 0;
    return;
  }
  std::string what;
  if (w[0] & HEALTH_NONFINITE) what += " a non-finite value";
  if (w[0] & HEALTH_DENSITY) what += std::string(what.empty() ? "" : ",") + " a non-positive density";
  if (w[0] & HEALTH_PRESSURE) what += std::string(what.empty() ? "" : ",") + " a non-positive pressure";
  throw Crashed("The simulation has crashed: the state holds" + what + " (element " + std::to_string(w[1]) +
                "); set a new state to continue");
}

static int epb_of(const hg_ctx* c, int variant) {
  return c->ns ? epb_ns_of(c->P, variant) : epb_stage(c->P, variant);
}
static int grid_for(const hg_ctx* c) {
  const int epb = epb_of(c, c->tiling);
  return (c->n_el + epb - 1) / epb;
}
// per-CTA residual partials: room for the tiling variant with the most CTAs
static int max_grid(const hg_ctx* c) {
  const int epb = std::min(epb_of(c, 0), epb_of(c, 1));
  return (c->n_el + epb - 1) / epb;
}

#define HG_DISPATCH_P(P_, FN, ...)                      \
  switch (P_) {                                         \
    case 2: FN<2, real>(__VA_ARGS__); break;            \
    case 3: FN<3, real>(__VA_ARGS__); break;            \
    case 4: FN<4, real>(__VA_ARGS__); break;            \
    case 5: FN<5, real>(__VA_ARGS__); break;            \
    case 6: FN<6, real>(__VA_ARGS__); break;            \
    case 7: FN<7, real>(__VA_ARGS__); break;            \
    case 8: FN<8, real>(__VA_ARGS__); break;            \
    case 9: FN<9, real>(__VA_ARGS__); break;            \
    default: throw std::runtime_error("unsupported polynomial order"); \
  }

// Euler kernels: orders 1-12
#define HG_DISPATCH_P_EULER(P_, FN, ...)                \
  switch (P_) {                                         \
    case 2: FN<2, real>(__VA_ARGS__); break;            \
    case 3: FN<3, real>(__VA_ARGS__); break;            \
    case 4: FN<4, real>(__VA_ARGS__); break;            \
    case 5: FN<5, real>(__VA_ARGS__); break;            \
    case 6: FN<6, real>(__VA_ARGS__); break;            \
    case 7: FN<7, real>(__VA_ARGS__); break;            \
    case 8: FN<8, real>(__VA_ARGS__); break;            \
    case 9: FN<9, real>(__VA_ARGS__); break;            \
    case 10: FN<10, real>(__VA_ARGS__); break;          \
    case 11: FN<11, real>(__VA_ARGS__); break;          \
    case 12: FN<12, real>(__VA_ARGS__); break;          \
    case 13: FN<13, real>(__VA_ARGS__); break;          \
    default: throw std::runtime_error("unsupported polynomial order"); \
  }

template <typename real>
static void run_trace(hg_ctx* c) { HG_DISPATCH_P_EULER(c->P, launch_trace_P, c); }

template <int P, typename real>
static void ns_dispatch(hg_ctx* c, const NSArgs<real>& a) {
  // orders 9-10 run one element per CTA in both tilings: one instantiation serves
  if (c->tiling && P < 10) launch_ns_PV<P, real, 1>(c, a);
  else launch_ns_PV<P, real, 0>(c, a);
}

// Navier-Stokes kernels: orders 1-8, 9 and 10
#define HG_DISPATCH_P_NS(P_, FN, ...)                   \
  switch (P_) {                                         \
    case 2: FN<2, real>(__VA_ARGS__); break;            \
    case 3: FN<3, real>(__VA_ARGS__); break;            \
    case 4: FN<4, real>(__VA_ARGS__); break;            \
    case 5: FN<5, real>(__VA_ARGS__); break;            \
    case 6: FN<6, real>(__VA_ARGS__); break;            \
    case 7: FN<7, real>(__VA_ARGS__); break;            \
    case 8: FN<8, real>(__VA_ARGS__); break;            \
    case 9: FN<9, real>(__VA_ARGS__); break;            \
    case 10: FN<10, real>(__VA_ARGS__); break;          \
    case 11: FN<11, real>(__VA_ARGS__); break;          \
    default: throw std::runtime_error("unsupported polynomial order"); \
  }
template <int P, typename real>
static void stage_dispatch(hg_ctx* c, const StageArgs<real>& a) {
  if (c->tiling) launch_stage_PV<P, real, 1>(c, a);
  else launch_stage_PV<P, real, 0>(c, a);
}

template <typename real>
static void run_ns_stage(hg_ctx* c, double ca, double cb, double cc, bool first, bool update, double* qdot, bool resid) {
  NSArgs<real> a{};
  a.n_el = c->n_el;
  a.side = c->d_side;
  a.side_geo = static_cast<const real*>(c->d_side_geo);
  a.side_invh = c->d_side_invh;
  a.vol_geo = static_cast<const real*>(c->d_vol_geo);
  a.jac = static_cast<const real*>(c->d_jac);
  a.mats = c->d_mats;
  a.zones = c->d_zones;
  a.bq = c->d_bq;
  a.FX = static_cast<const real*>(c->d_FX);
  a.NF = static_cast<const real*>(c->d_NF);
  a.NFG = static_cast<const real*>(c->d_NFG);
  a.NJ = static_cast<const real*>(c->d_NJ);
  a.Q = c->d_Q;
  a.G = static_cast<real*>(c->d_G);
  a.T_in = static_cast<const real*>(c->d_T[c->cur]);
  a.T_out = static_cast<real*>(c->d_T[c->cur ^ 1]);
  a.GT = static_cast<real*>(c->d_GT[c->cur]);
  a.GT_out = static_cast<real*>(c->d_GT[c->cur ^ 1]);
  a.dQ = static_cast<real*>(c->d_dQ);
  a.viscous = (c->pc.mu != 0.0 || c->av == HG_AV_PHYSICAL) ? 1 : 0;
  // BR1 always needs the lifted gradient; IP only for gradient traces (viscous fluxes) or the indicator
  // (the jumps indicator every stage, the modal and learned ones on the first stage of a step)
  a.run_gradient = (!c->ip || a.viscous ||
                    (c->av != HG_AV_NONE && (c->sensor_kind == HG_SENSOR_JUMPS || first))) ? 1 : 0;
  a.QDot = qdot;
  a.resid = resid ? c->d_resid : nullptr;
  a.a = ca; a.b = cb; a.c = cc;
  a.first = first ? 1 : 0;
  a.update = update ? 1 : 0;
  a.riemann = c->riemann;
  a.ip = c->ip ? 1 : 0;
  a.grad_faces = c->grad_faces ? 1 : 0;
  a.sigma0 = c->sigma0;
  a.epsilon = c->epsilon;
  a.pc = c->pc;
  a.av = c->av;
  a.av_el = c->d_av_el;
  a.side_area = c->d_side_area;
  if (!c->stepping) c->mu_step = c->cur;
  a.mu_av = c->d_mu_av[c->mu_step];
  a.mu_next = c->d_mu_av[c->cur ^ 1];
  a.sensor = sensor_args(c);
  a.health = c->d_health;
  a.health_host = c->d_health_flag;
  a.run_stage = c->ns_phase != 1;
  if (c->ns_phase == 2) a.run_gradient = 0;
  a.fuse = (ns_fused(c) && !c->prologue) ? 1 : 0;
  a.last = c->last_stage ? 1 : 0;
  if (a.fuse) a.run_gradient = 0;   // the previous stage (or the prologue) left GT and mu_av of this state
  if (c->prologue) {                // gradient traces and indicator of the resident state only
    a.run_gradient = 1;
    a.run_stage = 0;
  }
  c->mu_last = c->mu_step;
  if (c->exact && a.run_stage) launch_exact_flux<real>(c);
  HG_DISPATCH_P_NS(c->P, ns_dispatch, c, a);
  if (!a.run_stage) return;
  c->last_T = c->cur;   // trace buffer of the state this stage evaluated (surface integrals read it)
  if (update) c->cur ^= 1;
}

template <typename real>
static void run_stage(hg_ctx* c, double ca, double cb, double cc, bool first, bool update, double* qdot, bool resid) {
  if (c->ns) { run_ns_stage<real>(c, ca, cb, cc, first, update, qdot, resid); return; }
  StageArgs<real> a{};
  a.n_el = c->n_el;
  a.side = c->d_side;
  a.side_geo = static_cast<const real*>(c->d_side_geo);
  a.vol_geo = static_cast<const real*>(c->d_vol_geo);
  a.mats = c->d_mats;
  a.zones = c->d_zones;
  a.bq = c->d_bq;
  a.FX = static_cast<const real*>(c->d_FX);
  a.NF = static_cast<const real*>(c->d_NF);
  a.Q = c->d_Q;
  a.G = static_cast<real*>(c->d_G);
  a.T_in = static_cast<const real*>(c->d_T[c->cur]);
  a.T_out = static_cast<real*>(c->d_T[c->cur ^ 1]);
  a.QDot = qdot;
  a.resid = resid ? c->d_resid : nullptr;
  a.health = c->d_health;
  a.health_host = c->d_health_flag;
  a.a = ca; a.b = cb; a.c = cc;
  a.first = first ? 1 : 0;
  a.update = update ? 1 : 0;
  a.riemann = c->riemann;
  a.pc = c->pc;
  if (c->exact) launch_exact_flux<real>(c);
  HG_DISPATCH_P_EULER(c->P, stage_dispatch, c, a);
  c->last_T = c->cur;   // trace buffer of the state this stage evaluated (surface integrals read it)
  if (update) c->cur ^= 1;
}

void ctx_stage(hg_ctx* c, double ca, double cb, double cc, bool first, bool update, double* qdot, bool resid) {
  if (is_composite(c)) {
    // faces between orders and subdivided edges first, then every part's fused stage; the parts'
    // launches are counted on the composite.  Navier-Stokes (BR1): the mortar kernel's gradient face
    // terms, the parts' gradient kernels, the mortar kernel's inviscid + viscous fluxes (they need
    // the gradient traces), the parts' stage kernels.  Interior penalty: no gradient face terms; the
    // flux pass adds the penalty and the gradient-face terms.
    auto parts_stage = [&](int phase) {
      for (hg_ctx* p : c->parts) {
        const int64_t l0 = p->launches;
        p->ns_phase = phase;
        ctx_stage(p, ca, cb, cc, first, update, qdot ? p->d_QDot : nullptr, resid);
        p->ns_phase = 0;
        c->launches += p->launches - l0;
        p->launches = l0;
      }
    };
    if (c->ns) {
      if (!c->ip) launch_mortar(c, MORTAR_GRADIENT);   // the interior-penalty gradient is element-local
      if (c->av != HG_AV_NONE) launch_mortar(c, MORTAR_JUMPS);   // jumps of the faces between parts
      parts_stage(1);
      launch_mortar(c, MORTAR_FLUX);
      parts_stage(2);
    } else {
      launch_mortar(c, MORTAR_FLUX);
      parts_stage(0);
    }
    c->last_T = c->cur;
    if (update) c->cur ^= 1;
    return;
  }
  if (c->precision == HG_PREC_FP32) run_stage<float>(c, ca, cb, cc, first, update, qdot, resid);
  else run_stage<double>(c, ca, cb, cc, first, update, qdot, resid);
}

static void traces(hg_ctx* c) {
  if (c->precision == HG_PREC_FP32) run_trace<float>(c);
  else run_trace<double>(c);
}

// One step of a reference scheme; residual maxima are collected on the last stage.
// The indicator buffer of the step is the one of its starting trace parity (mu_step), and the last
// stage is flagged (a fused interior-penalty stage then writes the next step's indicator).
static void one_step(hg_ctx* c, int scheme, double t, double dt) {
  (void)t;
  struct Step {
    hg_ctx* c;
    explicit Step(hg_ctx* c_) : c(c_) { c->stepping = true; c->mu_step = c->cur; }
    ~Step() { c->stepping = false; c->last_stage = false; }
  } guard(c);
  if (scheme == HG_SCHEME_EULER) {
    c->last_stage = true;
    ctx_stage(c, 0.0, dt, 1.0, true, true, nullptr, true);
  } else if (scheme == HG_SCHEME_RK3) {
    const double am[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
    const double gm[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
    for (int m = 0; m < 3; ++m) {
      c->last_stage = m == 2;
      ctx_stage(c, am[m], 1.0, gm[m] * dt, m == 0, true, nullptr, m == 2);
    }
  } else if (scheme == HG_SCHEME_RK5) {
    const double am[5] = {0.0, -0.4178904745, -1.192151694643, -1.697784692471, -1.514183444257};
    const double gm[5] = {0.1496590219993, 0.3792103129999, 0.8229550293869, 0.6994504559488, 0.1530572479681};
    for (int m = 0; m < 5; ++m) {
      c->last_stage = m == 4;
      ctx_stage(c, am[m], dt, gm[m], m == 0, true, nullptr, m == 4);
    }
  } else {
    throw std::runtime_error("unknown time scheme");
  }
}

// The fused interior-penalty path's prologue: gradient traces and indicator of the resident state (the
// gradient kernel alone), after the state or the indicator has been replaced.
static void ns_prologue(hg_ctx* c) {
  if (!ns_fused(c) || !c->state_set) return;
  c->prologue = true;
  try {
    ctx_stage(c, 0.0, 0.0, 0.0, true, false, nullptr, false);
  } catch (...) {
    c->prologue = false;
    throw;
  }
  c->prologue = false;
}

// ------------------------------------------------------------------ dt estimate
// TimeIntegrator_EstimateTimeStep (DGTimeIntegrator.f90:462-511) keeps running maxima of |u| and a over
// the nodes (iXi outer, iEta inner) of the elements in mesh order, SAVEd across calls, and takes
// dt = MIN(dt, M sqrt(gamma) CFL dx / (umax + amax) / (N + 1)) after each element.  A node whose internal
// energy has gone negative (transients of the CylinderMach2 benchmark) gives a = sqrt(<0) = NaN.  The
// reference's compiled MAX / MIN behave as one x86 maxsd / minsd with the running value first: a NaN
// operand replaces the running value and the next ordinary value replaces the NaN -- with that rule the
// benchmark's asserted iteration count (15599) is reproduced.  Per element this kernel reports, for
// |u| and a, the plain maximum (flag 0: no NaN among its nodes) or the maximum after its last NaN node,
// NaN if that is the last node (flag 1): the running value after the element is then run_max(R, value)
// or that value; the host applies the element sequence.
__global__ void element_speed_kernel(int n_el, int P, const double* Q, double gamma, double gm1, double* out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_el) return;
  const double* qe = Q + size_t(e) * P * P * 4;
  double ua = -INFINITY, uafter = -INFINITY, aa = -INFINITY, aafter = -INFINITY;
  bool unan = false, ulast = false, anan = false, alast = false;
  for (int i = 0; i < P; ++i)
    for (int j = 0; j < P; ++j) {
      const double* q = qe + 4 * (j * P + i);
      const double u = sqrt(q[1] * q[1] + q[2] * q[2]) / q[0];
      const double uu = q[1] / q[0], vv = q[2] / q[0];
      const double a = sqrt(gamma * gm1 * (q[3] / q[0] - 0.5 * (uu * uu) - 0.5 * (vv * vv)));
      if (u != u) { unan = ulast = true; uafter = -INFINITY; }
      else { ulast = false; ua = u > ua ? u : ua; uafter = u > uafter ? u : uafter; }
      if (a != a) { anan = alast = true; aafter = -INFINITY; }
      else { alast = false; aa = a > aa ? a : aa; aafter = a > aafter ? a : aafter; }
    }
  out[4 * size_t(e) + 0] = unan ? (ulast ? NAN : uafter) : ua;
  out[4 * size_t(e) + 1] = unan ? 1.0 : 0.0;
  out[4 * size_t(e) + 2] = anan ? (alast ? NAN : aafter) : aa;
  out[4 * size_t(e) + 3] = anan ? 1.0 : 0.0;
}

// The reference's MAX / MIN on the running value a and a new operand b (see element_speed_kernel).
static inline double run_max(double a, double b) { return a > b ? a : b; }
static inline double run_min(double a, double b) { return a < b ? a : b; }
static inline double element_running(double R, const double* v) { return v[1] != 0.0 ? v[0] : run_max(R, v[0]); }

// ------------------------------------------------------------------ creation
void ctx_build(hg_ctx* c, const hg_mesh_desc* m, const hg_physics_desc* ph, const hg_bc_desc* bcs, int n_bcs,
               const std::vector<int2>* flux_sides) {
  if (!m || !ph) throw std::runtime_error("null descriptor");
  int dev = 0;
  HG_CUDA(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  HG_CUDA(cudaGetDeviceProperties(&prop, dev));
  if (prop.major < 10) throw std::runtime_error("libhorsesgpu requires an sm_100 (Blackwell) device");
  const int E = m->n_elements;
  if (E <= 0) throw std::runtime_error("mesh has no elements");
  const int N = m->N[0];
  for (int e = 0; e < E; ++e)
    if (m->N[e] != N) throw std::runtime_error("mixed polynomial orders are not supported by this kernel set");
  if (ph->navier_stokes ? (N < 1 || N > HG_MAX_ORDER_NS) : (N < 1 || N > HG_MAX_ORDER_EULER))
    throw std::runtime_error(ph->navier_stokes ? "polynomial order must be in 1..10 for the Navier-Stokes build"
                                               : "polynomial order must be in 1..12");
  if (m->n_mortars > 0) throw std::runtime_error("subdivided edges need the composite context");
  const int P = N + 1, NP = P * P;
  // the Navier-Stokes build with Re = 0 has mu = 0: its viscous terms vanish identically
  if (ph->av_type < HG_AV_NONE || ph->av_type > HG_AV_PHYSICAL) throw std::runtime_error("unknown artificial dissipation type");
  c->av = ph->navier_stokes ? ph->av_type : HG_AV_NONE;   // artificial dissipation exists in the Navier-Stokes build
  // the Navier-Stokes build with Re = 0 has mu = 0: its viscous terms vanish identically unless
  // artificial dissipation is on
  c->ns = ph->navier_stokes != 0 && (ph->reynolds != 0.0 || c->av != HG_AV_NONE);
  c->ip = ph->viscous == 1;
  c->grad_faces = c->ip && ph->ip_method != 2;
  c->sigma0 = ph->sigma0_ip;
  c->epsilon = ph->ip_method == 0 ? -1.0 : (ph->ip_method == 1 ? 1.0 : 0.0);
  c->n_el = E; c->N = N; c->P = P; c->node_type = ph->node_type; c->riemann = ph->riemann;
  c->ndof = int64_t(E) * NP * 4;
  const double gamma = ph->gamma > 0 ? ph->gamma : 1.4;
  c->gamma = gamma; c->mach = ph->mach;
  c->pc.gamma = gamma;
  c->pc.gm1 = gamma - 1.0;
  c->pc.cp = gamma / (gamma - 1.0);
  c->pc.cv = 1.0 / (gamma - 1.0);
  c->pc.invSqrtGammaMach = 1.0 / (std::sqrt(gamma) * ph->mach);
  c->pc.mu = (ph->navier_stokes != 0 && ph->reynolds != 0.0) ? 1.0 / ph->reynolds : 0.0;
  c->pc.cpPr = c->pc.cp / ph->prandtl;
  c->pc.lambda = -2.0 / 3.0;
  c->temperature_ref = ph->temperature_ref;

  // nodal operators
  NodalOps ops = make_nodal_ops(N, ph->node_type);
  std::vector<double> mats;
  mats.insert(mats.end(), ops.hatD.begin(), ops.hatD.end());
  mats.insert(mats.end(), ops.lb0.begin(), ops.lb0.end());
  mats.insert(mats.end(), ops.lb1.begin(), ops.lb1.end());
  mats.insert(mats.end(), ops.lbw0.begin(), ops.lbw0.end());
  mats.insert(mats.end(), ops.lbw1.begin(), ops.lbw1.end());
  mats.insert(mats.end(), ops.D.begin(), ops.D.end());
  mats.insert(mats.end(), ops.dlbw0.begin(), ops.dlbw0.end());
  mats.insert(mats.end(), ops.dlbw1.begin(), ops.dlbw1.end());
  mats.insert(mats.end(), ops.w.begin(), ops.w.end());
  mats.insert(mats.end(), ops.Vinv.begin(), ops.Vinv.end());
  mats.insert(mats.end(), ops.xi.begin(), ops.xi.end());   // probes: nodes and barycentric weights
  mats.insert(mats.end(), ops.wb.begin(), ops.wb.end());
  c->sensor_s0 = std::log10(1.0 / std::pow(double(N + 1), 4.0));   // modal ramp defaults
  c->sensor_kappa = 1.0;

  // volume metrics
  std::vector<double> vg(size_t(E) * NP * 5);
  for (size_t n = 0; n < size_t(E) * NP; ++n) {
    for (int k = 0; k < 4; ++k) vg[n * 5 + k] = m->Ja[n * 4 + k];
    if (!(m->jac[n] > 0.0)) throw std::runtime_error("non-positive mapping jacobian");
    vg[n * 5 + 4] = 1.0 / m->jac[n];
  }

  // zones
  std::vector<Zone> zones(std::max(1, n_bcs));
  c->zone_type.assign(std::max(1, n_bcs), -1);
  c->zone_row0.assign(std::max(1, n_bcs), -1);
  for (int z = 0; z < n_bcs; ++z) {
    c->zone_type[z] = bcs[z].type;
    zones[z].type = bcs[z].type;
    zones[z].riemann = bcs[z].riemann;
    for (int k = 0; k < 4; ++k) zones[z].q[k] = bcs[z].state[k];
    zones[z].Tw = bcs[z].wall_T;
    zones[z].vw[0] = bcs[z].wall_v[0];
    zones[z].vw[1] = bcs[z].wall_v[1];
    zones[z].wall_type = bcs[z].wall_type;
    zones[z].outflow_type = bcs[z].outflow_type;
    zones[z].nd_mode = bcs[z].nd_mode;
    zones[z].nd_outflow_total = bcs[z].nd_outflow_total;
    if (bcs[z].riemann == HG_RIEMANN_EXACT) c->exact = true;
  }

  // side tables
  // {neighbour trace slot, flags, zone, per-node state row}; rows are assigned by hg_set_boundary_state
  std::vector<int4> side(size_t(E) * 4, make_int4(-2, 0, -1, -1));
  c->zone_sides.assign(std::max(1, n_bcs), std::vector<int>());
  std::vector<double> sinvh(size_t(E) * 4, 0.0);
  std::vector<double> sg(size_t(E) * 4 * P * 3, 0.0);
  auto set_geo = [&](int e, int s, int edge, bool rev) {
    for (int k = 0; k < P; ++k) {
      const int cidx = rev ? (P - 1 - k) : k;
      double* g = &sg[((size_t(e) * 4 + s) * P + k) * 3];
      g[0] = m->edge_n[(size_t(edge) * P + cidx) * 2];
      g[1] = m->edge_n[(size_t(edge) * P + cidx) * 2 + 1];
      g[2] = m->edge_dS[size_t(edge) * P + cidx];
    }
  };
  for (int f = 0; f < m->n_edges; ++f) {
    const int L = m->edge_elem[2 * f], R = m->edge_elem[2 * f + 1];
    const int sL = m->edge_side[2 * f] - 1, sR = m->edge_side[2 * f + 1] - 1;
    const bool inv = m->edge_inverse[f] != 0;
    if (L < 0 || L >= E || sL < 0 || sL > 3) throw std::runtime_error("bad edge connectivity");
    const int marker = m->edge_marker[f];
    if (marker == 0) {
      if (R < 0 || R >= E || sR < 0 || sR > 3) throw std::runtime_error("interior edge without RIGHT element");
      side[size_t(L) * 4 + sL] = make_int4(R * 4 + sR, SIDE_LEFT | (inv ? SIDE_REVERSED : 0), -1, -1);
      side[size_t(R) * 4 + sR] = make_int4(L * 4 + sL, SIDE_RIGHT | (inv ? SIDE_REVERSED : 0), -1, -1);
      set_geo(L, sL, f, false);
      set_geo(R, sR, f, inv);
      if (m->edge_invh) sinvh[size_t(L) * 4 + sL] = sinvh[size_t(R) * 4 + sR] = m->edge_invh[f];
    } else {
      if (marker < 1 || marker > n_bcs) throw std::runtime_error("boundary edge with unknown marker");
      const hg_bc_desc& b = bcs[marker - 1];
      const int z = marker - 1;
      switch (b.type) {
        case HG_BC_PERIODIC: {
          const int p = m->periodic_partner ? m->periodic_partner[f] : -1;
          if (p < 0 || p >= m->n_edges) throw std::runtime_error("periodic edge without partner");
          const int pe = m->edge_elem[2 * p], ps = m->edge_side[2 * p] - 1;
          side[size_t(L) * 4 + sL] = make_int4(pe * 4 + ps, SIDE_LEFT | (inv ? SIDE_REVERSED : 0), z, -1);
          break;
        }
        case HG_BC_EULERWALL: side[size_t(L) * 4 + sL] = make_int4(-1, SIDE_WALL, z, -1); break;
        case HG_BC_DIRICHLET:
        case HG_BC_VISCOUSWALL:
        case HG_BC_FARFIELD:
        case HG_BC_PRESSUREOUTLET:
        case HG_BC_NEWDIRICHLET: side[size_t(L) * 4 + sL] = make_int4(-1, SIDE_STATE, z, -1); break;
        default: throw std::runtime_error("unknown boundary condition kind");
      }
      c->zone_sides[z].push_back(L * 4 + sL);
      set_geo(L, sL, f, false);
      if (m->edge_invh) sinvh[size_t(L) * 4 + sL] = m->edge_invh[f];
    }
  }
  if (flux_sides)
    for (const int2& fs : *flux_sides) {
      if (fs.x < 0 || size_t(fs.x) >= side.size() || side[fs.x].x != -2) throw std::runtime_error("bad mortar side");
      side[fs.x] = make_int4(fs.y, SIDE_FLUX, -1, -1);
    }
  for (size_t s = 0; s < side.size(); ++s)
    if (side[s].x == -2) throw std::runtime_error("element side not covered by any edge");

  // Affine detection: every node of an element carries the same metrics and every
  // side the same normal and dS (to 1e-14 relative); then the kernel reads one
  // value per element / side instead of one per node.
  {
    auto close = [](double a, double b, double scale) { return std::fabs(a - b) <= 1e-14 * scale; };
    bool aff = true;
    for (int e = 0; e < E && aff; ++e) {
      const double* g0 = &vg[size_t(e) * NP * 5];
      double sc = 0.0;
      for (int k = 0; k < 4; ++k) sc = std::fmax(sc, std::fabs(g0[k]));
      for (int n = 1; n < NP && aff; ++n)
        for (int k = 0; k < 5; ++k)
          if (!close(g0[n * 5 + k], g0[k], k < 4 ? sc : std::fabs(g0[4]))) { aff = false; break; }
      for (int s = 0; s < 4 && aff; ++s) {
        const double* s0 = &sg[(size_t(e) * 4 + s) * P * 3];
        for (int k = 1; k < P && aff; ++k)
          for (int q = 0; q < 3; ++q)
            if (!close(s0[k * 3 + q], s0[q], q < 2 ? 1.0 : std::fabs(s0[2]))) { aff = false; break; }
      }
    }
    c->affine = aff;
    if (aff) {
      std::vector<double> vg1(size_t(E) * 5), sg1(size_t(E) * 4 * 3);
      for (int e = 0; e < E; ++e) {
        for (int k = 0; k < 5; ++k) vg1[size_t(e) * 5 + k] = vg[size_t(e) * NP * 5 + k];
        for (int s = 0; s < 4; ++s)
          for (int q = 0; q < 3; ++q) sg1[(size_t(e) * 4 + s) * 3 + q] = sg[(size_t(e) * 4 + s) * P * 3 + q];
      }
      vg.swap(vg1);
      sg.swap(sg1);
    }
  }

  // dt support: corner distances
  c->dx.assign(E, 0.0);
  if (m->vertices) {
    for (int e = 0; e < E; ++e) {
      const double* v = m->vertices + size_t(e) * 8;
      auto d = [&](int a, int b) { return std::sqrt((v[2 * a] - v[2 * b]) * (v[2 * a] - v[2 * b]) + (v[2 * a + 1] - v[2 * b + 1]) * (v[2 * a + 1] - v[2 * b + 1])); };
      c->dx[e] = std::fmin(std::fmin(d(0, 1), d(1, 2)), std::fmin(d(2, 3), d(0, 3)));
    }
  }

  HG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  c->own_stream = true;
  const size_t rs = c->precision == HG_PREC_FP32 ? sizeof(float) : sizeof(double);
  c->d_side = dalloc<int4>(side.size());
  // geometry in the arithmetic precision of the context (FP32 bulk path: float, half the bytes)
  auto upload_real = [&](void*& dst, const double* src, size_t n) {
    if (c->precision == HG_PREC_FP32) {
      std::vector<float> f(src, src + n);
      dst = dalloc<float>(n);
      HG_CUDA(cudaMemcpy(dst, f.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    } else {
      dst = dalloc<double>(n);
      HG_CUDA(cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyHostToDevice));
    }
  };
  upload_real(c->d_side_geo, sg.data(), sg.size());
  upload_real(c->d_vol_geo, vg.data(), vg.size());
  c->d_mats = dalloc<double>(mats.size());
  c->d_zones = dalloc<Zone>(zones.size());
  c->d_Q = dalloc<double>(c->ndof);
  c->d_G = dalloc<char>(c->ndof * rs);
  c->d_T[0] = dalloc<char>(size_t(E) * 4 * P * 4 * rs);
  c->d_T[1] = dalloc<char>(size_t(E) * 4 * P * 4 * rs);
  c->d_QDot = dalloc<double>(c->ndof);
  c->d_resid = dalloc<double>(size_t(max_grid(c)) * 4);
  c->d_resid_out = dalloc<double>(4);
  c->d_elmax = dalloc<double>(size_t(E) * 4);
  if (c->av != HG_AV_NONE) {
    // Edge_t%Area = sum_p dS(p) w(p) in the edge's node order (QuadMesh_Construct.incf:270-303), per side;
    // per element Ceps sqrt(Volume)/(N+1) and the sum of the four areas (JumpsBasedElementViscosity)
    if (!m->volume) throw std::runtime_error("artificial dissipation needs element volumes");
    std::vector<double> area(size_t(E) * 4, 0.0), avel(size_t(E) * 2, 0.0);
    for (int f = 0; f < m->n_edges; ++f) {
      double A = 0.0;
      for (int p = 0; p < P; ++p) A += m->edge_dS[size_t(f) * P + p] * ops.w[p];
      const int L = m->edge_elem[2 * f], R = m->edge_elem[2 * f + 1];
      area[size_t(L) * 4 + m->edge_side[2 * f] - 1] = A;
      if (m->edge_marker[f] == 0) area[size_t(R) * 4 + m->edge_side[2 * f + 1] - 1] = A;
    }
    for (int e = 0; e < E; ++e) {
      const double maxVisc = std::sqrt(m->volume[e]) / (N + 1);
      avel[2 * size_t(e)] = ph->av_intensity * maxVisc;
      const double* A = &area[size_t(e) * 4];
      avel[2 * size_t(e) + 1] = A[0] + A[1] + A[2] + A[3];
    }
    c->d_av_el = dalloc<double>(avel.size());
    c->d_side_area = dalloc<double>(area.size());
    for (auto& m_ : c->d_mu_av) {
      m_ = dalloc<double>(size_t(E));
      HG_CUDA(cudaMemset(m_, 0, size_t(E) * sizeof(double)));
    }
    HG_CUDA(cudaMemcpy(c->d_av_el, avel.data(), avel.size() * sizeof(double), cudaMemcpyHostToDevice));
    HG_CUDA(cudaMemcpy(c->d_side_area, area.data(), area.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (c->ns) {
    if (c->ip && !m->edge_invh) throw std::runtime_error("interior penalty needs edge_invh");
    c->d_side_invh = dalloc<double>(sinvh.size());
    for (auto& g_ : c->d_GT) g_ = dalloc<char>(size_t(E) * 4 * P * 8 * rs);
    c->d_dQ = dalloc<char>(size_t(c->ndof) * 2 * rs);
    HG_CUDA(cudaMemcpy(c->d_side_invh, sinvh.data(), sinvh.size() * sizeof(double), cudaMemcpyHostToDevice));
    if (!c->affine) {
      upload_real(c->d_jac, m->jac, size_t(E) * NP);
    }
  }
  if (c->riemann == HG_RIEMANN_EXACT) c->exact = true;
  if (c->exact) {
    c->d_FX = dalloc<char>(size_t(E) * 4 * P * 4 * rs);
    // the sides whose Riemann problem the exact solver takes (the stage kernels' own selection)
    std::vector<int> ex;
    for (size_t es = 0; es < side.size(); ++es) {
      const int kind = side[es].y & 15;
      if (kind == SIDE_WALL || kind == SIDE_FLUX) continue;
      int solver = c->riemann;
      if (side[es].z >= 0 && zones[side[es].z].riemann >= 0) solver = zones[side[es].z].riemann;
      if (solver == HG_RIEMANN_EXACT) ex.push_back(int(es));
    }
    c->n_exact_sides = int(ex.size());
    c->d_exact_sides = dalloc<int>(ex.size());
    HG_CUDA(cudaMemcpy(c->d_exact_sides, ex.data(), ex.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  c->h_side = side;
  HG_CUDA(cudaMemcpy(c->d_side, side.data(), side.size() * sizeof(int4), cudaMemcpyHostToDevice));
  HG_CUDA(cudaMemcpy(c->d_mats, mats.data(), mats.size() * sizeof(double), cudaMemcpyHostToDevice));
  HG_CUDA(cudaMemcpy(c->d_zones, zones.data(), zones.size() * sizeof(Zone), cudaMemcpyHostToDevice));
  HG_CUDA(cudaMemset(c->d_resid, 0, size_t(max_grid(c)) * 4 * sizeof(double)));
}

extern "C" int hg_create(const hg_mesh_desc* mesh, const hg_physics_desc* phys, const hg_bc_desc* bcs, int32_t n_bcs,
                         int32_t precision, hg_ctx** out) {
  if (!out) return 1;
  *out = nullptr;
  hg_ctx* c = new hg_ctx();
  c->precision = precision;
  try {
    if (precision != HG_PREC_FP64 && precision != HG_PREC_FP32) throw std::runtime_error("unknown precision");
    if (!mesh || !phys) throw std::runtime_error("null descriptor");
    bool mixed = mesh->n_mortars > 0;
    for (int e = 1; e < mesh->n_elements && !mixed; ++e) mixed = mesh->N[e] != mesh->N[0];
    if (mixed) composite_build(c, mesh, phys, bcs, n_bcs);
    else ctx_build(c, mesh, phys, bcs, n_bcs, nullptr);
    health_alloc(c);
    for (hg_ctx* p : c->parts) health_share(p, c);
  } catch (const std::exception& ex) {
    g_create_err = ex.what();
    ctx_free(c);
    delete c;
    return 1;
  }
  g_create_err.clear();
  *out = c;
  return 0;
}

extern "C" void hg_destroy(hg_ctx* c) {
  if (!c) return;
  autosave_finish(c);
  if (c->stream) cudaStreamSynchronize(c->stream);
  ctx_free(c);
  delete c;
}

extern "C" const char* hg_last_error(const hg_ctx* c) { return c ? c->err.c_str() : g_create_err.c_str(); }
extern "C" int64_t hg_ndof(const hg_ctx* c) { return c ? c->ndof : -1; }
extern "C" double* hg_device_state(hg_ctx* c) { return c ? c->d_Q : nullptr; }   // NULL for a composite
extern "C" int64_t hg_launch_count(const hg_ctx* c) { return c ? c->launches : -1; }

// ------------------------------------------------------------------ composite contexts
// A mesh with mixed orders or subdivided edges is served by one part per order (hg_mortar.cu); the
// entry points below scatter Storage%Q to the parts, gather from them, and combine their results.
#define HG_PART(call, p)                                             \
  do {                                                               \
    if ((call) != 0) throw std::runtime_error((p)->err);             \
  } while (0)

static double nanmax_h(double m, double v) { return (v > m || v != v) ? v : m; }

// a non-null QDot target: a composite's parts write their own buffers
static double* qdot_target(hg_ctx* c) { return is_composite(c) ? c->parts[0]->d_QDot : c->d_QDot; }

static void composite_scatter(hg_ctx* c, const double* Q) {
  for (size_t pi = 0; pi < c->parts.size(); ++pi) {
    hg_ctx* p = c->parts[pi];
    const size_t n = size_t(p->P) * p->P * 4;
    std::vector<double> q(p->ndof);
    for (int e = 0; e < c->n_el; ++e)
      if (c->el_part[e] == int(pi))
        std::copy(Q + c->el_offset[e], Q + c->el_offset[e] + n, q.begin() + size_t(c->el_local[e]) * n);
    HG_PART(hg_set_state(p, q.data(), p->ndof), p);
  }
}

static void composite_gather(hg_ctx* c, double* Q, bool qdot) {
  for (size_t pi = 0; pi < c->parts.size(); ++pi) {
    hg_ctx* p = c->parts[pi];
    const size_t n = size_t(p->P) * p->P * 4;
    std::vector<double> q(p->ndof);
    HG_CUDA(cudaMemcpyAsync(q.data(), qdot ? p->d_QDot : p->d_Q, p->ndof * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    HG_CUDA(cudaStreamSynchronize(c->stream));
    for (int e = 0; e < c->n_el; ++e)
      if (c->el_part[e] == int(pi))
        std::copy(q.begin() + size_t(c->el_local[e]) * n, q.begin() + size_t(c->el_local[e] + 1) * n, Q + c->el_offset[e]);
  }
}

static void composite_residuals(hg_ctx* c, double out[4]) {
  for (int k = 0; k < 4; ++k) out[k] = 0.0;
  for (hg_ctx* p : c->parts) {
    double r[4];
    const int64_t l0 = p->launches;
    HG_PART(hg_residuals(p, r), p);
    c->launches += p->launches - l0;
    p->launches = l0;
    for (int k = 0; k < 4; ++k) out[k] = nanmax_h(out[k], r[k]);
  }
}

static int largest_part(const hg_ctx* c) {
  int b = 0;
  for (size_t p = 1; p < c->parts.size(); ++p)
    if (c->parts[p]->n_el > c->parts[b]->n_el) b = int(p);
  return b;
}

static void check_ndof(hg_ctx* c, int64_t ndof) {
  if (ndof != c->ndof) throw std::runtime_error("ndof mismatch: expected " + std::to_string(c->ndof));
}

extern "C" int hg_set_state(hg_ctx* c, const double* Q, int64_t ndof) {
  try {
    if (is_composite(c)) {
      check_ndof(c, ndof);
      health_reset(c);
      composite_scatter(c, Q);
      c->cur = 0;
      c->state_set = true;
      return 0;
    }
    check_ndof(c, ndof);
    health_reset(c);
    HG_CUDA(cudaMemcpyAsync(c->d_Q, Q, ndof * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    c->cur = 0;
    traces(c);
    c->state_set = true;
    ns_prologue(c);
    HG_CUDA(cudaGetLastError());
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_get_state(hg_ctx* c, double* Q, int64_t ndof) {
  try {
    if (is_composite(c)) {
      check_ndof(c, ndof);
      composite_gather(c, Q, false);
      health_check(c);
      return 0;
    }
    check_ndof(c, ndof);
    HG_CUDA(cudaMemcpyAsync(Q, c->d_Q, ndof * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HG_CUDA(cudaStreamSynchronize(c->stream));
    health_check(c);
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

static void require_state(hg_ctx* c) {
  if (!c->state_set) throw std::runtime_error("state not set (call hg_set_state first)");
}

extern "C" int hg_time_derivative(hg_ctx* c, double t, double* QDot) {
  try {
    require_state(c);
    health_check(c);
    (void)t;
    ctx_stage(c, 0.0, 0.0, 0.0, true, false, qdot_target(c), true);
    HG_CUDA(cudaGetLastError());
    if (QDot && is_composite(c)) {
      composite_gather(c, QDot, true);
    } else if (QDot) {
      HG_CUDA(cudaMemcpyAsync(QDot, c->d_QDot, c->ndof * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      HG_CUDA(cudaStreamSynchronize(c->stream));
    }
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

static int scheme_stages(int scheme) { return scheme == HG_SCHEME_EULER ? 1 : (scheme == HG_SCHEME_RK3 ? 3 : 5); }

// A composite's parts step in lockstep with it: their trace parity and last evaluated traces follow
// the composite's after a capture (which ran nothing) and after a replay.
static void sync_parts(hg_ctx* c) {
  for (hg_ctx* p : c->parts) {
    p->cur = c->cur;
    p->last_T = c->last_T;
  }
}

// One step through a CUDA graph of that single step, one per trace-buffer parity at its start (an odd
// number of stages flips the parity), for callers that step one at a time: the reference's loop with
// a residual check per iteration.  The first step of a scheme and dt at a parity runs as plain
// launches (it also sets kernel attributes outside any capture), the second is captured.
static void graph_one_step(hg_ctx* c, int scheme, double t, double dt) {
  if (c->g1_scheme != scheme || c->g1_dt != dt) {
    for (auto& x : c->gexec1) {
      if (x) cudaGraphExecDestroy(x);
      x = nullptr;
    }
    c->g1_seen[0] = c->g1_seen[1] = 0;
    c->g1_scheme = scheme;
    c->g1_dt = dt;
  }
  const int p = c->cur;
  if (!c->gexec1[p]) {
    if (c->g1_seen[p]++ == 0) {
      one_step(c, scheme, t, dt);
      return;
    }
    const int64_t l0 = c->launches;
    HG_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    try {
      one_step(c, scheme, t, dt);
    } catch (...) {
      cudaGraph_t g0 = nullptr;
      cudaStreamEndCapture(c->stream, &g0);
      if (g0) cudaGraphDestroy(g0);
      c->launches = l0;
      c->cur = p;
      sync_parts(c);
      throw;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
    c->g1_launches[p] = c->launches - l0;
    c->g1_last_T[p] = c->last_T;
    c->launches = l0;
    c->cur = p;   // the capture ran nothing
    sync_parts(c);
    HG_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&c->gexec1[p], g, 0);
    cudaGraphDestroy(g);
    HG_CUDA(ie);
  }
  HG_CUDA(cudaGraphLaunch(c->gexec1[p], c->stream));
  c->launches += c->g1_launches[p];
  c->last_T = c->g1_last_T[p];
  c->cur = p ^ (scheme_stages(scheme) & 1);
  sync_parts(c);
}

extern "C" int hg_time_step(hg_ctx* c, int32_t scheme, double t, double dt) {
  try {
    require_state(c);
    health_check(c);
    if (!c->prof && c->stream != nullptr &&
        (scheme == HG_SCHEME_EULER || scheme == HG_SCHEME_RK3 || scheme == HG_SCHEME_RK5))
      graph_one_step(c, scheme, t, dt);
    else
      one_step(c, scheme, t, dt);
    HG_CUDA(cudaGetLastError());
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

// Steps in pairs through a CUDA graph captured from the context's stream: two steps leave the trace
// buffers in their starting parity, so one graph serves every pair.  Kernel arguments that change
// between steps would invalidate it; with a constant dt none do (the schemes' coefficients depend on
// dt only, the stepping time t enters no kernel).
static void graph_steps(hg_ctx* c, int scheme, int n_steps, double t0, double dt) {
  int s = 0;
  if (c->g_scheme != scheme || c->g_dt != dt) drop_graph(c);
  if (!c->gexec[c->cur]) {
    one_step(c, scheme, t0, dt);   // first launches set kernel attributes outside any capture
    ++s;
  }
  if (!c->gexec[c->cur]) {
    const int64_t l0 = c->launches;
    const int cur0 = c->cur;
    HG_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    try {
      one_step(c, scheme, t0, dt);
      one_step(c, scheme, t0, dt);
    } catch (...) {
      cudaGraph_t g0 = nullptr;
      cudaStreamEndCapture(c->stream, &g0);
      if (g0) cudaGraphDestroy(g0);
      c->launches = l0;
      c->cur = cur0;
      throw;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
    c->g_launches[cur0] = c->launches - l0;
    c->launches = l0;
    c->cur = cur0;   // two steps flip the parity an even number of times; the capture ran nothing
    HG_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&c->gexec[cur0], g, 0);
    cudaGraphDestroy(g);
    HG_CUDA(ie);
    c->g_scheme = scheme;
    c->g_dt = dt;
  }
  for (; s + 2 <= n_steps; s += 2) {
    HG_CUDA(cudaGraphLaunch(c->gexec[c->cur], c->stream));
    c->launches += c->g_launches[c->cur];
  }
  for (; s < n_steps; ++s) one_step(c, scheme, t0 + s * dt, dt);
}

extern "C" int hg_time_steps(hg_ctx* c, int32_t scheme, int32_t n_steps, double t0, double dt) {
  try {
    require_state(c);
    health_check(c);
    if (n_steps >= 5 && !c->prof && c->stream != nullptr) {
      graph_steps(c, scheme, n_steps, t0, dt);
    } else {
      for (int s = 0; s < n_steps; ++s) one_step(c, scheme, t0 + s * dt, dt);
    }
    HG_CUDA(cudaGetLastError());
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_residuals(hg_ctx* c, double out[4]) {
  try {
    if (is_composite(c)) {
      composite_residuals(c, out);
      health_check(c);
      return 0;
    }
    timed(c, HG_KERNEL_REDUCE,
          [&] { residual_reduce_kernel<<<1, 256, 0, c->stream>>>(grid_for(c), c->d_resid, c->d_resid_out); });
    ++c->launches;
    HG_CUDA(cudaGetLastError());
    HG_CUDA(cudaMemcpyAsync(out, c->d_resid_out, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HG_CUDA(cudaStreamSynchronize(c->stream));
    health_check(c);
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_estimate_dt(hg_ctx* c, double cfl, double dt_cap, double* dt) {
  try {
    require_state(c);
    const int threads = 256;
    if (is_composite(c)) {
      // per-element maxima from every part, then the running maxima over the mesh's element order
      std::vector<std::vector<double>> em(c->parts.size());
      for (size_t pi = 0; pi < c->parts.size(); ++pi) {
        hg_ctx* p = c->parts[pi];
        timed(c, HG_KERNEL_SPEED, [&] {
          element_speed_kernel<<<(p->n_el + threads - 1) / threads, threads, 0, c->stream>>>(
              p->n_el, p->P, p->d_Q, c->gamma, c->gamma - 1.0, p->d_elmax);
        });
        ++c->launches;
        HG_CUDA(cudaGetLastError());
        em[pi].resize(size_t(p->n_el) * 4);
        HG_CUDA(cudaMemcpyAsync(em[pi].data(), p->d_elmax, em[pi].size() * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
      }
      HG_CUDA(cudaStreamSynchronize(c->stream));
      health_check(c);
      double d = dt_cap;
      for (int e = 0; e < c->n_el; ++e) {
        const double* v = &em[c->el_part[e]][4 * size_t(c->el_local[e])];
        c->save_umax = element_running(c->save_umax, v);
        c->save_amax = element_running(c->save_amax, v + 2);
        d = run_min(d, c->mach * std::sqrt(c->gamma) * cfl * c->dx[e] / (c->save_umax + c->save_amax) / (c->el_N[e] + 1));
      }
      *dt = d;
      return 0;
    }
    timed(c, HG_KERNEL_SPEED, [&] {
      element_speed_kernel<<<(c->n_el + threads - 1) / threads, threads, 0, c->stream>>>(
          c->n_el, c->P, c->d_Q, c->gamma, c->gamma - 1.0, c->d_elmax);
    });
    ++c->launches;
    HG_CUDA(cudaGetLastError());
    std::vector<double> em(size_t(c->n_el) * 4);
    HG_CUDA(cudaMemcpyAsync(em.data(), c->d_elmax, em.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HG_CUDA(cudaStreamSynchronize(c->stream));
    health_check(c);
    // running maxima over elements in mesh order, kept across calls
    double d = dt_cap;
    for (int e = 0; e < c->n_el; ++e) {
      c->save_umax = element_running(c->save_umax, &em[4 * size_t(e)]);
      c->save_amax = element_running(c->save_amax, &em[4 * size_t(e) + 2]);
      d = run_min(d, c->mach * std::sqrt(c->gamma) * cfl * c->dx[e] / (c->save_umax + c->save_amax) / (c->N + 1));
    }
    *dt = d;
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_set_stream(hg_ctx* c, void* s) {
  try {
    HG_CUDA(cudaStreamSynchronize(c->stream));
    if (c->own_stream) HG_CUDA(cudaStreamDestroy(c->stream));
    c->own_stream = false;
    c->stream = static_cast<cudaStream_t>(s);
    for (hg_ctx* p : c->parts) p->stream = c->stream;
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_synchronize(hg_ctx* c) {
  try {
    HG_CUDA(cudaStreamSynchronize(c->stream));
    HG_CUDA(cudaGetLastError());
    health_check(c);
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_set_health_policy(hg_ctx* c, int32_t fatal_bits) {
  try {
    if (!c) return 1;
    if (fatal_bits & ~(HEALTH_NONFINITE | HEALTH_DENSITY | HEALTH_PRESSURE))
      throw std::runtime_error("unknown health bits");
    c->health_fatal = fatal_bits;
    for (hg_ctx* p : c->parts) p->health_fatal = fatal_bits;
    *reinterpret_cast<volatile int*>(c->h_health) = 1;   // re-examine the word under the new policy
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_health(hg_ctx* c, int32_t* bits, int32_t* element) {
  try {
    if (!c) return 1;
    HG_CUDA(cudaStreamSynchronize(c->stream));
    int w[2] = {0, -1};
    HG_CUDA(cudaMemcpy(w, c->d_health, sizeof(w), cudaMemcpyDeviceToHost));
    if (bits) *bits = w[0];
    if (element) *element = w[1];
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_profile(hg_ctx* c, int32_t enable) {
  try {
    prof_collect(c);
    if (enable) {
      for (int k = 0; k < HG_KERNEL_KINDS; ++k) { c->prof_ms[k] = 0.0; c->prof_n[k] = 0; }
    }
    c->prof = enable != 0;
    for (hg_ctx* p : c->parts) HG_PART(hg_profile(p, enable), p);
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_kernel_times(hg_ctx* c, double* ms, int64_t* launches, int32_t n) {
  try {
    prof_collect(c);
    for (hg_ctx* p : c->parts) prof_collect(p);
    for (int k = 0; k < n && k < HG_KERNEL_KINDS; ++k) {
      double t = c->prof_ms[k];
      int64_t m = c->prof_n[k];
      for (hg_ctx* p : c->parts) { t += p->prof_ms[k]; m += p->prof_n[k]; }
      if (ms) ms[k] = t;
      if (launches) launches[k] = m;
    }
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_set_sensor(hg_ctx* c, int32_t kind, double s0, double kappa, const float* mlp, const float* lo,
                             const float* hi) {
  try {
    if (is_composite(c)) throw std::runtime_error("shock sensors need a single-order mesh");
    if (kind < HG_SENSOR_JUMPS || kind > HG_SENSOR_LEARNED) throw std::runtime_error("unknown sensor kind");
    if (kind == HG_SENSOR_LEARNED && !mlp) throw std::runtime_error("the learned sensor needs its weights");
    if ((lo == nullptr) != (hi == nullptr)) throw std::runtime_error("feature box needs both bounds");
    HG_CUDA(cudaStreamSynchronize(c->stream));
    if (!std::isnan(s0)) c->sensor_s0 = s0;
    if (!std::isnan(kappa)) {
      if (!(kappa > 0.0)) throw std::runtime_error("sensor ramp half width must be positive");
      c->sensor_kappa = kappa;
    }
    auto put = [](float*& d, const float* h, size_t n) {
      if (!h) { if (d) { cudaFree(d); d = nullptr; } return; }
      if (!d) d = dalloc<float>(n);
      HG_CUDA(cudaMemcpy(d, h, n * sizeof(float), cudaMemcpyHostToDevice));
    };
    drop_graph(c);
    // the device keeps the weights with the hidden unit fastest (W1^T, W2^T), the order in which the
    // kernels' lanes read them; the caller's layout is the row-major one of hg_mlp_*
    std::vector<float> wt;
    if (mlp) {
      wt.assign(mlp, mlp + HG_MLP_PARAMS);
      for (int o = 0; o < MLP_H; ++o) {
        for (int q = 0; q < MLP_IN; ++q) wt[MLP_W1 + q * MLP_H + o] = mlp[MLP_W1 + o * MLP_IN + q];
        for (int q = 0; q < MLP_H; ++q) wt[MLP_W2 + q * MLP_H + o] = mlp[MLP_W2 + o * MLP_H + q];
      }
    }
    put(c->d_mlp, mlp ? wt.data() : nullptr, HG_MLP_PARAMS);
    put(c->d_feat_lo, lo, HG_SENSOR_FEATURES);
    put(c->d_feat_hi, hi, HG_SENSOR_FEATURES);
    c->sensor_kind = kind;
    ns_prologue(c);   // the fused path keeps the indicator of the resident state
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

template <int P, typename real>
static void sensor_eval_dispatch(hg_ctx* c, float* f, double* o) { launch_sensor_eval_P<P, real>(c, f, o); }

extern "C" int hg_sensor_eval(hg_ctx* c, float* features, double* out) {
  try {
    if (is_composite(c)) throw std::runtime_error("shock sensors need a single-order mesh");
    require_state(c);
    float* df = features ? dalloc<float>(size_t(c->n_el) * HG_SENSOR_FEATURES) : nullptr;
    double* dout = out ? dalloc<double>(size_t(c->n_el) * 4) : nullptr;
    try {
      if (c->precision == HG_PREC_FP32) {
        using real = float;
        HG_DISPATCH_P(c->P, sensor_eval_dispatch, c, df, dout);
      } else {
        using real = double;
        HG_DISPATCH_P(c->P, sensor_eval_dispatch, c, df, dout);
      }
      HG_CUDA(cudaGetLastError());
      if (df) HG_CUDA(cudaMemcpyAsync(features, df, size_t(c->n_el) * HG_SENSOR_FEATURES * sizeof(float),
                                      cudaMemcpyDeviceToHost, c->stream));
      if (dout) HG_CUDA(cudaMemcpyAsync(out, dout, size_t(c->n_el) * 4 * sizeof(double), cudaMemcpyDeviceToHost,
                                        c->stream));
      HG_CUDA(cudaStreamSynchronize(c->stream));
    } catch (...) {
      if (df) cudaFree(df);
      if (dout) cudaFree(dout);
      throw;
    }
    if (df) cudaFree(df);
    if (dout) cudaFree(dout);
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_element_viscosity(hg_ctx* c, double* mu) {
  try {
    if (is_composite(c)) {   // each part's elements, back in mesh order
      if (c->av == HG_AV_NONE) throw std::runtime_error("artificial dissipation is off for this context");
      std::vector<std::vector<double>> pm(c->parts.size());
      for (size_t p = 0; p < c->parts.size(); ++p) {
        hg_ctx* q = c->parts[p];
        pm[p].resize(size_t(q->n_el));
        HG_CUDA(cudaMemcpyAsync(pm[p].data(), q->d_mu_av[q->mu_last], pm[p].size() * sizeof(double),
                                cudaMemcpyDeviceToHost, c->stream));
      }
      HG_CUDA(cudaStreamSynchronize(c->stream));
      for (int e = 0; e < c->n_el; ++e) mu[e] = pm[c->el_part[e]][c->el_local[e]];
      return 0;
    }
    if (!c->d_mu_av[0]) throw std::runtime_error("artificial dissipation is off for this context");
    HG_CUDA(cudaMemcpyAsync(mu, c->d_mu_av[c->mu_last], size_t(c->n_el) * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    HG_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_set_boundary_state(hg_ctx* c, int32_t zone, const double* uB, int64_t n_values) {
  try {
    if (is_composite(c)) {
      if (zone < 1 || zone > int(c->zone_type.size()) || c->zone_type[zone - 1] < 0)
        throw std::runtime_error("unknown zone " + std::to_string(zone));
      const std::vector<int>& ep = c->zone_edge_part[zone - 1];
      int64_t expect = 0;
      for (int p : ep) expect += int64_t(c->parts[p]->P) * 4;
      if (!uB || n_values != expect)
        throw std::runtime_error("zone " + std::to_string(zone) + " takes " + std::to_string(expect) + " values");
      // the zone's edges in mesh order, each with its part's nodes: split into the parts' own lists
      std::vector<std::vector<double>> buf(c->parts.size());
      int64_t at = 0;
      for (int p : ep) {
        const int64_t n = int64_t(c->parts[p]->P) * 4;
        buf[p].insert(buf[p].end(), uB + at, uB + at + n);
        at += n;
      }
      for (size_t p = 0; p < c->parts.size(); ++p)
        if (!buf[p].empty()) HG_PART(hg_set_boundary_state(c->parts[p], zone, buf[p].data(), int64_t(buf[p].size())), c->parts[p]);
      drop_graph(c);
      return 0;
    }
    if (zone < 1 || zone > int(c->zone_type.size()) || c->zone_type[zone - 1] < 0)
      throw std::runtime_error("unknown zone " + std::to_string(zone));
    const int z = zone - 1;
    if (c->zone_type[z] != HG_BC_DIRICHLET)
      throw std::runtime_error("per-node boundary states apply to Dirichlet zones only");
    const std::vector<int>& sides = c->zone_sides[z];
    const int64_t expect = int64_t(sides.size()) * c->P * 4;
    if (!uB || n_values != expect)
      throw std::runtime_error("zone " + std::to_string(zone) + " takes " + std::to_string(expect) + " values");
    HG_CUDA(cudaStreamSynchronize(c->stream));
    if (c->zone_row0[z] < 0) {
      // first call for this zone: give its sides consecutive rows and grow the state buffer
      const int row0 = c->n_bq_rows, rows = row0 + int(sides.size());
      double* nb = dalloc<double>(size_t(rows) * c->P * 4);
      if (c->d_bq) {
        HG_CUDA(cudaMemcpy(nb, c->d_bq, size_t(row0) * c->P * 4 * sizeof(double), cudaMemcpyDeviceToDevice));
        HG_CUDA(cudaFree(c->d_bq));
      }
      c->d_bq = nb;
      c->n_bq_rows = rows;
      c->zone_row0[z] = row0;
      for (size_t k = 0; k < sides.size(); ++k) c->h_side[sides[k]].w = row0 + int(k);
      HG_CUDA(cudaMemcpy(c->d_side, c->h_side.data(), c->h_side.size() * sizeof(int4), cudaMemcpyHostToDevice));
      drop_graph(c);   // captured launches hold the old buffer
    }
    HG_CUDA(cudaMemcpyAsync(c->d_bq + size_t(c->zone_row0[z]) * c->P * 4, uB, size_t(expect) * sizeof(double),
                            cudaMemcpyHostToDevice, c->stream));
    HG_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

// ------------------------------------------------------------------ surface integrals
extern "C" int hg_surface_integrals(hg_ctx* c, int32_t zone, double out[8]) {
  try {
    if (is_composite(c)) {
      require_state(c);
      if (!out) throw std::runtime_error("null output");
      for (int k = 0; k < 8; ++k) out[k] = 0.0;
      for (hg_ctx* p : c->parts) {
        double o[8];
        HG_PART(hg_surface_integrals(p, zone, o), p);
        for (int k = 0; k < 8; ++k) out[k] += o[k];
      }
      return 0;
    }
    require_state(c);
    if (!out) throw std::runtime_error("null output");
    if (zone < 1 || zone > int(c->zone_type.size()) || c->zone_type[zone - 1] < 0)
      throw std::runtime_error("unknown zone " + std::to_string(zone));
    const int z = zone - 1;
    if (c->d_zone_sides.size() < c->zone_sides.size()) c->d_zone_sides.resize(c->zone_sides.size(), nullptr);
    const std::vector<int>& sides = c->zone_sides[z];
    if (sides.empty()) {
      for (int k = 0; k < 8; ++k) out[k] = 0.0;
      return 0;
    }
    if (!c->d_zone_sides[z]) {
      c->d_zone_sides[z] = dalloc<int>(sides.size());
      HG_CUDA(cudaMemcpy(c->d_zone_sides[z], sides.data(), sides.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    if (!c->d_si_out) c->d_si_out = dalloc<double>(8);
    if (c->precision == HG_PREC_FP32) launch_surface_integrals<float>(c, zone, c->d_si_out);
    else launch_surface_integrals<double>(c, zone, c->d_si_out);
    HG_CUDA(cudaGetLastError());
    HG_CUDA(cudaMemcpyAsync(out, c->d_si_out, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HG_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_probes(hg_ctx* c, int32_t n, const int32_t* elements, const double* xi_eta, double* out) {
  int* d_el = nullptr;
  double* d_x = nullptr;
  double* d_o = nullptr;
  try {
    if (is_composite(c)) {
      require_state(c);
      if (n < 0 || (n > 0 && (!elements || !xi_eta || !out))) throw std::runtime_error("bad probe arguments");
      for (int k = 0; k < n; ++k)
        if (elements[k] < 0 || elements[k] >= c->n_el) throw std::runtime_error("probe element out of range");
      for (size_t pi = 0; pi < c->parts.size(); ++pi) {
        std::vector<int32_t> idx, le;
        std::vector<double> xe;
        for (int k = 0; k < n; ++k)
          if (c->el_part[elements[k]] == int(pi)) {
            idx.push_back(k);
            le.push_back(c->el_local[elements[k]]);
            xe.push_back(xi_eta[2 * k]);
            xe.push_back(xi_eta[2 * k + 1]);
          }
        if (idx.empty()) continue;
        std::vector<double> o(idx.size() * 4);
        HG_PART(hg_probes(c->parts[pi], int32_t(idx.size()), le.data(), xe.data(), o.data()), c->parts[pi]);
        for (size_t k = 0; k < idx.size(); ++k)
          for (int q = 0; q < 4; ++q) out[4 * size_t(idx[k]) + q] = o[4 * k + q];
      }
      return 0;
    }
    require_state(c);
    if (n < 0 || (n > 0 && (!elements || !xi_eta || !out))) throw std::runtime_error("bad probe arguments");
    for (int k = 0; k < n; ++k) {
      if (elements[k] < 0 || elements[k] >= c->n_el) throw std::runtime_error("probe element out of range");
      for (int d = 0; d < 2; ++d)
        if (!(xi_eta[2 * k + d] >= 0.0 && xi_eta[2 * k + d] <= 1.0))
          throw std::runtime_error("probe reference coordinates must lie in [0,1]");
    }
    if (n == 0) return 0;
    d_el = dalloc<int>(n);
    d_x = dalloc<double>(size_t(n) * 2);
    d_o = dalloc<double>(size_t(n) * 4);
    HG_CUDA(cudaMemcpyAsync(d_el, elements, size_t(n) * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    HG_CUDA(cudaMemcpyAsync(d_x, xi_eta, size_t(n) * 2 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    launch_probes(c, n, d_el, d_x, d_o);
    HG_CUDA(cudaGetLastError());
    HG_CUDA(cudaMemcpyAsync(out, d_o, size_t(n) * 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HG_CUDA(cudaStreamSynchronize(c->stream));
    cudaFree(d_el);
    cudaFree(d_x);
    cudaFree(d_o);
    return 0;
  } catch (const std::exception& ex) {
    if (d_el) cudaFree(d_el);
    if (d_x) cudaFree(d_x);
    if (d_o) cudaFree(d_o);
    return fail(c, ex);
  }
}

// ------------------------------------------------------------------ context groups
// Independent contexts (an ensemble packed by polynomial order, one context per order) stepped by
// one CUDA graph: each member's launches are captured on a stream of its own, forked from and joined
// back to the members' common stream, so the members' kernels run concurrently and one graph launch
// advances all of them by two steps.
struct hg_group {
  std::vector<hg_ctx*> m;
  std::vector<cudaStream_t> fork;
  std::vector<cudaEvent_t> join;
  cudaEvent_t start = nullptr;
  // one graph per trace-buffer parity of the first member; the members' parities relative to it and
  // their set-up generations must match the capture
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  int scheme = -1;
  double dt = 0.0;
  std::vector<int> rel;
  std::vector<int64_t> gen, per_launches[2];
  std::string err;
};

static void group_drop(hg_group* g) {
  for (auto& x : g->exec) {
    if (x) cudaGraphExecDestroy(x);
    x = nullptr;
  }
}

static void group_free(hg_group* g) {
  group_drop(g);
  for (cudaStream_t s : g->fork) if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : g->join) if (e) cudaEventDestroy(e);
  if (g->start) cudaEventDestroy(g->start);
}

extern "C" int hg_group_create(hg_ctx* const* ctxs, int32_t n, hg_group** out) {
  if (!out) return 1;
  *out = nullptr;
  hg_group* g = new hg_group();
  try {
    if (!ctxs || n < 1) throw std::runtime_error("a group needs at least one context");
    for (int i = 0; i < n; ++i) {
      if (!ctxs[i]) throw std::runtime_error("null context in group");
      if (is_composite(ctxs[i])) throw std::runtime_error("a mixed-order context cannot join a group");
      if (ctxs[i]->stream != ctxs[0]->stream) throw std::runtime_error("group members must share one stream");
      for (int j = 0; j < i; ++j) if (ctxs[j] == ctxs[i]) throw std::runtime_error("context listed twice");
      g->m.push_back(ctxs[i]);
    }
    g->fork.assign(n, nullptr);
    g->join.assign(n, nullptr);
    for (int i = 0; i < n; ++i) {
      HG_CUDA(cudaStreamCreateWithFlags(&g->fork[i], cudaStreamNonBlocking));
      HG_CUDA(cudaEventCreateWithFlags(&g->join[i], cudaEventDisableTiming));
    }
    HG_CUDA(cudaEventCreateWithFlags(&g->start, cudaEventDisableTiming));
  } catch (const std::exception& ex) {
    g_create_err = ex.what();
    group_free(g);
    delete g;
    return 1;
  }
  *out = g;
  return 0;
}

extern "C" void hg_group_destroy(hg_group* g) {
  if (!g) return;
  group_free(g);
  delete g;
}

extern "C" const char* hg_group_last_error(const hg_group* g) { return g ? g->err.c_str() : g_create_err.c_str(); }

extern "C" int hg_group_time_steps(hg_group* g, int32_t scheme, int32_t n_steps, double t0, double dt) {
  if (!g) return 1;
  const size_t n = g->m.size();
  std::vector<cudaStream_t> own(n);
  for (size_t i = 0; i < n; ++i) own[i] = g->m[i]->stream;
  try {
    for (hg_ctx* c : g->m) {
      require_state(c);
      if (c->prof) throw std::runtime_error("group stepping with kernel timing on: step the members instead");
      if (c->stream != g->m[0]->stream) throw std::runtime_error("group members must share one stream");
    }
    cudaStream_t main = g->m[0]->stream;
    int s = 0;
    if (n_steps >= 3) {
      bool valid = g->scheme == scheme && g->dt == dt && g->rel.size() == n;
      for (size_t i = 0; valid && i < n; ++i)
        valid = g->rel[i] == (g->m[i]->cur ^ g->m[0]->cur) && g->gen[i] == g->m[i]->gen;
      if (!valid) {
        group_drop(g);
        g->rel.assign(n, 0);
        g->gen.assign(n, 0);
        for (size_t i = 0; i < n; ++i) { g->rel[i] = g->m[i]->cur ^ g->m[0]->cur; g->gen[i] = g->m[i]->gen; }
        g->scheme = scheme;
        g->dt = dt;
      }
      if (!g->exec[g->m[0]->cur]) {
        for (hg_ctx* c : g->m) one_step(c, scheme, t0, dt);   // kernel attributes are set outside any capture
        ++s;
      }
      const int p = g->m[0]->cur;
      if (!g->exec[p]) {
        std::vector<int> cur0(n);
        std::vector<int64_t> l0(n);
        for (size_t i = 0; i < n; ++i) { cur0[i] = g->m[i]->cur; l0[i] = g->m[i]->launches; }
        HG_CUDA(cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal));
        try {
          HG_CUDA(cudaEventRecord(g->start, main));
          for (size_t i = 0; i < n; ++i) {
            HG_CUDA(cudaStreamWaitEvent(g->fork[i], g->start, 0));
            g->m[i]->stream = g->fork[i];
            one_step(g->m[i], scheme, t0, dt);
            one_step(g->m[i], scheme, t0, dt);
            g->m[i]->stream = own[i];
            HG_CUDA(cudaEventRecord(g->join[i], g->fork[i]));
            HG_CUDA(cudaStreamWaitEvent(main, g->join[i], 0));
          }
        } catch (...) {
          for (size_t i = 0; i < n; ++i) { g->m[i]->stream = own[i]; g->m[i]->cur = cur0[i]; g->m[i]->launches = l0[i]; }
          cudaGraph_t g0 = nullptr;
          cudaStreamEndCapture(main, &g0);
          if (g0) cudaGraphDestroy(g0);
          throw;
        }
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(main, &graph);
        g->per_launches[p].assign(n, 0);
        for (size_t i = 0; i < n; ++i) {
          g->per_launches[p][i] = g->m[i]->launches - l0[i];
          g->m[i]->launches = l0[i];
          g->m[i]->cur = cur0[i];
        }
        HG_CUDA(ce);
        const cudaError_t ie = cudaGraphInstantiate(&g->exec[p], graph, 0);
        cudaGraphDestroy(graph);
        HG_CUDA(ie);
      }
      for (; s + 2 <= n_steps; s += 2) {
        HG_CUDA(cudaGraphLaunch(g->exec[p], main));
        for (size_t i = 0; i < n; ++i) g->m[i]->launches += g->per_launches[p][i];
      }
    }
    for (; s < n_steps; ++s)
      for (hg_ctx* c : g->m) one_step(c, scheme, t0 + s * dt, dt);
    HG_CUDA(cudaGetLastError());
    return 0;
  } catch (const std::exception& ex) {
    for (size_t i = 0; i < n; ++i) g->m[i]->stream = own[i];
    g->err = ex.what();
    return 1;
  }
}

// ------------------------------------------------------------------ elements-per-CTA autotuner
extern "C" int hg_set_tiling(hg_ctx* c, int32_t variant) {
  try {
    if (is_composite(c)) {
      for (hg_ctx* p : c->parts) HG_PART(hg_set_tiling(p, variant), p);
      drop_graph(c);
      c->tiling = variant;
      return 0;
    }
    if (variant < 0 || variant >= HG_TILINGS) throw std::runtime_error("unknown tiling variant");
    HG_CUDA(cudaStreamSynchronize(c->stream));
    if (variant != c->tiling) drop_graph(c);
    c->tiling = variant;
    return 0;
  } catch (const std::exception& ex) { return fail(c, ex); }
}

extern "C" int hg_get_tiling(const hg_ctx* c, int32_t out[3]) {
  if (!c || !out) return 1;
  if (is_composite(c)) return hg_get_tiling(c->parts[largest_part(c)], out);
  const int epb = epb_of(c, c->tiling);
  out[0] = c->tiling;
  out[1] = epb;
  out[2] = block_of(c->P, epb);
  return 0;
}

// A device buffer freed when it goes out of scope (cudaFree waits for the device).
struct DevMem {
  double* p = nullptr;
  DevMem() = default;
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
  ~DevMem() { if (p) cudaFree(p); }
};

extern "C" int hg_autotune(hg_ctx* c, int32_t trials, int32_t* chosen, double* ms_per_variant) {
  if (!c) return 1;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  const bool prof = c->prof;
  try {
    require_state(c);
    if (trials < 1) throw std::runtime_error("autotune needs at least one trial");
    if (is_composite(c)) {
      // each part by itself (its mortar sides read the last mortar fluxes); reported: the largest
      // part's choice and the per-variant times summed over the parts
      HG_CUDA(cudaStreamSynchronize(c->stream));
      drop_graph(c);
      double sum[HG_TILINGS] = {};
      int chosen_big = 0;
      for (size_t pi = 0; pi < c->parts.size(); ++pi) {
        hg_ctx* p = c->parts[pi];
        int32_t ch = 0;
        double ms[HG_TILINGS] = {};
        const int64_t l0 = p->launches;
        HG_PART(hg_autotune(p, trials, &ch, ms), p);
        p->launches = l0;
        for (int v = 0; v < HG_TILINGS; ++v) sum[v] += ms[v];
        if (int(pi) == largest_part(c)) chosen_big = ch;
      }
      // residual partials of the resident state through the full composite stage
      ctx_stage(c, 0.0, 0.0, 0.0, true, false, qdot_target(c), true);
      HG_CUDA(cudaStreamSynchronize(c->stream));
      if (chosen) *chosen = chosen_big;
      if (ms_per_variant)
        for (int v = 0; v < HG_TILINGS; ++v) ms_per_variant[v] = sum[v];
      return 0;
    }
    HG_CUDA(cudaStreamSynchronize(c->stream));
    drop_graph(c);
    c->prof = false;
    HG_CUDA(cudaEventCreate(&ev[0]));
    HG_CUDA(cudaEventCreate(&ev[1]));
    double best = 0.0;
    int best_v = 0;
    // Single-order contexts time whole RK3 steps with dt = 0: every stage's launches as a step runs them
    // (updates, fused epilogues, the indicator on the last stage).  Q + 0 * G keeps the values but may
    // turn a -0 into +0, so the state is saved before and put back after, with its traces and indicator
    // formed again as hg_set_state forms them.  The parts of a mixed-order mesh, which are never stepped
    // alone, time residual launches of the resident state.
    const bool steps = !c->is_part;
    DevMem saved;
    if (steps) {
      saved.p = dalloc<double>(size_t(c->ndof));
      HG_CUDA(cudaMemcpyAsync(saved.p, c->d_Q, size_t(c->ndof) * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    }
    for (int v = 0; v < HG_TILINGS; ++v) {
      c->tiling = v;
      if (steps) {
        one_step(c, HG_SCHEME_RK3, 0.0, 0.0);
      } else {
        for (int w = 0; w < 2; ++w) ctx_stage(c, 0.0, 0.0, 0.0, true, false, qdot_target(c), false);
      }
      HG_CUDA(cudaEventRecord(ev[0], c->stream));
      for (int k = 0; k < trials; ++k) {
        if (steps) one_step(c, HG_SCHEME_RK3, 0.0, 0.0);
        else ctx_stage(c, 0.0, 0.0, 0.0, true, false, qdot_target(c), false);
      }
      HG_CUDA(cudaEventRecord(ev[1], c->stream));
      HG_CUDA(cudaEventSynchronize(ev[1]));
      float ms = 0.f;
      HG_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
      const double per = double(ms) / trials;
      if (ms_per_variant) ms_per_variant[v] = per;
      if (v == 0 || per < best) { best = per; best_v = v; }
    }
    c->tiling = best_v;
    if (steps) {   // the resident state back, and what hg_set_state forms from it
      HG_CUDA(cudaMemcpyAsync(c->d_Q, saved.p, size_t(c->ndof) * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
      c->cur = 0;
      traces(c);
      ns_prologue(c);
    }
    // leave the residual partials of the resident state in the chosen layout (as hg_time_derivative)
    ctx_stage(c, 0.0, 0.0, 0.0, true, false, qdot_target(c), true);
    HG_CUDA(cudaGetLastError());
    HG_CUDA(cudaStreamSynchronize(c->stream));
    c->prof = prof;
    if (chosen) *chosen = best_v;
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    return 0;
  } catch (const std::exception& ex) {
    for (cudaEvent_t e : ev) if (e) cudaEventDestroy(e);
    c->prof = prof;
    return fail(c, ex);
  }
}

extern "C" int hg_info(const hg_ctx* c, int32_t out[4]) {
  if (!c || !out) return 1;
  out[0] = c->N; out[1] = c->n_el; out[2] = c->affine ? 1 : 0; out[3] = c->precision;
  return 0;
}

extern "C" int hg_nodes(int32_t N, int32_t node_type, double* xi, double* w) {
  try {
    NodalOps o = make_nodal_ops(N, node_type);
    for (int i = 0; i <= N; ++i) { xi[i] = o.xi[i]; w[i] = o.w[i]; }
    return 0;
  } catch (const std::exception& ex) {
    g_create_err = ex.what();
    return 1;
  }
}
