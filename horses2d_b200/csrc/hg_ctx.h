// hg_ctx.h -- the library context and the launch helpers shared by the translation units of
// libhorsesgpu.so (host API in hg_api.cu; kernel instantiations in hg_inst_*.cu, compiled in parallel).
#pragma once
#include "../../include/horses_gpu.h"
#include "hg_stage.cuh"
#include "hg_ns.cuh"

#include <cuda_runtime.h>
#include <string>
#include <vector>
#include <memory>
#include <stdexcept>

using namespace hg;

struct hg_ctx {
  std::string err;
  int n_el = 0, N = 0, P = 0, node_type = 0, precision = 0, riemann = 0;
  int64_t ndof = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  PhysConst pc{};
  double mach = 0, gamma = 1.4;
  // device buffers
  int4* d_side = nullptr;
  void* d_side_geo = nullptr;     // geometry in the context's precision (FP32 path: float)
  void* d_vol_geo = nullptr;
  double* d_mats = nullptr;
  Zone* d_zones = nullptr;
  double* d_Q = nullptr;
  void* d_G = nullptr;
  void* d_T[2] = {nullptr, nullptr};
  double* d_QDot = nullptr;
  double* d_resid = nullptr;      // per-CTA partial maxima of |QDot| of the last stage [grid][4]
  double* d_resid_out = nullptr;  // reduced maxima [4]
  double* d_elmax = nullptr;      // [n_el][4] umax, amax per element and their NaN flags
  int cur = 0;                    // which trace buffer holds the current traces
  bool affine = false;            // per-element constant metrics and per-side constant normals
  bool ns = false, ip = false, grad_faces = false;   // Navier-Stokes kernels; interior penalty; SIPG/NIPG faces
  double sigma0 = 0.0, epsilon = 0.0, temperature_ref = 273.15;
  double* d_side_invh = nullptr;  // [n_el*4] invh of each side's edge
  int av = 0;                     // artificial dissipation HG_AV_*
  double* d_av_el = nullptr;      // [n_el][2] Ceps sqrt(Volume)/(N+1), sum of edge areas
  double* d_side_area = nullptr;  // [n_el*4] Area of each side's edge
  // element artificial viscosity [n_el], a pair: the indicator for the time step that starts at trace
  // parity p lives in d_mu_av[p] (a fused interior-penalty stage writes the next step's into the other)
  double* d_mu_av[2] = {nullptr, nullptr};
  int mu_step = 0;                // buffer the stages of the current step (or a bare evaluation) read
  int mu_last = 0;                // buffer the last evaluated stage read (hg_element_viscosity)
  bool last_stage = false;        // the stage being launched is the last of its time step
  bool stepping = false;          // inside one_step (mu_step fixed for the step)
  bool prologue = false;          // the next Navier-Stokes launch is the fused path's prologue
  bool is_part = false;           // an order part of a composite context
  // shock sensor (hg_sensor.cuh): indicator kind, modal ramp, learned-sensor weights and feature box
  int sensor_kind = 0;
  double sensor_s0 = 0.0, sensor_kappa = 1.0;
  float* d_mlp = nullptr;
  float* d_feat_lo = nullptr;
  float* d_feat_hi = nullptr;
  void* d_jac = nullptr;          // [n_el][NP] J (curved meshes), context precision
  void* d_GT[2] = {nullptr, nullptr};   // gradient traces [n_el*4][P][2][4] per trace parity (as d_T)
  void* d_dQ = nullptr;           // element gradients [n_el][2][4][NP] (Navier-Stokes)
  int tiling = 0;                 // elements-per-CTA variant of the stage kernels (hg_autotune / hg_set_tiling)
  bool exact = false;             // some face uses the exact Riemann solver (globally or by zone)
  void* d_FX = nullptr;           // its face fluxes of the current stage [n_el*4][P][4], context precision
  int* d_exact_sides = nullptr;   // the element sides (e*4+s) whose face uses the exact solver
  int n_exact_sides = 0;
  void* d_NF = nullptr;           // mortar fluxes of the SIDE_FLUX sides [slots][P][4], context precision
  void* d_NFG = nullptr;          // mortar BR1 gradient face terms of the SIDE_FLUX sides [slots][P][2][4]
  void* d_NJ = nullptr;           // mortar jump sums of the SIDE_FLUX sides [slots][2] (rho, rhoE; dissipation)
  int ns_phase = 0;               // a composite's Navier-Stokes part: 0 whole stage, 1 gradient kernel, 2 stage kernel
  // Mixed orders and subdivided edges: the context is a composite of one part per polynomial order
  // (each an ordinary context over its elements, on this context's stream); the faces between parts
  // and the subdivided edges are evaluated by the mortar kernel (hg_mortar.cu) before each stage.
  std::vector<hg_ctx*> parts;
  std::vector<int> el_part, el_local, el_N;   // per mesh element: part, index in the part, order
  std::vector<int64_t> el_offset;             // per mesh element: offset of its Q in Storage%Q (doubles)
  std::vector<std::vector<int>> zone_edge_part;   // per zone: the part of each of its edges, in mesh order
  int n_mortar_faces = 0;
  void* d_mfaces = nullptr;       // MortarFace records
  void* d_mmat = nullptr;         // projection matrices, context precision
  void* d_mgeo = nullptr;         // face-node rows {nx, ny, dS}, context precision
  // zones fed per node (hg_set_boundary_state): state rows [rows][P][4] indexed by side.w
  double* d_bq = nullptr;
  int n_bq_rows = 0;
  std::vector<std::vector<int>> zone_sides;   // per zone: element sides (e*4+s) of its edges, in mesh edge order
  std::vector<int> zone_type;                 // per zone: HG_BC_*
  std::vector<int> zone_row0;                 // per zone: first state row, -1 until fed per node
  std::vector<int4> h_side;                   // host copy of the side table
  std::vector<int*> d_zone_sides;             // per zone: its sides on the device (surface integrals), lazily
  double* d_si_out = nullptr;                 // surface-integral results [8]
  int last_T = 0;                             // trace buffer of the last residual evaluation's state
  bool state_set = false;
  int64_t launches = 0;
  // health of the stepped state (check_state in hg_stage.cuh): device word {bits, element} and a mapped,
  // pinned host flag that the kernels set beside it; a composite's parts share the composite's
  int* d_health = nullptr;
  int* h_health = nullptr;        // host address of the flag (its device address is d_health_flag)
  int* d_health_flag = nullptr;
  bool health_shared = false;
  int health_fatal = 1;           // HG_HEALTH_* bits that fail the step calls (hg_set_health_policy)
  std::vector<double> dx;         // per-element min corner distance (EstimateTimeStep)
  double save_umax = 0.0, save_amax = 0.0;
  // CUDA graphs of two time steps (hg_time_steps), one per trace-buffer parity at their start (a
  // step flips the parity once per stage): valid for one scheme and dt
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  int g_scheme = -1;
  int64_t gen = 0;                // bumped whenever captured launches go stale (context groups check it)
  double g_dt = 0.0;
  int64_t g_launches[2] = {0, 0};
  // CUDA graphs of one time step (hg_time_step), per parity at its start: captured the second time a
  // step of the same scheme and dt starts at that parity.
  // Rule for every graph above and below: a captured launch holds its kernel arguments and device
  // pointers by value, so any call that changes a kernel argument or replaces a device buffer must call
  // drop_graph (hg_api.cu); a call that only rewrites the contents of an existing buffer need not (the
  // replay reads the buffer then).  The step time t enters no kernel.
  cudaGraphExec_t gexec1[2] = {nullptr, nullptr};
  int g1_scheme = -1;
  double g1_dt = 0.0;
  int64_t g1_launches[2] = {0, 0};
  int g1_seen[2] = {0, 0};
  int g1_last_T[2] = {0, 0};
  // asynchronous restart files (hg_save_restart_async): pinned copy of the state, written by a host thread
  std::shared_ptr<struct AutosaveJob> autosave;
  // per-kernel timing (hg_profile): event pairs recorded around each launch
  bool prof = false;
  std::vector<cudaEvent_t> prof_pool;
  size_t prof_used = 0;
  std::vector<int> prof_kind;
  double prof_ms[HG_KERNEL_KINDS] = {};
  int64_t prof_n[HG_KERNEL_KINDS] = {};
};

#define HG_CUDA(call)                                                                           \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ------------------------------------------------------------------ per-kernel timing
inline void prof_collect(hg_ctx* c) {
  if (c->prof_used == 0) return;
  HG_CUDA(cudaStreamSynchronize(c->stream));
  for (size_t k = 0; k < c->prof_kind.size(); ++k) {
    float ms = 0.f;
    HG_CUDA(cudaEventElapsedTime(&ms, c->prof_pool[2 * k], c->prof_pool[2 * k + 1]));
    c->prof_ms[c->prof_kind[k]] += ms;
    c->prof_n[c->prof_kind[k]] += 1;
  }
  c->prof_kind.clear();
  c->prof_used = 0;
}

inline cudaEvent_t prof_event(hg_ctx* c) {
  if (c->prof_used == c->prof_pool.size()) {
    cudaEvent_t e;
    HG_CUDA(cudaEventCreate(&e));
    c->prof_pool.push_back(e);
  }
  return c->prof_pool[c->prof_used++];
}

// Launch f() on the context's stream; with timing on, bracket it by an event pair of kernel class `kind`.
template <class F>
inline void timed(hg_ctx* c, int kind, F&& f) {
  if (!c->prof) { f(); return; }
  if (c->prof_used >= 8192) prof_collect(c);
  cudaEvent_t a = prof_event(c), b = prof_event(c);
  HG_CUDA(cudaEventRecord(a, c->stream));
  f();
  HG_CUDA(cudaEventRecord(b, c->stream));
  c->prof_kind.push_back(kind);
}

// Prefer the largest shared-memory carve-out for a kernel (once per instantiation): the stage
// kernels are latency-bound and their resident CTAs per SM are capped by shared memory otherwise.
template <typename K>
inline void max_carveout(K kernel) {
  HG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                               int(cudaSharedmemCarveoutMaxShared)));
}

// Shared between hg_api.cu, hg_mortar.cu and hg_autosave.cu.
void autosave_finish(hg_ctx* c);   // waits for an asynchronous restart write (hg_destroy calls it)
void ctx_build(hg_ctx* c, const hg_mesh_desc* m, const hg_physics_desc* ph, const hg_bc_desc* bcs, int n_bcs,
               const std::vector<int2>* flux_sides);
void ctx_free(hg_ctx* c);
void ctx_stage(hg_ctx* c, double ca, double cb, double cc, bool first, bool update, double* qdot, bool resid);
void composite_build(hg_ctx* c, const hg_mesh_desc* m, const hg_physics_desc* ph, const hg_bc_desc* bcs, int n_bcs);
void composite_free(hg_ctx* c);
enum { MORTAR_FLUX = 0, MORTAR_GRADIENT = 1, MORTAR_FLUX_IP = 2, MORTAR_JUMPS = 3 };
void launch_mortar(hg_ctx* c, int mode);
inline bool is_composite(const hg_ctx* c) { return !c->parts.empty(); }
// Interior penalty with an element-local indicator (none, modal, learned) on a single-order context:
// one fused kernel per stage (hg_ns.cuh); the gradient kernel runs only as the prologue after the
// state or the indicator changes.
inline bool ns_fused(const hg_ctx* c) {
  return c->ns && c->ip && !c->is_part && !is_composite(c) && (c->av == HG_AV_NONE || c->sensor_kind != 0);
}
constexpr int HG_MAX_PARTS = 12;
constexpr int HG_MAX_ORDER_EULER = 12;
constexpr int HG_MAX_ORDER_NS = 10;

// Per-order launches, explicitly instantiated in hg_inst_*.cu (V = tiling variant: 0 in the plain
// units, 1 in the *_t1 units).
template <int P, typename real, int V> void launch_stage_PV(hg_ctx* c, const StageArgs<real>& a);
template <int P, typename real> void launch_trace_P(hg_ctx* c);
template <int P, typename real, int V> void launch_ns_PV(hg_ctx* c, const NSArgs<real>& a);
template <int P, typename real> void launch_sensor_eval_P(hg_ctx* c, float* feat, double* out);
template <typename real> void launch_exact_flux(hg_ctx* c);
template <typename real> void launch_surface_integrals(hg_ctx* c, int zone, double* d_out);
void launch_probes(hg_ctx* c, int n, const int* d_elements, const double* d_xi_eta, double* d_out);

inline SensorArgs sensor_args(const hg_ctx* c) {
  SensorArgs s;
  s.kind = c->sensor_kind;
  s.s0 = c->sensor_s0;
  s.kappa = c->sensor_kappa;
  s.mlp = c->d_mlp;
  s.lo = c->d_feat_lo;
  s.hi = c->d_feat_hi;
  return s;
}
