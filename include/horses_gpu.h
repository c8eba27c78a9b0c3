/*
 * horses_gpu.h -- C ABI of libhorsesgpu.so, the B200 (sm_100a) DGSEM residual
 * and low-storage Runge-Kutta time stepper that drops into HORSES2D.
 *
 * The reference computes the residual in Fortran:
 *   DGSpatial_computeTimeDerivative(mesh, time)
 *       Solver/src/Approximation/DGSpatialDiscretizationMethods.f90:94-116
 *   TimeScheme(mesh, NDOF, time, dt, Storage)   (Explicit Euler, Williamson RK3/RK5)
 *       Solver/src/Approximation/DGTimeIntegrator.f90:71-83, 263-365
 *   TimeIntegrator_EstimateTimeStep             DGTimeIntegrator.f90:462-511
 *   Mesh_ComputeResiduals                       Solver/src/Mesh/QuadMesh_Auxiliars.incf:22-38
 * A Fortran (iso_c_binding) shim replaces those bodies with calls below; the
 * driver, case files, NetCDF I/O and the problem-file plugin are unchanged.
 *
 * Conventions
 *  - Every function returns 0 on success, non-zero on error; hg_last_error()
 *    returns the message (the shim turns it into the reference's `stop`).
 *    HG_STATUS_CRASHED: the stepped state is no longer physical (see hg_health).
 *  - The state Q is the reference's flat Storage%Q (Generic/Storage.f90:31-73):
 *    element e holds 4*(N_e+1)^2 doubles at offset 4*cumP2(e), ordered
 *    Q[e][eta][xi][var] (var fastest).  hg_set_state / hg_get_state copy it
 *    between host memory and the device; between those calls Q stays resident
 *    in device memory.
 *  - One context per mesh; calls on a context are issued on its CUDA stream and
 *    are asynchronous unless they return data to the host.
 *  - There is no CPU fallback: without a usable sm_100 device hg_create fails.
 */
#ifndef HORSES_GPU_H
#define HORSES_GPU_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct hg_ctx hg_ctx;

enum { HG_NODES_LG = 1, HG_NODES_LGL = 2 };                     /* Generic/Defines.h LG, LGL */
enum { HG_RIEMANN_ROE = 0, HG_RIEMANN_HLL = 1, HG_RIEMANN_EXACT = 2, HG_RIEMANN_LXF = 3,
       HG_RIEMANN_INTERIOR = -1 };                              /* Physics/RiemannSolvers.f90; LXF is new */
enum { HG_SCHEME_EULER = 0, HG_SCHEME_RK3 = 1, HG_SCHEME_RK5 = 2 }; /* DGTimeIntegrator.f90:131-149 */
enum { HG_PREC_FP64 = 0, HG_PREC_FP32 = 1 };
/* Boundary-condition kinds, numbered as Generic/Defines.h PERIODIC_BC .. PRESSUREOUTLET_BC. */
enum { HG_BC_PERIODIC = 1, HG_BC_DIRICHLET = 2, HG_BC_EULERWALL = 3, HG_BC_VISCOUSWALL = 4,
       HG_BC_FARFIELD = 5, HG_BC_PRESSUREOUTLET = 6, HG_BC_NEWDIRICHLET = 7 };
/* Artificial dissipation (Approximation/DGArtificialDissipation.f90), jumps-based indicator. */
enum { HG_AV_NONE = 0, HG_AV_LAPLACIAN = 1, HG_AV_PHYSICAL = 2 };

/* Physics and discretization choices (Setup_t, PhysicsNS InitializePhysics). */
typedef struct {
  int32_t node_type;       /* HG_NODES_LG / HG_NODES_LGL */
  int32_t riemann;         /* interior inviscid Riemann solver */
  int32_t navier_stokes;   /* 0: Euler build, 1: Navier-Stokes build */
  int32_t viscous;         /* 0: BR1, 1: interior penalty */
  int32_t ip_method;       /* interior penalty: 0 SIPG, 1 NIPG, 2 IIPG (DGViscousMethods.f90:355-380) */
  double  sigma0_ip;       /* "Jumps penalty parameter" */
  double  mach, reynolds, prandtl;
  double  pressure_ref, temperature_ref, reynolds_length;
  double  gamma;           /* 1.4 for the reference's "Air" */
  double  gas_R;           /* 287.15 */
  int32_t av_type;         /* HG_AV_*: "Artificial dissipation (0/1)" + "Artificial dissipation type" */
  double  av_intensity;    /* "Artificial dissipation intensity" (Ceps, default 1) */
} hg_physics_desc;

/* One boundary zone (marker), as constructed by the reference's BC classes
 * (BoundaryConditions/DGBoundaryConditions.f90).  `state` is the zone's
 * dimensionless boundary state q (Dirichlet/Farfield/Outlet), already converted
 * by the host like DirichletBC_Construct does. */
typedef struct {
  int32_t type;            /* HG_BC_* */
  int32_t riemann;         /* zone Riemann solver, HG_RIEMANN_INTERIOR = interior one */
  double  state[4];        /* Dirichlet / Farfield / Pressure-outlet state */
  double  wall_T;          /* viscous wall temperature / reference temperature (isothermal walls) */
  double  wall_v[2];       /* viscous wall velocity, dimensionless: sqrt(gamma) * Mach * direction */
  int32_t wall_type;       /* 1 isothermal, 2 adiabatic */
  int32_t outflow_type;    /* pressure outlet: 1 reflective, 2 partially non-reflective (default) */
  int32_t nd_mode;         /* newDirichlet "Mode": 0 specify speed (default), 1 specify total pressure */
  int32_t nd_outflow_total;/* newDirichlet "Outflow pressure": 0 static (default), 1 total */
} hg_bc_desc;

/* The mesh after the reference's construction (QuadMesh_t after
 * constructFromFile + ConstructZones), flattened.  Per-node arrays follow the
 * Storage%Q node order (offset/4).  Edge arrays follow mesh%edges order with the
 * subdivided edges taken out (they are the mortar list below); an edge carries
 * N_edge+1 nodes, N_edge = max of its elements' orders (the edge's own order in the
 * reference), stored one edge after the other.
 * Mixed orders and subdivided edges (p-nonconforming projections types 3-6 and
 * SubdividedEdge_t, Mesh/QuadElement_EdgeProcedures.incf:749-1345) are supported for
 * the Euler build, and for the Navier-Stokes build (BR1 or interior penalty) without artificial
 * dissipation.  Orders: 1-12 (Euler build), 1-10 (Navier-Stokes build). */
typedef struct {
  int32_t n_elements;
  int32_t n_edges;
  const int32_t* N;             /* [n_elements] polynomial order */
  const double*  Ja;            /* [nodes][2][2]  Ja(i,j,dim,IX/IY), QuadElement_SetMappings */
  const double*  jac;           /* [nodes]        mapping jacobian */
  const double*  x;             /* [nodes][2]     node coordinates (dimensionless); may be NULL */
  const double*  volume;        /* [n_elements]   element area; may be NULL */
  const double*  vertices;      /* [n_elements][4][2] corner nodes (dimensionless), for hg_estimate_dt; may be NULL */
  const int32_t* edge_elem;     /* [n_edges][2]   LEFT, RIGHT element (0-based); RIGHT = -1 on boundaries */
  const int32_t* edge_side;     /* [n_edges][2]   edgeLocation 1..4 (EBOTTOM,ERIGHT,ETOP,ELEFT) of LEFT, RIGHT */
  const int32_t* edge_inverse;  /* [n_edges]      RIGHT (or periodic partner) traverses the edge backwards */
  const int32_t* edge_marker;   /* [n_edges]      0 interior, else boundary marker (1-based zone) */
  const double*  edge_n;        /* [n_edges][N_edge+1][2] unit normal, outward from LEFT, LEFT's node order */
  const double*  edge_dS;       /* [n_edges][N_edge+1]    surface jacobian */
  const int32_t* periodic_partner; /* [n_edges] partner boundary edge of a periodic edge, else -1 */
  const double*  edge_invh;     /* [n_edges] Area / min(volume) (interior penalty); may be NULL */
  /* Subdivided edges (SubdividedEdge_LinkWithElements, Mesh/QuadElement_EdgeProcedures.incf):
   * a LEFT element against two RIGHT elements, each covering half of the edge; LEFT runs the
   * edge forwards.  PN = max(N_LEFT, N_RIGHT_NORTH)+1 and PS = max(N_LEFT, N_RIGHT_SOUTH)+1
   * nodes on the north half (edge parameter 1/2..1) and the south half (0..1/2). */
  int32_t n_mortars;
  const int32_t* mortar_elem;   /* [n_mortars][3] LEFT, RIGHT_NORTH, RIGHT_SOUTH (0-based) */
  const int32_t* mortar_side;   /* [n_mortars][3] edgeLocation 1..4 of each */
  const int32_t* mortar_flip;   /* [n_mortars][2] RIGHT_NORTH, RIGHT_SOUTH traverse their half backwards */
  const double*  mortar_n;      /* [n_mortars][PN+PS][2] unit normals outward from LEFT (north then south) */
  const double*  mortar_dS;     /* [n_mortars][PN+PS]    surface jacobians of the halves */
  const double*  mortar_invh;   /* [n_mortars] Area / min(volume) of the three elements (interior penalty); may be NULL */
} hg_mesh_desc;

/* Create a context: uploads geometry, connectivity and boundary zones once.
 * bcs[k] describes marker k+1. */
int  hg_create(const hg_mesh_desc* mesh, const hg_physics_desc* phys, const hg_bc_desc* bcs, int32_t n_bcs,
               int32_t precision, hg_ctx** out);
void hg_destroy(hg_ctx* ctx);
const char* hg_last_error(const hg_ctx* ctx);   /* ctx may be NULL: last hg_create error */

/* Host <-> device state copies (reference layout). */
int  hg_set_state(hg_ctx* ctx, const double* Q, int64_t ndof);
int  hg_get_state(hg_ctx* ctx, double* Q, int64_t ndof);
int64_t hg_ndof(const hg_ctx* ctx);

/* == DGSpatial_computeTimeDerivative: QDot of the resident state.  QDot may be
 * NULL (result kept on the device for hg_residuals). */
int  hg_time_derivative(hg_ctx* ctx, double t, double* QDot);
/* == TimeScheme: one step of HG_SCHEME_* on the resident state. */
int  hg_time_step(hg_ctx* ctx, int32_t scheme, double t, double dt);
/* n_steps steps of constant dt starting at t0, without host synchronisation. */
int  hg_time_steps(hg_ctx* ctx, int32_t scheme, int32_t n_steps, double t0, double dt);
/* == Mesh_ComputeResiduals: max |QDot| per variable of the last stage. */
int  hg_residuals(hg_ctx* ctx, double out[4]);
/* Health of the stepped state (the reference's "The simulation has crashed", printed when Q holds a
 * NaN: DGTimeIntegrator.f90:224-233).  Every RK update on the device checks its nodes for a
 * non-finite value, rho <= 0 or p <= 0 and records HG_HEALTH_* bits and one offending element
 * (0-based).  The bits in the fatal set (hg_set_health_policy; default HG_HEALTH_NONFINITE, the
 * reference's criterion: transient nodes of negative pressure occur in its own benchmarks, e.g.
 * CylinderMach2) make hg_time_step / hg_time_steps return HG_STATUS_CRASHED, with the message in
 * hg_last_error, once the flagged step has completed: checked without a synchronisation at the start
 * of each step call (so the call after the bad step reports it), and at once by the synchronising
 * calls (hg_residuals, hg_get_state, hg_estimate_dt, hg_synchronize).  The record stays until
 * hg_set_state replaces the state.  hg_health synchronises and returns the bits (0: clean) and the
 * element (-1 when clean). */
enum { HG_STATUS_CRASHED = 2 };
enum { HG_HEALTH_NONFINITE = 1, HG_HEALTH_DENSITY = 2, HG_HEALTH_PRESSURE = 4 };
int  hg_health(hg_ctx* ctx, int32_t* bits, int32_t* element);
int  hg_set_health_policy(hg_ctx* ctx, int32_t fatal_bits);
/* == EstimateTimeStep, including the reference's running maxima (SAVE). */
int  hg_estimate_dt(hg_ctx* ctx, double cfl, double dt_cap, double* dt);

/* Dirichlet zone fed per node: the problem file's boundary-condition function
 * (BoundaryConditions/BoundaryConditionFunctionDrivers.incf, DirichletBC with a user
 * function), evaluated by the caller at the zone's edge nodes.  uB holds N+1 conservative
 * dimensionless states per edge of zone `zone` (1-based marker), edges in mesh order and
 * nodes in the edge's own order: n_values = edges x (N+1) x 4.  The states are held until
 * the next call and replace the zone's constant state in every later stage.  Other zone
 * kinds recompute their ghost state from the zone state each stage and are rejected. */
int  hg_set_boundary_state(hg_ctx* ctx, int32_t zone, const double* uB, int64_t n_values);

/* == the mesh functions of the surface monitors (Mesh/QuadMesh_Integrals.incf:67-346:
 * ScalarScalar "Surface" and "pressure", ScalarVector "pressure", VectorVector "mass-flow" and
 * "flow", TensorVector "viscous" with ComputeViscousTensor, Physics/ViscousFluxes.f90:416-461),
 * over zone `zone` (1-based marker) and the traces of the state of the last residual evaluation:
 * after hg_time_derivative the resident state, after a time step its last stage's input state,
 * as the reference's monitors (updated after TimeStep) read them.  Dimensionless, as the mesh
 * functions return them: out = {surface, pressure, pressure force x, y, viscous-tensor force
 * x, y (0 without viscosity), mass flow, volume flow}.  Lift / drag: (pressure force - sqrt(gamma)
 * M viscous force) p_ref L / (rho_ref V_ref^2 S / 2) (Monitors.f90:1130-1138). */
int  hg_surface_integrals(hg_ctx* ctx, int32_t zone, double out[8]);
/* == Probe_t update (Monitors.f90:740-830): the resident state at n probe points, each given as an
 * element (0-based) and its reference coordinates xi_eta[2k], xi_eta[2k+1] in [0,1] (the reference
 * locates them once at construction); out[n][4] = the conservative dimensionless state
 * sum_i l_xi(i) sum_j Q(i,j) l_eta(j) (BilinearForm, Generic/MatrixOperations.f90:185-209).  The
 * derived probe variables (u, v, p, Mach) and reference-value factors are the caller's. */
int  hg_probes(hg_ctx* ctx, int32_t n, const int32_t* elements, const double* xi_eta, double* out);

/* Stream control: run on the caller's stream (e.g. a framework's current stream). */
int  hg_set_stream(hg_ctx* ctx, void* cuda_stream);
int  hg_synchronize(hg_ctx* ctx);
/* Device pointer of the resident state (reference layout) for in-HBM benchmarking; NULL for a
 * mixed-order context, whose state lives in one packed array per order. */
double* hg_device_state(hg_ctx* ctx);
/* Number of kernel launches issued by this context so far. */
int64_t hg_launch_count(const hg_ctx* ctx);
/* Per-kernel device time (no reference counterpart; the reference has only its
 * whole-simulation stopwatch, DGTimeIntegrator.f90:173-242).  With timing on,
 * every launch is bracketed by a CUDA event pair on the context's stream.
 * hg_profile(ctx, 1) clears the totals and starts; hg_profile(ctx, 0) stops.
 * hg_kernel_times synchronises and returns, per HG_KERNEL_* class (first n),
 * the summed milliseconds and the launch count since timing started. */
enum { HG_KERNEL_STAGE = 0, HG_KERNEL_GRADIENT = 1, HG_KERNEL_TRACE = 2, HG_KERNEL_REDUCE = 3,
       HG_KERNEL_SPEED = 4, HG_KERNEL_FACEFLUX = 5, HG_KERNEL_MORTAR = 6,
       HG_KERNEL_KINDS = 7 };
int  hg_profile(hg_ctx* ctx, int32_t enable);
int  hg_kernel_times(hg_ctx* ctx, double* ms, int64_t* launches, int32_t n);
/* hg_residuals_noalloc -- no reference counterpart.  Per-variable max |x| (the reduction of
 * Mesh_ComputeResiduals, QuadMesh_Auxiliars.incf:22-38) of a caller-owned DEVICE array in the
 * reference layout (ndof doubles, 4 per node, 32-byte aligned), written to the HOST array out[4].
 * It allocates no device memory: partial maxima go to a fixed file-scope device scratch
 * (512 KB + 32 B), which bounds ndof to HG_NOALLOC_MAX_NDOF (= 16384 blocks x 8192 nodes x 4);
 * larger or malformed sizes are rejected before any launch.  For callers that hold a QDot (or
 * any state-shaped) array on the device and may not allocate, e.g. a monitor running inside a
 * fixed device-memory budget.  Runs on cuda_stream (NULL: legacy default stream) and
 * synchronises it, so it must not be called on a stream that is being captured.  Each call looks
 * up the scratch address on the current device (cudaGetSymbolAddress).  Calls that overlap in time
 * on one device share the scratch and race: serialise them.
 * Returns 0 ok, 1 bad argument (null, ndof <= 0, not a multiple of 4, above the limit,
 * misaligned), 2 set-up failed, 3 launch or copy failed, 4 an error from earlier work was already
 * pending on this thread (left pending; nothing launched). */
#define HG_NOALLOC_MAX_NDOF 536870912LL
int  hg_residuals_noalloc(const double* qdot, int64_t ndof, void* cuda_stream, double out[4]);
/* Shock sensor of the artificial dissipation (no reference counterpart beyond HG_SENSOR_JUMPS, the
 * reference's jumps-based indicator, DGArtificialDissipation.f90:277-338, the default).  The
 * viscosity law is always mu_e = av_intensity * sqrt(Volume)/(N+1) * G.
 *   HG_SENSOR_MODAL    G = ramp(s; s0, kappa), s = max over rho, p of log10(E_N/E) of the element's
 *                      orthonormal-Legendre modal energies (modal decay); the ramp is the reference's
 *                      sine ramp; s0 = NaN keeps log10((N+1)^-4), kappa = NaN keeps 1.
 *   HG_SENSOR_LEARNED  G = max(0, (y - 0.05) / 0.95), y the MLP's output (16 -> 32 -> 32 -> 1, tanh,
 *                      sigmoid) on HG_SENSOR_FEATURES modal features (zero below 5 % of the maximum
 *                      viscosity), or the modal G where a feature leaves [lo, hi] (fallback);
 *                      mlp = HG_MLP_PARAMS floats: W1[32][16] b1[32] W2[32][32] b2[32] W3[32] b3.
 * hg_sensor_eval: per element, the features ([n_el][16] floats, may be NULL) and {modal G, learned G
 * (-1 without weights), out-of-distribution flag, G used by the current kind (-1 for jumps)}
 * ([n_el][4] doubles, may be NULL) of the resident state.  hg_element_viscosity: mu_e of the last
 * stage ([n_el] doubles; contexts with artificial dissipation). */
enum { HG_SENSOR_JUMPS = 0, HG_SENSOR_MODAL = 1, HG_SENSOR_LEARNED = 2 };
#define HG_SENSOR_FEATURES 16
#define HG_MLP_PARAMS 1633
int  hg_set_sensor(hg_ctx* ctx, int32_t kind, double s0, double kappa, const float* mlp, const float* lo,
                   const float* hi);
int  hg_sensor_eval(hg_ctx* ctx, float* features, double* out);
int  hg_element_viscosity(hg_ctx* ctx, double* mu);
/* Learned-sensor network on the GPU (no context): batched inference y = sigmoid(MLP(X)) for n
 * samples of HG_SENSOR_FEATURES floats; the mean weighted binary cross-entropy on the logit and its
 * gradient (w may be NULL: unit weights); and Adam training (beta 0.9/0.999, eps 1e-8) over
 * `epochs` shuffled passes (seeded) in mini-batches, params updated in place, epoch_loss[epochs]
 * optional.  All arrays are host arrays.  Returns 0 ok, 1 bad argument, 3 CUDA failure. */
int  hg_mlp_forward(const float* params, const float* X, int64_t n, float* y);
int  hg_mlp_grad(const float* params, const float* X, const float* t, const float* w, int64_t n, double* loss,
                 float* grad);
int  hg_mlp_train(float* params, const float* X, const float* t, const float* w, int64_t n, int32_t epochs,
                  int32_t batch, double lr, uint64_t seed, double* epoch_loss);
/* Context groups (no reference counterpart): independent contexts -- an ensemble of cases,
 * packed into one context per polynomial order -- advanced together.  hg_group_time_steps
 * runs n_steps steps of every member; from three steps on, it captures two steps of all
 * members into one CUDA graph in which each member's launches run on a stream of their own
 * (forked from and joined back to the members' common stream), so the members' kernels
 * overlap and one graph launch advances the whole ensemble by two steps.  Members must share
 * one stream (hg_set_stream) and have their state set; kernel timing must be off.  The graph
 * is rebuilt when the scheme, dt or a member's set-up changes.  The group holds no data of
 * its own: destroying it leaves the members as they are. */
typedef struct hg_group hg_group;
int  hg_group_create(hg_ctx* const* ctxs, int32_t n, hg_group** out);
void hg_group_destroy(hg_group* group);
int  hg_group_time_steps(hg_group* group, int32_t scheme, int32_t n_steps, double t0, double dt);
const char* hg_group_last_error(const hg_group* group);   /* group may be NULL: last hg_group_create error */

/* Elements-per-CTA autotuner (no reference counterpart).  The stage kernels exist in
 * HG_TILINGS tilings: variant 0 packs several elements per CTA (fewer, larger CTAs), variant 1
 * one or two (more CTAs in flight: small meshes, the smaller buckets of an ensemble).
 * hg_autotune times `trials` RK3 steps with dt = 0 in each variant (every stage's launches,
 * fused epilogues and the indicator included, while Q + 0 * G leaves the state as it was; the
 * parts of a mixed-order mesh time residual evaluations instead) with CUDA events on the
 * context's stream, keeps the faster one (chosen, and ms per step -- per evaluation for
 * mixed-order meshes -- for each variant in ms_per_variant[HG_TILINGS], both may be NULL), and
 * leaves the residual of the resident state for hg_residuals as hg_time_derivative does; the
 * state is not changed.
 * hg_set_tiling forces a variant; hg_get_tiling: out = {variant, elements per CTA, threads
 * per CTA}.  Results are the same in every variant to rounding of the per-CTA reductions. */
#define HG_TILINGS 2
int  hg_autotune(hg_ctx* ctx, int32_t trials, int32_t* chosen, double* ms_per_variant);
int  hg_set_tiling(hg_ctx* ctx, int32_t variant);
int  hg_get_tiling(const hg_ctx* ctx, int32_t out[3]);
/* Context facts: out = {N, n_elements, affine geometry path (0/1), precision}. */
int  hg_info(const hg_ctx* ctx, int32_t out[4]);
/* Mesh-file connectivity in O(E) (host code; replaces Mesh/MeshFile.f90:254-267, 287-652:
 * computeFaces, mergeDividedFaces (twice), computeElementOfEdges, computeFaceMarkers,
 * computeCurvedEdges, whose linked-list searches make preprocessing O(E^2)).  Same lists, same
 * order and conventions as the reference; all ids 1-based as in the mesh file.
 * In:  points_of_quads[E][4], points_of_bdryedges[B][2], bdry_marker[B], curved_edges_points[C][2].
 * Out (caller-sized for `capacity` edges; 4E always suffices): n_edges;
 *   points_of_edges[F][3]: the two ends as first listed, and the middle node of a subdivided
 *     (hanging-node) edge, else 0;
 *   elements_of_edges[F][3]: LEFT, RIGHT (0 on a boundary) or, for a subdivided edge, the element
 *     holding both ends, the one holding end 1 and the middle, the one holding end 2 and the middle;
 *   edge_marker[F]: 0 interior, else the boundary marker;
 *   curved_edges[C]: the edge of each curve, curve_inverted[C]: 1 when the curve runs from the
 *     edge's second end to its first (its coordinates are then to be reversed).
 * Returns 0, or 1 with the reason in hg_mesh_last_error(). */
int  hg_mesh_connectivity(int32_t n_points, int32_t n_elements, const int32_t* points_of_quads,
                          int32_t n_bdry_edges, const int32_t* points_of_bdryedges, const int32_t* bdry_marker,
                          int32_t n_curved, const int32_t* curved_edges_points, int32_t capacity,
                          int32_t* n_edges, int32_t* points_of_edges, int32_t* elements_of_edges,
                          int32_t* edge_marker, int32_t* curved_edges, int32_t* curve_inverted);
const char* hg_mesh_last_error(void);
/* Restart files (*.HiORst), host code without a NetCDF library; they replace the reference's
 * TimeIntegrator_Autosave (Solver/src/Approximation/DGTimeIntegrator.f90:413-454, called every
 * `Autosave interval` iterations and at the end, :216-218, :247) and DGSEM_loadRestartFile
 * (Solver/src/Approximation/DGSEM_class.f90:263-291, IC "Restart").  The file is NetCDF classic
 * (CDF-1) with dimensions one=1, NDOF, N, NCONS=4, no_of_elements and variables double t(one),
 * double Q(NDOF), int iter(one), laid out as the reference writes it (files written here are
 * byte-identical to the reference's for the same values); the reader accepts any classic file
 * (CDF-1 or CDF-2) that holds t, Q and iter.  Q is Storage%Q: the state layout of hg_set_state.
 * hg_read_restart with Q == NULL only reports the sizes (*ndof).  Errors: hg_restart_last_error(). */
int  hg_write_restart(const char* path, double t, int32_t iter, const double* Q, int64_t ndof, int32_t N,
                      int32_t n_elements);
int  hg_read_restart(const char* path, double* t, int32_t* iter, double* Q, int64_t capacity, int64_t* ndof);
/* The context's resident state to a restart file, and a restart file into the context (sizes must match). */
int  hg_save_restart(hg_ctx* ctx, const char* path, double t, int32_t iter);
int  hg_load_restart(hg_ctx* ctx, const char* path, double* t, int32_t* iter);
const char* hg_restart_last_error(void);
/* The same file written while the context keeps stepping: the state (as of the launches queued so
 * far) is copied on the context's stream to pinned host memory and a host thread writes the file
 * once the copy has landed.  One write is in flight at a time (the next call, hg_restart_wait and
 * hg_destroy wait for it); hg_restart_wait reports its outcome (reason in hg_last_error). */
int  hg_save_restart_async(hg_ctx* ctx, const char* path, double t, int32_t iter);
int  hg_restart_wait(hg_ctx* ctx);
/* Interpolation nodes and weights on [0,1] used by the kernels for order N
 * (NodesAndWeightsClass.f90:251-332 computeNodesAndWeights).  xi, w: N+1 doubles. */
int  hg_nodes(int32_t N, int32_t node_type, double* xi, double* w);

#ifdef __cplusplus
}
#endif
#endif
