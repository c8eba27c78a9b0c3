/*
 * oracle_api.h -- C interface of the CPU FP64 oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain C++ restatement of the
 * HORSES2D DGSEM residual and time integrator (Fortran reference), used by
 * tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py as the
 * checker.  Nothing in the product package links or calls it.
 *
 * Conventions follow the reference:
 *   - state Q is the flat Storage%Q array (Generic/Storage.f90:31-73): element
 *     e occupies NCONS*(N_e+1)^2 doubles at offset 4*cumP2(e-1), laid out
 *     Q[e][eta][xi][var] in C order (var fastest);
 *   - mesh arrays are the .HiOMesh NetCDF variables with 1-based node ids
 *     (Mesh/MeshFile.f90:77-279).
 */
#ifndef HG_ORACLE_API_H
#define HG_ORACLE_API_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Boundary-condition kinds (Generic/Defines.h FACE_INTERIOR .. NEWDIRICHLET_BC). */
enum { OR_BC_PERIODIC = 1, OR_BC_DIRICHLET = 2, OR_BC_EULERWALL = 3, OR_BC_VISCOUSWALL = 4,
       OR_BC_FARFIELD = 5, OR_BC_PRESSUREOUTLET = 6, OR_BC_NEWDIRICHLET = 7 };
/* Riemann solvers (Physics/RiemannSolvers.f90); LXF is new (no reference). */
enum { OR_RIEMANN_ROE = 0, OR_RIEMANN_HLL = 1, OR_RIEMANN_EXACT = 2, OR_RIEMANN_LXF = 3,
       OR_RIEMANN_INTERIOR = -1 };
enum { OR_NODES_LG = 1, OR_NODES_LGL = 2 };
enum { OR_SCHEME_EULER = 0, OR_SCHEME_RK3 = 1, OR_SCHEME_RK5 = 2 };
enum { OR_VISC_BR1 = 0, OR_VISC_IP = 1 };
enum { OR_IP_SIPG = 0, OR_IP_NIPG = 1, OR_IP_IIPG = 2 };
enum { OR_AV_NONE = 0, OR_AV_LAPLACIAN = 1, OR_AV_PHYSICAL = 2 };
enum { OR_IND_JUMPS = 0, OR_IND_MODAL = 1, OR_IND_EXTERNAL = 2 };

typedef struct {
  int    type;              /* OR_BC_* */
  int    riemann;           /* per-zone solver override, OR_RIEMANN_INTERIOR = use interior one */
  int    periodic_dir;      /* 1 = x, 2 = y */
  int    connected_marker;  /* periodic partner marker (1-based) */
  double pressure;          /* Dirichlet / farfield / outlet, dimensional Pa (<=0: reference) */
  double temperature;       /* K (<=0: reference) */
  double mach;              /* (<0: case Mach) */
  double aoa_deg;           /* angle of attack, degrees */
  int    wall_type;         /* viscous wall: 1 isothermal, 2 adiabatic */
  double wall_T;            /* isothermal wall temperature, K */
  double wall_v[2];         /* wall velocity, dimensionless: sqrt(gamma) * Mach * direction */
  int    outflow_type;      /* pressure outlet: 1 reflective, 2 partially non-reflective */
  int    nd_mode;           /* newDirichlet "Mode": 0 specify speed (default), 1 specify total pressure */
  int    nd_outflow_total;  /* newDirichlet "Outflow pressure": 0 static (default), 1 total */
} or_bc;

typedef struct {
  int    nodes;             /* OR_NODES_LG / OR_NODES_LGL */
  int    riemann;           /* interior Riemann solver */
  int    navier_stokes;     /* 0: Euler build, 1: Navier-Stokes build */
  int    viscous;           /* OR_VISC_BR1 / OR_VISC_IP */
  int    ip_method;         /* OR_IP_* */
  double sigma0_ip;         /* jumps penalty parameter */
  double sigma1_ip;         /* gradient jumps penalty parameter */
  double mach, reynolds, prandtl;
  double pressure_ref, temperature_ref, reynolds_length;
  int    n_markers;
  const or_bc* bcs;         /* [n_markers], zone k+1 */
  int    av_type;           /* artificial dissipation: OR_AV_NONE / LAPLACIAN / PHYSICAL (jumps-based indicator) */
  double av_intensity;      /* "Artificial dissipation intensity" (Ceps) */
  int    av_indicator;      /* OR_IND_JUMPS (reference), OR_IND_MODAL, OR_IND_EXTERNAL (G from or_set_av_g) */
  double av_s0, av_kappa;   /* modal ramp centre and half width */
} or_case;

typedef struct {
  int n_nodes, n_elements, n_bdry_edges;
  const double* points;       /* [n_nodes][2], dimensional */
  const int*    quads;        /* [n_elements][4], 1-based */
  const int*    bdry_edges;   /* [n_bdry_edges][2], 1-based */
  const int*    bdry_marker;  /* [n_bdry_edges] */
  int n_curved, curve_np1;
  const int*    curved_edges; /* [n_curved][2], 1-based */
  const double* curve_x;      /* [n_curved][curve_np1], dimensional */
  const double* curve_y;
  const int*    poly_order;   /* [n_elements] */
} or_mesh;

void*   or_create(const or_case* c, const or_mesh* m, char* err, int errlen);
void    or_destroy(void* h);
int64_t or_ndof(void* h);
int     or_n_elements(void* h);
int     or_n_edges(void* h);
void    or_element_orders(void* h, int* N_out);
void    or_node_coords(void* h, double* X);                /* [ndof/4][2] dimensionless */
void    or_set_state(void* h, const double* Q);
void    or_get_state(void* h, double* Q);
void    or_get_qdot(void* h, double* QDot);
void    or_time_derivative(void* h, double t);
void    or_time_step(void* h, int scheme, double t, double dt);
double  or_estimate_dt(void* h, double cfl, double dt_cap);
void    or_set_minmax_nan(int mode);   /* NaN handling of the dt estimate's MAX / MIN (api.cpp) */
void    or_residuals(void* h, double out[4]);
/* Reference TimeIntegrator_Integrate (Approximation/DGTimeIntegrator.f90:159-255):
 * mode 1 transient, 0 steady.  Returns the number of iterations run. */
int     or_integrate(void* h, int scheme, int mode, double t0, double t_end, int max_iter,
                     double cfl, double dt_cap, double residual_target, double* t_out);
void    or_zone_state(void* h, int zone, double* q);  /* dimensionless state of zone (marker) 1..n */
void    or_set_av_g(void* h, const double* G);   /* per-element indicator G for OR_IND_EXTERNAL */
void    or_av_viscosity(void* h, double* mu);     /* element viscosity of the current state (after a derivative) */
void    or_set_threads(int n);             /* OpenMP threads of the calling thread's regions */
/* Physics constants resolved by InitializePhysics (Physics/PhysicsNS.f90:405-481). */
void    or_ref_values(void* h, double out[8]); /* rho, a, p, V, T, L, mu_dimless, invSqrtGammaMach */
/* Geometry export for cross-checking host-side mesh builders. */
void    or_element_geometry(void* h, double* Ja, double* jac, double* volume); /* Ja [ndof/4][2][2], jac [ndof/4], volume [E] */
int     or_edge_count_by_type(void* h, int type);
/* Flattened mesh in the layout of include/horses_gpu.h hg_mesh_desc: subdivided edges form the
 * mortar list, the other edges keep their order (renumbered).  or_export_sizes: {F edges, their
 * nodes FN, M subdivided edges, their half-edge nodes MN}.  Array sizes: N[E], Ja[nodes*4],
 * jac[nodes], x[nodes*2], volume[E], vertices[E*8], edge_elem[2F], edge_side[2F], edge_inverse[F],
 * edge_marker[F], edge_n[FN*2], edge_dS[FN], periodic_partner[F], edge_invh[F], mortar_elem[3M],
 * mortar_side[3M], mortar_flip[2M], mortar_n[MN*2], mortar_dS[MN], mortar_invh[M].  Returns 0. */
void    or_export_sizes(void* h, int out[4]);
/* Boundary states given by functions (the problem-file plugin's BoundaryConditionFunction,
 * BoundaryConditions/BoundaryConditionFunctionDrivers.incf): or_zone_edge_nodes returns the
 * number of edge nodes of a zone and (if X != NULL) their coordinates [n][2], edges in
 * mesh order; or_set_zone_state sets the zone's boundary state uB [n][4] at those nodes. */
/* Surface integrals of zone (marker) `zone` over the traces of the last residual evaluation
 * (Mesh/QuadMesh_Integrals.incf), dimensionless: out = {surface, pressure, pressure force x, y,
 * viscous-tensor force x, y, mass flow, volume flow}.  Returns 0, or -1 for an unknown zone. */
int     or_surface_integrals(void* h, int zone, double out[8]);
/* Probe (Monitors.f90:740-830): the state at reference coordinates (xi, eta) of element e (0-based). */
int     or_probe(void* h, int e, double xi, double eta, double out[4]);
int     or_zone_edge_nodes(void* h, int zone, double* X);
/* The mesh file's edge lists as computeFaces / mergeDividedFaces / computeElementOfEdges /
 * computeFaceMarkers / computeCurvedEdges leave them (1-based, list order): points[F][3] (0 when a
 * simple edge), elements[F][3] (0 unused), marker[F], curve_edge[n_curved], curve_inv[n_curved];
 * any pointer may be NULL.  Returns F. */
int     or_mesh_lists(void* h, int* points, int* elements, int* marker, int* curve_edge, int* curve_inv);
void    or_set_zone_state(void* h, int zone, const double* uB);
int     or_export_mesh(void* h, int* N, double* Ja, double* jac, double* x, double* volume, double* vertices,
                       int* edge_elem, int* edge_side, int* edge_inverse, int* edge_marker, double* edge_n,
                       double* edge_dS, int* periodic_partner, double* edge_invh, int* mortar_elem,
                       int* mortar_side, int* mortar_flip, double* mortar_n, double* mortar_dS,
                       double* mortar_invh);

#ifdef __cplusplus
}
#endif
#endif
