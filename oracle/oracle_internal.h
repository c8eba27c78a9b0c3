/*
 * oracle_internal.h -- data model of the CPU FP64 oracle (TEST INFRASTRUCTURE).
 *
 * Mirrors the reference objects it restates:
 *   NodesAndWeights_t  (Approximation/NodesAndWeightsClass.f90:28-60)
 *   QuadElement_t      (Mesh/QuadElement.f90:51-80)
 *   Edge_t and its extensions (Mesh/QuadElement.f90:95-230)
 * Index conventions: reference LEFT=2, RIGHT=1, RIGHT_NORTH=1, RIGHT_SOUTH=3
 * (Generic/Defines.h); here storage/quad slots are 0-based (ref-1), so
 * slot 0 = RIGHT / RIGHT_NORTH / ONE, slot 1 = LEFT, slot 2 = RIGHT_SOUTH.
 */
#pragma once
#include <vector>
#include <string>
#include <memory>
#include <map>
#include <cmath>
#include "oracle_api.h"

namespace orc {

constexpr int NCONS = 4;
constexpr double PI = 3.141592653589793238462643;
enum { IRHO = 0, IRHOU = 1, IRHOV = 2, IRHOE = 3 };
enum { EBOTTOM = 1, ERIGHT = 2, ETOP = 3, ELEFT = 4 };
enum { FORWARD = 1, BACKWARD = -1 };
enum { SLOT_RIGHT = 0, SLOT_LEFT = 1, SLOT_RN = 0, SLOT_RS = 2 };
enum EdgeKind { E_STRAIGHT, E_CURVED, E_SUBDIV, E_CURVED_SUBDIV, E_STRAIGHT_BDRY, E_CURVED_BDRY };
enum { WEAK_RIEMANN = 1, WEAK_PRESCRIBED = 2 };
enum { VBC_UNDEFINED = 0, VBC_DIRICHLET = 1, VBC_NEUMANN = 2, VBC_PERIODIC = 3, VBC_ADIABATIC = 4 };

struct Spectral {
  int N = 0, P = 0, nodes = 0;
  std::vector<double> xi, w, wb;
  std::vector<double> D, hatD;        // (i,l) -> [i*P+l]
  std::vector<double> lb[2], lbw[2];  // [0] = at xi=0 (reference LEFT), [1] = at xi=1 (RIGHT)
  std::vector<double> dlb[2], dlbw[2];
  std::vector<double> lj(double x) const;    // barycentric Lagrange basis at x
};

struct Physics {
  double gamma = 1.4, R = 287.15, gm1 = 0.4, gogm1 = 3.5, invgm1 = 2.5;
  double cp = 0, cv = 0;          // dimensionless (gogm1, invgm1)
  double lambda = -2.0 / 3.0;
  // reference values (_DIMENSIONLESS_TAU)
  double L = 1, T = 0, p = 0, rho = 0, a = 0, V = 0, Mach = 0, mu_ref = 0, kappa_ref = 0;
  // dimensionless
  double mu = 0, kappa = 0, Re = 0, Pr = 0, sqrtGammaMach = 0, gammaMach2 = 0, invSqrtGammaMach = 0;
};

struct Element {
  int id = 0, N = 0, P = 0;
  const Spectral* sp = nullptr;
  int nodes[4] = {0, 0, 0, 0};     // 0-based node indices
  int64_t offset = 0;              // offset in doubles into Q
  int edges[4] = {-1, -1, -1, -1}; // edge index per EBOTTOM..ELEFT (0-based position 0..3)
  int edgesDirection[4] = {0, 0, 0, 0};
  int quadPosition[4] = {0, 0, 0, 0};   // 0-based storage slot
  std::vector<double> X;   // [(j*P+i)*2+d]
  std::vector<double> Ja;  // [(j*P+i)*4 + d*2 + c]   Ja(i,j,d,c)
  std::vector<double> jac; // [j*P+i]
  double volume = 0, mu_a = 0;
  bool boundaryElement = false;
};

struct EdgeStorage {
  const Spectral* sp = nullptr;
  std::vector<double> Q;   // [i*4+v]
  std::vector<double> dQ;  // [(d*P+i)*4+v]
};

struct Edge {
  int id = 0;
  EdgeKind kind = E_STRAIGHT;
  int edgeType = 0;                 // 0 interior or boundary marker
  std::vector<int> nodes;           // 0-based node ids (2 or 3)
  int quads[3] = {-1, -1, -1};      // element index per slot
  int edgeLocation[3] = {0, 0, 0};  // EBOTTOM.. per slot
  bool inverse = false;
  bool transform[2] = {false, false};   // [slot]
  int N = 0, NLow = 0, NCurve = 0;
  const Spectral* sp = nullptr;
  std::vector<double> X;      // [d*P+p]
  std::vector<double> dX;     // [d*Pn+p] (Pn = 1 straight, P curved)
  std::vector<double> dS;     // [Pn]
  std::vector<double> n;      // [d*Pn+p]
  std::vector<double> T_forward, T_backward;  // [(N+1) x (NLow+1)], [(NLow+1) x (N+1)]
  EdgeStorage storage[3];
  double Area = 0, invh = 0, mu_a = 0;
  // boundary
  int inviscidBCType = WEAK_RIEMANN;
  int riemannOverride = OR_RIEMANN_INTERIOR;
  bool associated = false;
  std::vector<double> uB_own, FB, uSB_own, gB_own;
  const std::vector<double>* uB = nullptr;   // alias (periodic) or &uB_own
  const std::vector<double>* uSB = nullptr;
  const std::vector<double>* gB = nullptr;
  std::vector<int> viscousBCType;
  int zone = -1;
  int periodic_partner = -1;
  // mortars (SubdividedEdge_t)
  int N_N = 0, N_S = 0;
  const Spectral* spN = nullptr;
  const Spectral* spS = nullptr;
  std::vector<double> normal_N, normal_S, dS_N, dS_S;      // [d*Pm+p], [Pm]
  std::vector<double> T_LN_FWD, T_LS_FWD, T_LN_BKW, T_LS_BKW, T_RN_FWD, T_RS_FWD, T_RN_BKW, T_RS_BKW;
  bool straight_like() const { return kind == E_STRAIGHT || kind == E_SUBDIV || kind == E_STRAIGHT_BDRY; }
  bool is_bdry() const { return kind == E_STRAIGHT_BDRY || kind == E_CURVED_BDRY; }
  bool is_subdiv() const { return kind == E_SUBDIV || kind == E_CURVED_SUBDIV; }
  bool is_curved() const { return kind == E_CURVED || kind == E_CURVED_SUBDIV || kind == E_CURVED_BDRY; }
  double nx(int p) const { return straight_like() ? n[0] : n[p]; }
  double ny(int p) const { return straight_like() ? n[1] : n[P() + p]; }
  int P() const { return N + 1; }
};

struct Zone {
  int marker = 0;
  or_bc bc{};
  std::vector<int> edges;
  std::vector<double> q;   // dimensionless BC state where relevant
  bool associated = false;
};

struct Oracle {
  or_case cas{};
  std::vector<or_bc> bcs;
  Physics ph;
  std::map<int, std::unique_ptr<Spectral>> spectra;   // key N
  std::vector<double> nodeX;                          // [node][2] (mutable: hanging nodes move)
  std::vector<Element> el;
  std::vector<Edge> ed;
  std::vector<Zone> zones;                            // index = marker (0 interior)
  std::vector<double> Q, QDot, dQ, G;
  std::vector<double> av_mu;                          // element artificial viscosity of the current state
  std::vector<double> av_g_ext;                       // externally supplied indicator G (OR_IND_EXTERNAL)
  bool av_hold = false;                               // later RK stages: keep the modal / external viscosity
  // the mesh file's lists as MeshFile builds them (1-based; exported for the library's builder tests)
  std::vector<int> mf_points, mf_elements, mf_marker, mf_curve_edge, mf_curve_inv;
  int64_t ndof = 0;
  // EstimateTimeStep SAVE variables (DGTimeIntegrator.f90:471-473)
  double save_umax = 0.0, save_amax = 0.0;
  const Spectral* spectral(int N);
};

// spectral.cpp
void build_spectral(Spectral& s, int N, int nodes);
void barycentric_weights(int N, const double* x, double* w);
void interp_matrix(int N, int M, const double* oldNodes, const double* wb, const double* newNodes, double* T);
bool almost_equal(double a, double b);
void legendre_gauss(int N, double* x, double* w);
void legendre_gauss_lobatto(int N, double* x, double* w);
// mesh.cpp
void build_mesh(Oracle& o, const or_mesh& m);
// residual.cpp
void time_derivative(Oracle& o, double t);
void init_physics(Oracle& o);
void setup_zones(Oracle& o);

}  // namespace orc
