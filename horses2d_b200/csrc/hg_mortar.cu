// hg_mortar.cu -- mixed polynomial orders and subdivided edges (Euler build; Navier-Stokes with BR1).
//
// The reference couples elements of different orders through the edge's own order N_edge =
// max(N_L, N_R): the lower-order trace is interpolated to the edge nodes (T_forward), the Riemann
// flux is evaluated there, scaled by dS and L2-projected back (T_backward = M^-1 T^T M_edge)
// (projection types 3-6, Mesh/QuadElement_EdgeProcedures.incf:749-1345, selection :161-197).  A
// subdivided edge (SubdividedEdge_t, hanging node) holds one LEFT element against two RIGHT
// elements: LEFT's trace is interpolated to the nodes of each half, the fluxes of both halves are
// projected back and summed on LEFT, and each RIGHT element takes its half
// (ComputeRiemannSolver_SubdividedEdge / CurvedSubdividedEdge,
// Approximation/DGSpatialDiscretizationMethods.f90:761-1140; matrices SubdividedEdge_LinkWithElements,
// Mesh/QuadElement_EdgeProcedures.incf).
//
// B200 layout: a context over such a mesh is a composite of one ordinary context (part) per order,
// each running the per-order fused stage kernel over its own packed elements.  Element sides on a
// p-nonconforming or subdivided edge are marked SIDE_FLUX in their part: before every stage one
// launch of mortar_kernel (one warp per face) reads the parts' traces, evaluates these faces and
// writes each side's lifted flux -- projected to that element's side nodes, dS and sign applied --
// to the part's NF buffer, which the stage kernel reads in place of a Riemann evaluation.
#include "hg_ctx.h"
#include "hg_spectral.h"

#include <algorithm>
#include <cmath>
#include <map>

namespace {

// One face of the mortar kernel.  kind 0: edge between two orders (sides L, R); kind 1: subdivided
// edge (sides L, RN, RS).  Projections tf/tb: kind 0 {L, R} (-1: identity), kind 1 {LN, LS, RN, RS};
// offsets into the matrix pool, row-major [rows][cols].
struct MortarFace {
  double invh;    // interior penalty: Area / min(volume) of the face's elements
  double area;    // the edge's Area (artificial dissipation's Laplacian face term)
  int kind;
  int part[3], el[3], side[3], slot[3], P[3];
  int PE[2];      // edge nodes (kind 0), or north and south half nodes (kind 1)
  int inv;        // kind 0: RIGHT traverses the edge backwards
  int tf[4], tb[4];
  int geo[2];     // rows {nx, ny, dS} of the edge (kind 0) or of the north and south halves (kind 1)
  int wq[2];      // offsets of the edge's (halves') quadrature weights in the matrix pool (jumps)
};

template <typename real>
struct MortarArgs {
  int n;
  const MortarFace* f;
  const real* mat;
  const real* geo;
  const real* T[HG_MAX_PARTS];     // Q traces of the parts' current state
  const real* GT[HG_MAX_PARTS];    // gradient traces (Navier-Stokes)
  real* NF[HG_MAX_PARTS];          // MORTAR_FLUX output
  real* NFG[HG_MAX_PARTS];         // MORTAR_GRADIENT output
  real* NJ[HG_MAX_PARTS];          // MORTAR_JUMPS output: per side slot {rho, rhoE} jump sums of its face
  const double* mu[HG_MAX_PARTS];  // element artificial viscosity of the parts' current state
  int av;                          // artificial dissipation HG_AV_* (fluxes: edge viscosity terms)
  int mode;                        // MORTAR_FLUX, MORTAR_FLUX_IP, MORTAR_GRADIENT or MORTAR_JUMPS
  int visc;                        // fluxes: add the viscous flux (BR1 average; IP adds the penalty)
  int grad_faces;                  // MORTAR_FLUX_IP: SIPG / NIPG gradient-face terms
  double sigma0, epsilon;          // interior penalty parameter and the method's epsilon (-1, 1, 0)
  int riemann;
  PhysConst pc;
};

constexpr int MW = 4;        // faces (warps) per CTA
constexpr int MP = 16;       // node capacity of a side or half edge (orders up to 15)

// row `r` of (matrix m, or the identity) applied to the node vector src[cols][S] (first NC values)
template <int NC, int S, typename real>
__device__ __forceinline__ void project_row(const real* mat, int m, int cols, int r, const real* src, real* out) {
  if (m < 0) {
#pragma unroll
    for (int k = 0; k < NC; ++k) out[k] = src[r * S + k];
    return;
  }
  real acc[NC];
#pragma unroll
  for (int k = 0; k < NC; ++k) acc[k] = real(0);
  const real* row = mat + m + size_t(r) * cols;
  for (int l = 0; l < cols; ++l) {
    const real t = row[l];
#pragma unroll
    for (int k = 0; k < NC; ++k) acc[k] = acc[k] + t * src[l * S + k];
  }
#pragma unroll
  for (int k = 0; k < NC; ++k) out[k] = acc[k];
}

// Value at one edge node from the two sides' projected traces: MORTAR_FLUX the lifted flux
// (Fi - Fv) dS (4 values), MORTAR_GRADIENT the BR1 terms u* dS n, u* = (qL + qR)/2 (8 values),
// MORTAR_FLUX_IP the flux with the interior-penalty term -sigma0 mu N^2 invh (qL - qR) in Fv and the
// gradient-face terms of both sides, +-eps mu/2 Fv(q, (qL - qR) n) dS (4 + 8 + 8 values;
// IP_RiemannSolver / IP_GradientRiemannSolver, Approximation/DGViscous_IP.f90:120-134, 240-247).
template <int MODE, typename real>
__device__ __forceinline__ void node_value(const MortarArgs<real>& a, const Phys<real>& ph, const real* qL,
                                           const real* qR, const real* dL, const real* dR, const real* g,
                                           real penalty, real mu_ed, real area, real* out) {
  if constexpr (MODE == MORTAR_GRADIENT) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const real us = real(0.5) * (qL[k] + qR[k]);
      out[k] = us * g[2] * g[0];
      out[4 + k] = us * g[2] * g[1];
    }
  } else {
    real F[4];
    if (a.riemann == RIEMANN_EXACT) exact(ph, qL, qR, g[0], g[1], F);
    else riemann(a.riemann, ph, qL, qR, g[0], g[1], F);
    // the edge's viscosity: Physical dissipation adds the edge viscosity to mu in the viscous flux and the
    // penalty (penalty arrives with mu + mu_ed); Laplacian adds -mu_ed Area (qL - qR)
    // (DGArtificialDissipation.f90:208-249, JumpsBasedEdgeViscosity)
    const real mu = a.av == HG_AV_PHYSICAL ? real(a.pc.mu) + mu_ed : real(a.pc.mu);
    if (a.visc) {
      real FLx[4], FLy[4], FRx[4], FRy[4];
      viscous_flux(ph, qL, dL, dL + 4, FLx, FLy);
      viscous_flux(ph, qR, dR, dR + 4, FRx, FRy);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        real fv = real(0.5) * (mu * FLx[k] + mu * FRx[k]) * g[0] + real(0.5) * (mu * FLy[k] + mu * FRy[k]) * g[1];
        if (MODE == MORTAR_FLUX_IP) fv = fv - penalty * (qL[k] - qR[k]);
        F[k] = F[k] - fv;
      }
    }
    if (a.av == HG_AV_LAPLACIAN) {
#pragma unroll
      for (int k = 0; k < 4; ++k) F[k] = F[k] - (-(mu_ed * area * (qL[k] - qR[k])));
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = F[k] * g[2];
    if constexpr (MODE == MORTAR_FLUX_IP) {
#pragma unroll
      for (int k = 4; k < 20; ++k) out[k] = real(0);
      if (a.visc && a.grad_faces) {
        real fgx[4], fgy[4], Ax[4], Ay[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) { fgx[k] = (qL[k] - qR[k]) * g[0]; fgy[k] = (qL[k] - qR[k]) * g[1]; }
        const real cL = real(0.5) * real(a.epsilon) * mu, cR = -cL;
        viscous_flux(ph, qL, fgx, fgy, Ax, Ay);
#pragma unroll
        for (int k = 0; k < 4; ++k) { out[4 + k] = cL * Ax[k] * g[2]; out[8 + k] = cL * Ay[k] * g[2]; }
        viscous_flux(ph, qR, fgx, fgy, Ax, Ay);
#pragma unroll
        for (int k = 0; k < 4; ++k) { out[12 + k] = cR * Ax[k] * g[2]; out[16 + k] = cR * Ay[k] * g[2]; }
      }
    }
  }
}

template <typename real, int MODE>
__global__ void __launch_bounds__(MW * 32) mortar_kernel(MortarArgs<real> a) {
  constexpr int NC = MODE == MORTAR_GRADIENT ? 8 : (MODE == MORTAR_FLUX_IP ? 20 : (MODE == MORTAR_JUMPS ? 2 : 4));
  __shared__ real sT[MW][3][MP][4];   // Q traces of the face's element sides
  __shared__ real sG[MW][3][MP][8];   // their gradient traces (x then y), viscous fluxes only
  __shared__ real sF[MW][2][MP][NC];  // values at the edge (half) nodes
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int fi = blockIdx.x * MW + w;
  if (fi >= a.n) return;   // whole warps leave together; the kernel synchronises warps only
  const MortarFace& f = a.f[fi];
  const int ns = f.kind == 0 ? 2 : 3;
  const bool grads = MODE != MORTAR_GRADIENT && MODE != MORTAR_JUMPS && a.visc;
  for (int t = lane; t < ns * MP; t += 32) {
    const int s = t / MP, k = t % MP;
    if (k < f.P[s]) {
      const size_t row = (size_t(f.el[s]) * 4 + f.side[s]) * f.P[s] + k;
      const real* tp = a.T[f.part[s]] + row * 4;
#pragma unroll
      for (int q = 0; q < 4; ++q) sT[w][s][k][q] = tp[q];
      if (grads) {
        const real* gp = a.GT[f.part[s]] + row * 8;
#pragma unroll
        for (int q = 0; q < 8; ++q) sG[w][s][k][q] = gp[q];
      }
    }
  }
  __syncwarp();
  Phys<real> ph;
  ph.load(a.pc);
  // edge-node values: kind 0 one edge on lanes 0..PE-1; kind 1 the north half on lanes 0-15, the
  // south half on lanes 16-31
  {
    const int h = f.kind == 0 ? 0 : lane >> 4;
    const int i = f.kind == 0 ? lane : lane & 15;
    const int PE = f.PE[h];
    if (i < PE) {
      real qL[4], qR[4], dL[8], dR[8], v[NC];
      const int sR = f.kind == 0 ? 1 : 1 + h;
      const int mL = f.kind == 0 ? f.tf[0] : f.tf[h];
      const int mR = f.kind == 0 ? f.tf[1] : f.tf[2 + h];
      const int rR = (f.kind == 0 && f.inv) ? PE - 1 - i : i;
      project_row<4, 4>(a.mat, mL, f.P[0], i, &sT[w][0][0][0], qL);
      project_row<4, 4>(a.mat, mR, f.P[sR], rR, &sT[w][sR][0][0], qR);
      if (grads) {
        project_row<8, 8>(a.mat, mL, f.P[0], i, &sG[w][0][0][0], dL);
        project_row<8, 8>(a.mat, mR, f.P[sR], rR, &sG[w][sR][0][0], dR);
      }
      const real* g = a.geo + size_t(f.geo[h] + i) * 3;
      if constexpr (MODE == MORTAR_JUMPS) {
        // Edge_ComputeJumps at edge node i: w (2 (qL - qR) / (qL + qR))^2 dS for rho and rhoE
        // (Mesh/QuadElement_EdgeProcedures.incf:1348-1394; subdivided edges: each half at its own nodes)
        const real wi = a.mat[f.wq[h] + i];
        const real jr = real(2) * (qL[0] - qR[0]) / (qL[0] + qR[0]);
        const real je = real(2) * (qL[3] - qR[3]) / (qL[3] + qR[3]);
        sF[w][h][i][0] = wi * jr * jr * g[2];
        sF[w][h][i][1] = wi * je * je * g[2];
      } else {
        // the edge viscosity (JumpsBasedEdgeViscosity): the mean over the face's elements
        double mu_ed = 0.0;
        if (a.av != HG_AV_NONE) {
          const double mL = a.mu[f.part[0]][f.el[0]], m1 = a.mu[f.part[1]][f.el[1]];
          mu_ed = f.kind == 0 ? (m1 + mL) / 2.0 : ((m1 + mL) + a.mu[f.part[2]][f.el[2]]) / 3.0;
        }
        // penalty sigma0 (mu + mu_a) N^2 invh at the edge's (half edge's) order
        const double mu_p = a.pc.mu + (a.av == HG_AV_PHYSICAL ? mu_ed : 0.0);
        const real penalty = real(a.sigma0 * mu_p * double(PE - 1) * double(PE - 1) * f.invh);
        node_value<MODE>(a, ph, qL, qR, dL, dR, g, penalty, real(mu_ed), real(f.area), v);
#pragma unroll
        for (int k = 0; k < NC; ++k) sF[w][h][i][k] = v[k];
      }
    }
  }
  __syncwarp();
  if constexpr (MODE == MORTAR_JUMPS) {
    // the face's jump sums, in the edge's node order (north half, then south half): every element side
    // of the face takes the whole edge's value, as each element sums the jumps of its four edges
    if (lane == 0) {
      real sr = real(0), se = real(0);
      for (int hh = 0; hh < (f.kind == 0 ? 1 : 2); ++hh) {
        real hr = real(0), he = real(0);
        for (int i = 0; i < f.PE[hh]; ++i) { hr = hr + sF[w][hh][i][0]; he = he + sF[w][hh][i][1]; }
        sr = sr + hr;
        se = se + he;
      }
      for (int s = 0; s < ns; ++s) {
        real* jp = a.NJ[f.part[s]] + size_t(f.slot[s]) * 2;
        jp[0] = sr;
        jp[1] = se;
      }
    }
    return;
  }
  // back to the elements: LEFT + Tb F (both halves of a subdivided edge), RIGHT - Tb F in its own order;
  // MORTAR_FLUX_IP: also the gradient-face terms, LEFT's from values 4-11, RIGHT's from 12-19 (no sign)
  auto store = [&](int s, int i, const real* v, real sign) {
    if constexpr (MODE == MORTAR_FLUX_IP) {
      real* np = a.NF[f.part[s]] + (size_t(f.slot[s]) * f.P[s] + i) * 4;
#pragma unroll
      for (int k = 0; k < 4; ++k) np[k] = sign * v[k];
      real* gp = a.NFG[f.part[s]] + (size_t(f.slot[s]) * f.P[s] + i) * 8;
      const int o = s == 0 ? 4 : 12;
#pragma unroll
      for (int k = 0; k < 8; ++k) gp[k] = v[o + k];
    } else {
      real* const* outp = MODE == MORTAR_GRADIENT ? a.NFG : a.NF;
      real* np = outp[f.part[s]] + (size_t(f.slot[s]) * f.P[s] + i) * NC;
#pragma unroll
      for (int k = 0; k < NC; ++k) np[k] = sign * v[k];
    }
  };
  if (f.kind == 0) {
    const int PE = f.PE[0];
    real out[NC];
    if (lane < f.P[0]) {
      project_row<NC, NC>(a.mat, f.tb[0], PE, lane, &sF[w][0][0][0], out);
      store(0, lane, out, real(1));
    } else if (lane >= 16 && lane - 16 < f.P[1]) {
      const int j = lane - 16;
      project_row<NC, NC>(a.mat, f.tb[1], PE, f.inv ? f.P[1] - 1 - j : j, &sF[w][0][0][0], out);
      store(1, j, out, real(-1));
    }
  } else {
    const int h = lane >> 4, i = lane & 15;
    if (h == 0 && i < f.P[0]) {
      real acc[NC];
#pragma unroll
      for (int k = 0; k < NC; ++k) acc[k] = real(0);
      for (int hh = 0; hh < 2; ++hh) {
        const int cols = f.PE[hh];
        const real* row = a.mat + f.tb[hh] + size_t(i) * cols;
        for (int l = 0; l < cols; ++l) {
          const real t = row[l];
#pragma unroll
          for (int k = 0; k < NC; ++k) acc[k] = acc[k] + t * sF[w][hh][l][k];
        }
      }
      store(0, i, acc, real(1));
    } else if (h == 1) {
      for (int r = 0; r < 2; ++r) {
        if (i < f.P[1 + r]) {
          real out[NC];
          project_row<NC, NC>(a.mat, f.tb[2 + r], f.PE[r], i, &sF[w][r][0][0], out);
          store(1 + r, i, out, real(-1));
        }
      }
    }
  }
}

template <typename T>
T* dalloc_n(size_t n) {
  void* p = nullptr;
  HG_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  return static_cast<T*>(p);
}

void upload_prec(void*& dst, const std::vector<double>& src, int precision) {
  if (precision == HG_PREC_FP32) {
    std::vector<float> f(src.begin(), src.end());
    dst = dalloc_n<float>(f.size());
    HG_CUDA(cudaMemcpy(dst, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
  } else {
    dst = dalloc_n<double>(src.size());
    HG_CUDA(cudaMemcpy(dst, src.data(), src.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
}

// Matrix pool: interpolation from an element's nodes to given points (T_forward) and its L2 back
// projection with the edge quadrature (T_backward(i, l) = T_forward(l, i) w_edge(l) / w_el(i)).
struct MatPool {
  std::vector<double> v;
  int node_type = 0;
  std::map<int, NodalOps> ops;
  const NodalOps& op(int N) {
    auto it = ops.find(N);
    if (it == ops.end()) it = ops.emplace(N, make_nodal_ops(N, node_type)).first;
    return it->second;
  }
  // forward matrix [Ne+1 rows = points][Nel+1]; flip: the element's nodes run the other way
  std::vector<double> forward(int Nel, const std::vector<double>& pts, bool flip) {
    const NodalOps& e = op(Nel);
    std::vector<double> T(pts.size() * e.P);
    for (size_t r = 0; r < pts.size(); ++r) {
      const std::vector<double> l = lagrange_basis(e, pts[r]);
      for (int c = 0; c < e.P; ++c) T[r * e.P + (flip ? e.P - 1 - c : c)] = l[c];
    }
    return T;
  }
  std::vector<double> backward(int Nel, int Nedge, const std::vector<double>& Tf, bool flip) {
    const NodalOps& e = op(Nel);
    const NodalOps& g = op(Nedge);
    // unflipped forward matrix first (the flip reverses the rows of the back projection)
    std::vector<double> Tb(size_t(e.P) * g.P);
    for (int i = 0; i < e.P; ++i)
      for (int l = 0; l < g.P; ++l) {
        const int ci = flip ? e.P - 1 - i : i;   // column of Tf holding element node i
        Tb[size_t(flip ? e.P - 1 - i : i) * g.P + l] = ((1.0 / e.w[i]) * Tf[size_t(l) * e.P + ci]) * g.w[l];
      }
    return Tb;
  }
  int add(const std::vector<double>& m) {
    const int off = int(v.size());
    v.insert(v.end(), m.begin(), m.end());
    return off;
  }
};

}  // namespace

void launch_mortar(hg_ctx* c, int mode) {
  if (c->n_mortar_faces == 0) return;
  const int grid = (c->n_mortar_faces + MW - 1) / MW;
  auto go = [&](auto tag) {
    using real = decltype(tag);
    MortarArgs<real> a{};
    a.n = c->n_mortar_faces;
    a.f = static_cast<const MortarFace*>(c->d_mfaces);
    a.mat = static_cast<const real*>(c->d_mmat);
    a.geo = static_cast<const real*>(c->d_mgeo);
    for (size_t p = 0; p < c->parts.size(); ++p) {
      hg_ctx* q = c->parts[p];
      a.T[p] = static_cast<const real*>(q->d_T[q->cur]);
      a.GT[p] = static_cast<const real*>(q->d_GT[q->cur]);
      a.NF[p] = static_cast<real*>(q->d_NF);
      a.NFG[p] = static_cast<real*>(q->d_NFG);
      a.NJ[p] = static_cast<real*>(q->d_NJ);
      a.mu[p] = q->d_mu_av[q->cur];   // the parts' gradient kernels of this stage wrote it (jumps indicator)
    }
    if (mode == MORTAR_FLUX && c->ns && c->ip) mode = MORTAR_FLUX_IP;
    a.mode = mode;
    a.av = c->av;
    a.visc = c->ns && (c->pc.mu != 0.0 || c->av == HG_AV_PHYSICAL);
    a.grad_faces = c->grad_faces ? 1 : 0;
    a.sigma0 = c->sigma0;
    a.epsilon = c->epsilon;
    a.riemann = c->riemann;
    a.pc = c->pc;
    timed(c, HG_KERNEL_MORTAR, [&] {
      if (mode == MORTAR_GRADIENT) mortar_kernel<real, MORTAR_GRADIENT><<<grid, MW * 32, 0, c->stream>>>(a);
      else if (mode == MORTAR_FLUX_IP) mortar_kernel<real, MORTAR_FLUX_IP><<<grid, MW * 32, 0, c->stream>>>(a);
      else if (mode == MORTAR_JUMPS) mortar_kernel<real, MORTAR_JUMPS><<<grid, MW * 32, 0, c->stream>>>(a);
      else mortar_kernel<real, MORTAR_FLUX><<<grid, MW * 32, 0, c->stream>>>(a);
    });
  };
  if (c->precision == HG_PREC_FP32) go(float{});
  else go(double{});
  ++c->launches;
}

void composite_free(hg_ctx* c) {
  for (hg_ctx* p : c->parts) {
    ctx_free(p);
    delete p;
  }
  c->parts.clear();
  for (void* p : {c->d_mfaces, c->d_mmat, c->d_mgeo})
    if (p) cudaFree(p);
  c->d_mfaces = c->d_mmat = c->d_mgeo = nullptr;
}

void composite_build(hg_ctx* c, const hg_mesh_desc* m, const hg_physics_desc* ph, const hg_bc_desc* bcs, int n_bcs) {
  if (ph->av_type < HG_AV_NONE || ph->av_type > HG_AV_PHYSICAL) throw std::runtime_error("unknown artificial dissipation type");
  if (ph->navier_stokes && ph->av_type != HG_AV_NONE && !m->volume)
    throw std::runtime_error("artificial dissipation needs element volumes");
  const int E = m->n_elements;
  if (E <= 0) throw std::runtime_error("mesh has no elements");
  c->el_N.assign(m->N, m->N + E);
  const int max_order = ph->navier_stokes ? HG_MAX_ORDER_NS : HG_MAX_ORDER_EULER;
  for (int e = 0; e < E; ++e)
    if (c->el_N[e] < 1 || c->el_N[e] > max_order)
      throw std::runtime_error("polynomial order must be in 1.." + std::to_string(max_order) +
                               (ph->navier_stokes ? " for the Navier-Stokes build" : ""));
  // parts: one per order, ascending; elements in mesh order within a part
  std::vector<int> orders(c->el_N);
  std::sort(orders.begin(), orders.end());
  orders.erase(std::unique(orders.begin(), orders.end()), orders.end());
  if (int(orders.size()) > HG_MAX_PARTS) throw std::runtime_error("too many polynomial orders");
  const int NPART = int(orders.size());
  std::vector<int> part_of_order(HG_MAX_ORDER_EULER + 1, -1);
  for (int p = 0; p < NPART; ++p) part_of_order[orders[p]] = p;
  c->el_part.resize(E);
  c->el_local.resize(E);
  c->el_offset.resize(E);
  std::vector<int> part_n(NPART, 0);
  std::vector<std::vector<int>> part_el(NPART);
  std::vector<int64_t> node0(E);
  int64_t nodes = 0;
  for (int e = 0; e < E; ++e) {
    const int p = part_of_order[c->el_N[e]];
    c->el_part[e] = p;
    c->el_local[e] = part_n[p]++;
    part_el[p].push_back(e);
    node0[e] = nodes;
    c->el_offset[e] = nodes * 4;
    nodes += int64_t(c->el_N[e] + 1) * (c->el_N[e] + 1);
  }
  c->n_el = E;
  c->ndof = nodes * 4;
  c->N = orders.back();
  c->P = c->N + 1;
  c->node_type = ph->node_type;
  c->riemann = ph->riemann;
  c->av = ph->navier_stokes ? ph->av_type : HG_AV_NONE;
  c->ns = ph->navier_stokes != 0 && (ph->reynolds != 0.0 || c->av != HG_AV_NONE);
  c->ip = ph->viscous == 1;
  c->grad_faces = c->ip && ph->ip_method != 2;
  c->sigma0 = ph->sigma0_ip;
  c->epsilon = ph->ip_method == 0 ? -1.0 : (ph->ip_method == 1 ? 1.0 : 0.0);
  if (c->ns && c->ip && (!m->edge_invh || (m->n_mortars > 0 && !m->mortar_invh)))
    throw std::runtime_error("interior penalty needs edge_invh (and mortar_invh for subdivided edges)");  const double gamma = ph->gamma > 0 ? ph->gamma : 1.4;
  c->gamma = gamma; c->mach = ph->mach;
  c->pc.gamma = gamma;
  c->pc.gm1 = gamma - 1.0;
  c->pc.cp = gamma / (gamma - 1.0);
  c->pc.cv = 1.0 / (gamma - 1.0);
  c->pc.invSqrtGammaMach = 1.0 / (std::sqrt(gamma) * ph->mach);

  // edges: node offsets, owning part (conforming) or mortar face (two orders)
  const int F = m->n_edges;
  std::vector<int64_t> enode(F + 1, 0);
  std::vector<int> edge_part(F, -1);
  for (int f = 0; f < F; ++f) {
    const int L = m->edge_elem[2 * f], R = m->edge_elem[2 * f + 1];
    if (L < 0 || L >= E) throw std::runtime_error("bad edge connectivity");
    const bool interior = m->edge_marker[f] == 0;
    if (interior && (R < 0 || R >= E)) throw std::runtime_error("interior edge without RIGHT element");
    const int NE = interior ? std::max(c->el_N[L], c->el_N[R]) : c->el_N[L];
    enode[f + 1] = enode[f] + NE + 1;
    if (!interior || c->el_N[L] == c->el_N[R]) edge_part[f] = c->el_part[L];
  }
  // zones: the part of each zone edge, in mesh order (per-node boundary states are split by it)
  c->zone_type.assign(std::max(1, n_bcs), -1);
  for (int z = 0; z < n_bcs; ++z) c->zone_type[z] = bcs[z].type;
  c->zone_edge_part.assign(std::max(1, n_bcs), std::vector<int>());
  for (int f = 0; f < F; ++f) {
    const int mk = m->edge_marker[f];
    if (mk == 0) continue;
    if (mk < 1 || mk > n_bcs) throw std::runtime_error("boundary edge with unknown marker");
    c->zone_edge_part[mk - 1].push_back(edge_part[f]);
    if (bcs[mk - 1].type == HG_BC_PERIODIC) {
      const int q = m->periodic_partner ? m->periodic_partner[f] : -1;
      if (q < 0 || q >= F) throw std::runtime_error("periodic edge without partner");
      if (c->el_N[m->edge_elem[2 * q]] != c->el_N[m->edge_elem[2 * f]])
        throw std::runtime_error("periodic edges between different polynomial orders are not supported");
    }
  }
  // local edge numbering per part
  std::vector<int> edge_local(F, -1);
  std::vector<std::vector<int>> part_edges(NPART);
  for (int f = 0; f < F; ++f)
    if (edge_part[f] >= 0) {
      edge_local[f] = int(part_edges[edge_part[f]].size());
      part_edges[edge_part[f]].push_back(f);
    }

  // mortar faces, their projection matrices and geometry; SIDE_FLUX slots per part
  MatPool pool;
  pool.node_type = ph->node_type;
  // Area of every edge, sum_p dS(p) w(p) at the edge's order (QuadMesh_Construct.incf:270-303), and per
  // element side (the artificial dissipation's indicator and Laplacian face term)
  std::vector<double> edge_area(F, 0.0), side_area_mesh(size_t(E) * 4, 0.0);
  for (int f = 0; f < F; ++f) {
    const int NE = int(enode[f + 1] - enode[f]) - 1;
    const std::vector<double>& w = pool.op(NE).w;
    double A = 0.0;
    for (int p = 0; p <= NE; ++p) A += m->edge_dS[enode[f] + p] * w[p];
    edge_area[f] = A;
    side_area_mesh[size_t(m->edge_elem[2 * f]) * 4 + m->edge_side[2 * f] - 1] = A;
    if (m->edge_marker[f] == 0) side_area_mesh[size_t(m->edge_elem[2 * f + 1]) * 4 + m->edge_side[2 * f + 1] - 1] = A;
  }
  std::vector<double> geo;
  std::vector<MortarFace> faces;
  std::vector<std::vector<int2>> flux_sides(NPART);
  auto side_slot = [&](int e, int s) {
    const int p = c->el_part[e];
    const int slot = int(flux_sides[p].size());
    flux_sides[p].push_back(make_int2(c->el_local[e] * 4 + s, slot));
    return slot;
  };
  auto fill_side = [&](MortarFace& mf, int k, int e, int s) {
    mf.part[k] = c->el_part[e];
    mf.el[k] = c->el_local[e];
    mf.side[k] = s;
    mf.P[k] = c->el_N[e] + 1;
    mf.slot[k] = side_slot(e, s);
  };
  for (int f = 0; f < F; ++f) {
    if (edge_part[f] >= 0) continue;
    const int L = m->edge_elem[2 * f], R = m->edge_elem[2 * f + 1];
    const int sL = m->edge_side[2 * f] - 1, sR = m->edge_side[2 * f + 1] - 1;
    if (sL < 0 || sL > 3 || sR < 0 || sR > 3) throw std::runtime_error("bad edge connectivity");
    MortarFace mf{};
    mf.kind = 0;
    fill_side(mf, 0, L, sL);
    fill_side(mf, 1, R, sR);
    mf.part[2] = mf.el[2] = mf.side[2] = mf.slot[2] = mf.P[2] = 0;
    const int NE = std::max(c->el_N[L], c->el_N[R]);
    mf.PE[0] = NE + 1;
    mf.PE[1] = 0;
    mf.inv = m->edge_inverse[f] != 0;
    mf.invh = m->edge_invh ? m->edge_invh[f] : 0.0;
    for (int k = 0; k < 4; ++k) mf.tf[k] = mf.tb[k] = -1;
    const std::vector<double> xe = pool.op(NE).xi;
    for (int k = 0; k < 2; ++k) {
      const int Nk = c->el_N[k == 0 ? L : R];
      if (Nk == NE) continue;
      const std::vector<double> Tf = pool.forward(Nk, xe, false);
      mf.tf[k] = pool.add(Tf);
      mf.tb[k] = pool.add(pool.backward(Nk, NE, Tf, false));
    }
    mf.geo[0] = int(geo.size() / 3);
    mf.geo[1] = 0;
    for (int64_t n = enode[f]; n < enode[f + 1]; ++n) {
      geo.push_back(m->edge_n[2 * n]);
      geo.push_back(m->edge_n[2 * n + 1]);
      geo.push_back(m->edge_dS[n]);
    }
    mf.wq[0] = pool.add(pool.op(NE).w);
    mf.wq[1] = 0;
    mf.area = edge_area[f];
    faces.push_back(mf);
  }
  int64_t mnode = 0;
  for (int q = 0; q < m->n_mortars; ++q) {
    const int* el = m->mortar_elem + 3 * q;
    const int* sd = m->mortar_side + 3 * q;
    for (int k = 0; k < 3; ++k)
      if (el[k] < 0 || el[k] >= E || sd[k] < 1 || sd[k] > 4) throw std::runtime_error("bad subdivided-edge connectivity");
    const int NL = c->el_N[el[0]], NRN = c->el_N[el[1]], NRS = c->el_N[el[2]];
    const int NN = std::max(NL, NRN), NS = std::max(NL, NRS);
    MortarFace mf{};
    mf.kind = 1;
    for (int k = 0; k < 3; ++k) fill_side(mf, k, el[k], sd[k] - 1);
    mf.PE[0] = NN + 1;
    mf.PE[1] = NS + 1;
    mf.inv = 0;
    mf.invh = m->mortar_invh ? m->mortar_invh[q] : 0.0;
    std::vector<double> xN = pool.op(NN).xi, xS = pool.op(NS).xi;
    std::vector<double> hN(xN.size()), hS(xS.size());
    for (size_t p = 0; p < xN.size(); ++p) hN[p] = 0.5 + 0.5 * xN[p];
    for (size_t p = 0; p < xS.size(); ++p) hS[p] = 0.5 * xS[p];
    const bool flipN = m->mortar_flip[2 * q] != 0, flipS = m->mortar_flip[2 * q + 1] != 0;
    const std::vector<double> TLN = pool.forward(NL, hN, false), TLS = pool.forward(NL, hS, false);
    const std::vector<double> TRN = pool.forward(NRN, xN, flipN), TRS = pool.forward(NRS, xS, flipS);
    mf.tf[0] = pool.add(TLN);
    mf.tf[1] = pool.add(TLS);
    mf.tf[2] = pool.add(TRN);
    mf.tf[3] = pool.add(TRS);
    mf.tb[0] = pool.add(pool.backward(NL, NN, TLN, false));
    mf.tb[1] = pool.add(pool.backward(NL, NS, TLS, false));
    mf.tb[2] = pool.add(pool.backward(NRN, NN, TRN, flipN));
    mf.tb[3] = pool.add(pool.backward(NRS, NS, TRS, flipS));
    mf.geo[0] = int(geo.size() / 3);
    for (int p = 0; p < NN + 1; ++p, ++mnode) {
      geo.push_back(m->mortar_n[2 * mnode]);
      geo.push_back(m->mortar_n[2 * mnode + 1]);
      geo.push_back(m->mortar_dS[mnode]);
    }
    mf.geo[1] = int(geo.size() / 3);
    for (int p = 0; p < NS + 1; ++p, ++mnode) {
      geo.push_back(m->mortar_n[2 * mnode]);
      geo.push_back(m->mortar_n[2 * mnode + 1]);
      geo.push_back(m->mortar_dS[mnode]);
    }
    mf.wq[0] = pool.add(pool.op(NN).w);
    mf.wq[1] = pool.add(pool.op(NS).w);
    // Area of the whole edge, sum_p dS(p) w(p) at the LEFT element's order (QuadMesh_Construct.incf:
    // 270-303): a straight edge's dS is twice each half's; a curved one's is recovered from
    // invh = Area / min(volumes) (to rounding)
    {
      const double* dN = &geo[size_t(mf.geo[0]) * 3];
      const double* dSo = &geo[size_t(mf.geo[1]) * 3];
      bool straight = dN[2] == dSo[2];
      for (int p = 0; p < NN + 1 && straight; ++p) straight = dN[3 * p + 2] == dN[2];
      for (int p = 0; p < NS + 1 && straight; ++p) straight = dSo[3 * p + 2] == dN[2];
      double A = 0.0;
      if (straight) {
        const std::vector<double>& wL = pool.op(NL).w;
        for (int p = 0; p < NL + 1; ++p) A += (2.0 * dN[2]) * wL[p];
      } else if (m->volume) {
        A = mf.invh * std::min({m->volume[el[0]], m->volume[el[1]], m->volume[el[2]]});
      }
      mf.area = A;
      for (int k = 0; k < 3; ++k) side_area_mesh[size_t(el[k]) * 4 + sd[k] - 1] = A;
    }
    faces.push_back(mf);
  }
  for (const MortarFace& mf : faces)
    for (int k = 0; k < (mf.kind == 0 ? 2 : 3); ++k)
      if (mf.P[k] > MP || mf.PE[0] > MP || mf.PE[1] > MP) throw std::runtime_error("order too high for a mortar face");

  // the parts: ordinary contexts over sub-descriptors of one order
  for (int p = 0; p < NPART; ++p) {
    const int Np = orders[p], Pp = Np + 1, NPp = Pp * Pp;
    const std::vector<int>& els = part_el[p];
    const std::vector<int>& eds = part_edges[p];
    const int Ep = int(els.size()), Fp = int(eds.size());
    std::vector<int> sN(Ep, Np), eelem(2 * Fp), eside(2 * Fp), einv(Fp), emark(Fp), epart(Fp, -1);
    std::vector<double> Ja(size_t(Ep) * NPp * 4), jac(size_t(Ep) * NPp), x(size_t(Ep) * NPp * 2), vol(Ep),
        vert(size_t(Ep) * 8), en(size_t(Fp) * Pp * 2), eds_(size_t(Fp) * Pp), invh(Fp, 0.0);
    for (int k = 0; k < Ep; ++k) {
      const int e = els[k];
      const int64_t n0 = node0[e];
      std::copy(m->Ja + n0 * 4, m->Ja + (n0 + NPp) * 4, Ja.begin() + size_t(k) * NPp * 4);
      std::copy(m->jac + n0, m->jac + n0 + NPp, jac.begin() + size_t(k) * NPp);
      if (m->x) std::copy(m->x + n0 * 2, m->x + (n0 + NPp) * 2, x.begin() + size_t(k) * NPp * 2);
      vol[k] = m->volume ? m->volume[e] : 0.0;
      if (m->vertices) std::copy(m->vertices + size_t(e) * 8, m->vertices + size_t(e) * 8 + 8, vert.begin() + size_t(k) * 8);
    }
    for (int k = 0; k < Fp; ++k) {
      const int f = eds[k];
      const int L = m->edge_elem[2 * f], R = m->edge_elem[2 * f + 1];
      eelem[2 * k] = c->el_local[L];
      eelem[2 * k + 1] = (m->edge_marker[f] == 0) ? c->el_local[R] : -1;
      eside[2 * k] = m->edge_side[2 * f];
      eside[2 * k + 1] = m->edge_side[2 * f + 1];
      einv[k] = m->edge_inverse[f];
      emark[k] = m->edge_marker[f];
      if (m->periodic_partner && m->periodic_partner[f] >= 0) epart[k] = edge_local[m->periodic_partner[f]];
      if (m->edge_invh) invh[k] = m->edge_invh[f];
      for (int n = 0; n < Pp; ++n) {
        en[(size_t(k) * Pp + n) * 2] = m->edge_n[(enode[f] + n) * 2];
        en[(size_t(k) * Pp + n) * 2 + 1] = m->edge_n[(enode[f] + n) * 2 + 1];
        eds_[size_t(k) * Pp + n] = m->edge_dS[enode[f] + n];
      }
    }
    hg_mesh_desc sub{};
    sub.n_elements = Ep;
    sub.n_edges = Fp;
    sub.N = sN.data();
    sub.Ja = Ja.data();
    sub.jac = jac.data();
    sub.x = m->x ? x.data() : nullptr;
    sub.volume = m->volume ? vol.data() : nullptr;
    sub.vertices = m->vertices ? vert.data() : nullptr;
    sub.edge_elem = eelem.data();
    sub.edge_side = eside.data();
    sub.edge_inverse = einv.data();
    sub.edge_marker = emark.data();
    sub.edge_n = en.data();
    sub.edge_dS = eds_.data();
    sub.periodic_partner = epart.data();
    sub.edge_invh = m->edge_invh ? invh.data() : nullptr;
    hg_ctx* pc = new hg_ctx();
    pc->is_part = true;
    pc->precision = c->precision;
    c->parts.push_back(pc);
    ctx_build(pc, &sub, ph, bcs, n_bcs, &flux_sides[p]);
    // the part runs on the composite's stream
    HG_CUDA(cudaStreamDestroy(pc->stream));
    pc->own_stream = false;
    pc->stream = nullptr;
    const size_t rs = c->precision == HG_PREC_FP32 ? sizeof(float) : sizeof(double);
    pc->d_NF = dalloc_n<char>(flux_sides[p].size() * Pp * 4 * rs);
    HG_CUDA(cudaMemset(pc->d_NF, 0, std::max<size_t>(flux_sides[p].size() * Pp * 4 * rs, 1)));
    if (c->ns) {
      pc->d_NFG = dalloc_n<char>(flux_sides[p].size() * Pp * 8 * rs);
      HG_CUDA(cudaMemset(pc->d_NFG, 0, std::max<size_t>(flux_sides[p].size() * Pp * 8 * rs, 1)));
    }
    if (c->av != HG_AV_NONE) {
      pc->d_NJ = dalloc_n<char>(flux_sides[p].size() * 2 * rs);
      HG_CUDA(cudaMemset(pc->d_NJ, 0, std::max<size_t>(flux_sides[p].size() * 2 * rs, 1)));
      // the jumps indicator divides by the element's four edge Areas: the part built them from its own
      // (conforming) edges only, so they are replaced by the whole mesh's, edges between orders and
      // subdivided edges included (JumpsBasedElementViscosity, DGArtificialDissipation.f90:277-338)
      std::vector<double> avel(size_t(Ep) * 2), sarea(size_t(Ep) * 4);
      for (int k = 0; k < Ep; ++k) {
        const int e = els[k];
        const double* A = &side_area_mesh[size_t(e) * 4];
        avel[2 * size_t(k)] = ph->av_intensity * (std::sqrt(m->volume[e]) / (Np + 1));
        avel[2 * size_t(k) + 1] = A[0] + A[1] + A[2] + A[3];
        for (int sd_ = 0; sd_ < 4; ++sd_) sarea[size_t(k) * 4 + sd_] = A[sd_];
      }
      HG_CUDA(cudaMemcpy(pc->d_av_el, avel.data(), avel.size() * sizeof(double), cudaMemcpyHostToDevice));
      HG_CUDA(cudaMemcpy(pc->d_side_area, sarea.data(), sarea.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
  }
  // per-element corner distances of the whole mesh (EstimateTimeStep runs over mesh order)
  c->dx.assign(E, 0.0);
  if (m->vertices)
    for (int e = 0; e < E; ++e) {
      const double* v = m->vertices + size_t(e) * 8;
      auto d = [&](int a, int b) { return std::sqrt((v[2 * a] - v[2 * b]) * (v[2 * a] - v[2 * b]) + (v[2 * a + 1] - v[2 * b + 1]) * (v[2 * a + 1] - v[2 * b + 1])); };
      c->dx[e] = std::fmin(std::fmin(d(0, 1), d(1, 2)), std::fmin(d(2, 3), d(0, 3)));
    }
  c->pc = c->parts[0]->pc;   // physics constants (the parts share them)
  HG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  c->own_stream = true;
  for (hg_ctx* pc : c->parts) pc->stream = c->stream;
  c->n_mortar_faces = int(faces.size());
  c->d_mfaces = dalloc_n<MortarFace>(faces.size());
  HG_CUDA(cudaMemcpy(c->d_mfaces, faces.data(), faces.size() * sizeof(MortarFace), cudaMemcpyHostToDevice));
  upload_prec(c->d_mmat, pool.v, c->precision);
  upload_prec(c->d_mgeo, geo, c->precision);
}
