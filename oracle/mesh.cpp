/*
 * mesh.cpp -- mesh connectivity and geometry of the oracle (TEST INFRASTRUCTURE).
 *
 * Restates, in the reference's own order of operations:
 *   ReadMesh / computeFaces / mergeDividedFaces / computeElementOfEdges /
 *   computeFaceMarkers / computeCurvedEdges        Mesh/MeshFile.f90:77-339, 360-520
 *   IntegerArrayLinkedList Add/Search/SearchIfPresent/SearchIfContained/Remove
 *                                                  Foundation/IntegerArrayLinkedList.f90
 *   constructElementsAndEdges                      Mesh/QuadMesh_Construct.incf:22-265
 *   Edge_SetCurve / CurvedEdge_SetCurve / evaluateX / evaluatedX / getX / getdX /
 *   (Curved)SubdividedEdge_ConstructMortars        Mesh/QuadElement_EdgeMappings.incf
 *   Edge_LinkWithElements / SubdividedEdge_LinkWithElements / BdryEdge_LinkWithElements /
 *   Edge_Invert / mortar transformation matrices   Mesh/QuadElement_EdgeProcedures.incf:30-520
 *   searchEdge / compareEdges                      Mesh/QuadElement_Auxiliars.incf:27-117
 *   QuadElement_SetMappings                        Mesh/QuadElement_QuadMappings.incf:22-367
 *
 * The edge list is kept as an ordered vector with the linked list's semantics
 * (append at tail, keep first occurrence, remove in place); position lookups use
 * hash maps, which changes only the cost, not the order.
 */
#include "oracle_internal.h"
#include <algorithm>
#include <stdexcept>
#include <unordered_map>
#include <cstdio>

namespace orc {

namespace {

struct Entry { int N; int v[3]; bool attribute; };

struct EdgeList {
  std::vector<Entry> e;
  static uint64_t key2(int a, int b) { if (a > b) std::swap(a, b); return (uint64_t(uint32_t(a)) << 32) | uint32_t(b); }
  // IntegerArrayLinkedList_Search for 2-point arrays (1-based position or -1).
  int search2(int a, int b) const {
    for (size_t i = 0; i < e.size(); ++i) {
      if (e[i].N != 2) return -1;   // the reference scan stalls on the first entry of another size
      if ((e[i].v[0] == a && e[i].v[1] == b) || (e[i].v[0] == b && e[i].v[1] == a)) return int(i) + 1;
    }
    return -1;
  }
};

}  // namespace

// Fast path used while building the face list: the list only ever holds 2-point
// entries at that stage, so Search reduces to a hash lookup.
static void compute_faces(const or_mesh& m, EdgeList& L) {
  std::unordered_map<uint64_t, int> pos;
  pos.reserve(size_t(m.n_elements) * 3);
  for (int e = 0; e < m.n_elements; ++e)
    for (int f = 0; f < 4; ++f) {
      const int a = m.quads[e * 4 + f], b = m.quads[e * 4 + (f + 1) % 4];
      const uint64_t k = EdgeList::key2(a, b);
      if (pos.count(k)) continue;
      pos[k] = int(L.e.size()) + 1;
      L.e.push_back({2, {a, b, 0}, false});
    }
  for (int b = 0; b < m.n_bdry_edges; ++b) {
    auto it = pos.find(EdgeList::key2(m.bdry_edges[2 * b], m.bdry_edges[2 * b + 1]));
    if (it != pos.end()) L.e[it->second - 1].attribute = true;
  }
}

static bool contains(const Entry& en, int x) {
  for (int k = 0; k < en.N; ++k) if (en.v[k] == x) return true;
  return false;
}

// SearchIfPresent(ONE, [x], howMany[, attributes])
static std::vector<int> search_if_present(const EdgeList& L, int x, int howMany, std::vector<bool>* atts) {
  std::vector<int> pos(howMany, -1);
  if (atts) atts->assign(howMany, false);
  int c = 0;
  for (size_t i = 0; i < L.e.size() && c < howMany; ++i)
    if (contains(L.e[i], x)) { pos[c] = int(i) + 1; if (atts) (*atts)[c] = L.e[i].attribute; ++c; }
  return pos;
}

static void merge_divided_faces(const or_mesh& m, EdgeList& L) {
  // node -> entry positions index, rebuilt lazily after every merge (merges are rare)
  for (int node = 1; node <= m.n_nodes; ++node) {
    std::vector<bool> atts;
    std::vector<int> edges = search_if_present(L, node, 4, &atts);
    if (edges[3] != -1) continue;
    if (edges[2] == -1) continue;
    if (std::any_of(atts.begin(), atts.end(), [](bool a) { return a; })) continue;
    int points[3];
    for (int j = 0; j < 3; ++j) {
      const Entry& en = L.e[edges[j] - 1];
      if (en.v[0] != node) points[j] = en.v[0];
      else if (en.v[1] != node) points[j] = en.v[1];
      else points[j] = -1;
    }
    bool merged = false;
    for (int j = 0; j < 3 && !merged; ++j) {
      std::vector<int> neigh = search_if_present(L, points[j], 8, nullptr);
      for (int k = 0; k < 8; ++k) {
        if (neigh[k] == -1) continue;
        const Entry en = L.e[neigh[k] - 1];
        int point;
        if (en.v[0] != points[j] && en.v[0] != node) point = en.v[0];
        else if (en.v[1] != points[j] && en.v[1] != node) point = en.v[1];
        else point = -1;
        if (point == points[0] || point == points[1] || point == points[2]) {
          const int s1 = en.v[0], s2 = en.v[1], s3 = node;
          auto remove = [&](int a, int b) {
            const int p = L.search2(a, b);
            if (p >= 1) L.e.erase(L.e.begin() + (p - 1));
          };
          remove(s1, s2);
          remove(s1, s3);
          remove(s2, s3);
          L.e.push_back({3, {s1, s2, s3}, false});
          merged = true;
          break;
        }
      }
    }
  }
}

static void compute_element_of_edges(const or_mesh& m, const EdgeList& L, std::vector<std::vector<int>>& eoe) {
  // node -> elements containing it, in element order
  std::vector<std::vector<int>> nodeEls(m.n_nodes + 1);
  for (int e = 0; e < m.n_elements; ++e)
    for (int k = 0; k < 4; ++k) {
      auto& v = nodeEls[m.quads[e * 4 + k]];
      if (v.empty() || v.back() != e + 1) v.push_back(e + 1);
    }
  auto has = [&](int e1, int node) {
    for (int k = 0; k < 4; ++k) if (m.quads[(e1 - 1) * 4 + k] == node) return true;
    return false;
  };
  eoe.resize(L.e.size());
  for (size_t i = 0; i < L.e.size(); ++i) {
    const Entry& en = L.e[i];
    if (en.N == 2) {
      std::vector<int> els;
      for (int e1 : nodeEls[en.v[0]]) {
        if (has(e1, en.v[1])) { els.push_back(e1); if (els.size() == 2) break; }
      }
      eoe[i] = els;
    } else {
      int r[3] = {-1, -1, -1};
      std::vector<int> cand = nodeEls[en.v[0]];
      cand.insert(cand.end(), nodeEls[en.v[1]].begin(), nodeEls[en.v[1]].end());
      std::sort(cand.begin(), cand.end());
      cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
      for (int e1 : cand) {
        if (has(e1, en.v[0]) && has(e1, en.v[1])) r[0] = e1;
        else if (has(e1, en.v[0]) && has(e1, en.v[2])) r[1] = e1;
        else if (has(e1, en.v[1]) && has(e1, en.v[2])) r[2] = e1;
        else continue;
        if (r[0] != -1 && r[1] != -1 && r[2] != -1) break;
      }
      eoe[i] = {r[0], r[1], r[2]};
    }
  }
}

// ---------------------------------------------------------------- edge geometry
static void edge_set_curve_straight(Oracle& o, Edge& f) {
  const int P = f.P();
  const double* n1 = &o.nodeX[2 * f.nodes[0]];
  const double* n2 = &o.nodeX[2 * f.nodes[1]];
  f.X.assign(2 * P, 0.0);
  for (int p = 0; p < P; ++p)
    for (int d = 0; d < 2; ++d) f.X[d * P + p] = n1[d] * (1.0 - f.sp->xi[p]) + n2[d] * f.sp->xi[p];
  double dS[2] = {n2[1] - n1[1], n1[0] - n2[0]};
  f.dS.assign(1, std::sqrt(dS[0] * dS[0] + dS[1] * dS[1]));
  f.n = {dS[0] / f.dS[0], dS[1] / f.dS[0]};
  f.dX = {n2[0] - n1[0], n2[1] - n1[1]};
}

static void edge_set_curve_curved(Oracle& o, Edge& f, const double* px, const double* py, int order) {
  const int N = f.N, P = N + 1, NC = f.NCurve;
  std::vector<double> cgl(order + 1), cgli(NC + 1);
  for (int k = 0; k <= order; ++k) cgl[k] = 0.5 + 0.5 * std::cos(PI * (order - k) / (1.0 * order));
  for (int k = 0; k <= NC; ++k) cgli[k] = 0.5 + 0.5 * std::cos(PI * (NC - k) / (1.0 * NC));
  std::vector<double> wb(order + 1), T((NC + 1) * (order + 1));
  barycentric_weights(order, cgl.data(), wb.data());
  interp_matrix(order, NC, cgl.data(), wb.data(), cgli.data(), T.data());
  std::vector<double> Xi(2 * (NC + 1), 0.0);
  for (int k = 0; k <= NC; ++k) {
    double sx = 0, sy = 0;
    for (int q = 0; q <= order; ++q) { sx += px[q] * T[k * (order + 1) + q]; sy += py[q] * T[k * (order + 1) + q]; }
    Xi[k] = sx; Xi[(NC + 1) + k] = sy;
  }
  std::vector<double> wb2(NC + 1), T2(P * (NC + 1));
  barycentric_weights(NC, cgli.data(), wb2.data());
  interp_matrix(NC, N, cgli.data(), wb2.data(), f.sp->xi.data(), T2.data());
  f.X.assign(2 * P, 0.0);
  for (int p = 0; p < P; ++p)
    for (int d = 0; d < 2; ++d) {
      double s = 0;
      for (int k = 0; k <= NC; ++k) s += Xi[d * (NC + 1) + k] * T2[p * (NC + 1) + k];
      f.X[d * P + p] = s;
    }
  f.dX.assign(2 * P, 0.0);
  for (int p = 0; p < P; ++p)
    for (int d = 0; d < 2; ++d) {
      double s = 0;
      for (int q = 0; q < P; ++q) s += f.X[d * P + q] * f.sp->D[p * P + q];
      f.dX[d * P + p] = s;
    }
  f.dS.assign(P, 0.0); f.n.assign(2 * P, 0.0);
  for (int p = 0; p < P; ++p) {
    const double dx = f.dX[p], dy = f.dX[P + p];
    f.dS[p] = std::sqrt(dx * dx + dy * dy);
    f.n[p] = dy / f.dS[p];
    f.n[P + p] = -dx / f.dS[p];
  }
}

// evaluateX(xi, direction): straight (Edge_AnalyticalX) or curved interpolant
static void edge_evaluate_x(const Oracle& o, const Edge& f, double xi, int dir, double* out) {
  const double cx = (dir == BACKWARD) ? 1.0 - xi : xi;
  if (f.kind == E_CURVED || f.kind == E_CURVED_SUBDIV) {
    const int P = f.P();
    std::vector<double> l = f.sp->lj(cx);
    for (int d = 0; d < 2; ++d) { double s = 0; for (int p = 0; p < P; ++p) s += f.X[d * P + p] * l[p]; out[d] = s; }
  } else {
    const double* n1 = &o.nodeX[2 * f.nodes[0]];
    const double* n2 = &o.nodeX[2 * f.nodes[1]];
    for (int d = 0; d < 2; ++d) out[d] = n1[d] * (1.0 - cx) + n2[d] * cx;
  }
}

static void edge_evaluate_dx(const Oracle& o, const Edge& f, double xi, int dir, double* out) {
  if (f.kind == E_CURVED || f.kind == E_CURVED_SUBDIV) {
    const double cx = (dir == BACKWARD) ? 1.0 - xi : xi;
    const int P = f.P();
    std::vector<double> l = f.sp->lj(cx);
    for (int d = 0; d < 2; ++d) { double s = 0; for (int p = 0; p < P; ++p) s += f.dX[d * P + p] * l[p]; out[d] = double(dir) * s; }
  } else {
    const double* n1 = &o.nodeX[2 * f.nodes[0]];
    const double* n2 = &o.nodeX[2 * f.nodes[1]];
    for (int d = 0; d < 2; ++d) out[d] = double(dir) * (n2[d] - n1[d]);
  }
}

// CurvedEdge_InterpolantdS: interpolate dS * n at xi (FORWARD)
static void edge_evaluate_ds(const Edge& f, double xi, double* out) {
  const int P = f.P();
  std::vector<double> l = f.sp->lj(xi);
  for (int d = 0; d < 2; ++d) {
    double s = 0;
    for (int p = 0; p < P; ++p) s += (f.dS[p] * f.n[d * P + p]) * l[p];
    out[d] = s;
  }
}

static void edge_invert(Oracle& o, Edge& f, bool changeSign) {
  std::swap(f.nodes[0], f.nodes[1]);
  const int P = f.P();
  for (int d = 0; d < 2; ++d) std::reverse(f.X.begin() + d * P, f.X.begin() + (d + 1) * P);
  if (f.straight_like()) {
    f.dX[0] = -f.dX[0]; f.dX[1] = -f.dX[1];
    if (changeSign) { f.n[0] = -f.n[0]; f.n[1] = -f.n[1]; }
  } else {
    for (int d = 0; d < 2; ++d) {
      std::reverse(f.dX.begin() + d * P, f.dX.begin() + (d + 1) * P);
      for (int p = 0; p < P; ++p) f.dX[d * P + p] = -f.dX[d * P + p];
      std::reverse(f.n.begin() + d * P, f.n.begin() + (d + 1) * P);
      if (changeSign) for (int p = 0; p < P; ++p) f.n[d * P + p] = -f.n[d * P + p];
    }
    std::reverse(f.dS.begin(), f.dS.end());
  }
  (void)o;
}

static void negate_normal(Edge& f) { for (auto& v : f.n) v = -v; }

// searchEdge / compareEdges: position (1..4) and direction of an edge in an element
static void search_edge(const int* nodesEl, int a, int b, bool& needsInversion, int& position, int& direction) {
  for (int edge = 1; edge <= 4; ++edge) {
    const int c1 = nodesEl[edge - 1], c2 = nodesEl[edge % 4];
    if (c1 == a && c2 == b) {
      position = edge; direction = (edge == EBOTTOM || edge == ERIGHT) ? FORWARD : BACKWARD;
      needsInversion = direction != FORWARD; return;
    }
    if (c1 == b && c2 == a) {
      position = edge; direction = (edge == EBOTTOM || edge == ERIGHT) ? BACKWARD : FORWARD;
      needsInversion = direction != FORWARD; return;
    }
  }
  throw std::runtime_error("edge not found in element");
}

static void init_storage(EdgeStorage& s, const Spectral* sp) {
  s.sp = sp;
  s.Q.assign(size_t(NCONS) * sp->P, 0.0);
  s.dQ.assign(size_t(2) * NCONS * sp->P, 0.0);
}

// T_backward = Minv_el * T_fwd^T * M_edge  (TripleMatrixProduct with trB)
static std::vector<double> backward_matrix(const Spectral* el, const Spectral* edg, const std::vector<double>& Tf) {
  const int Pe = el->P, Pm = edg->P;
  std::vector<double> Tb(size_t(Pe) * Pm);
  for (int i = 0; i < Pe; ++i)
    for (int l = 0; l < Pm; ++l) Tb[i * Pm + l] = ((1.0 / el->w[i]) * Tf[l * Pe + i]) * edg->w[l];
  return Tb;
}

static std::vector<double> forward_matrix(const Spectral* el, const Spectral* edg, const double* newNodes) {
  std::vector<double> T(size_t(edg->P) * el->P);
  interp_matrix(el->N, edg->N, el->xi.data(), el->wb.data(), newNodes, T.data());
  return T;
}

static void link_interior(Oracle& o, Edge& f, int eL, int eR) {
  Element& L = o.el[eL];
  Element& R = o.el[eR];
  int nodesID[2] = {f.nodes[0], f.nodes[1]};
  bool inv; int pos, dir;
  search_edge(L.nodes, nodesID[0], nodesID[1], inv, pos, dir);
  L.edges[pos - 1] = f.id; f.quads[SLOT_LEFT] = eL;
  L.edgesDirection[pos - 1] = FORWARD; L.quadPosition[pos - 1] = SLOT_LEFT; f.edgeLocation[SLOT_LEFT] = pos;
  if (inv) {
    edge_invert(o, f, pos == EBOTTOM || pos == ERIGHT);
    std::swap(nodesID[0], nodesID[1]);
  } else if (pos == ETOP || pos == ELEFT) {
    negate_normal(f);
  }
  init_storage(f.storage[SLOT_LEFT], L.sp);
  if (L.N == f.N) f.transform[SLOT_LEFT] = false;
  else {
    f.transform[SLOT_LEFT] = true; f.NLow = L.N;
    f.T_forward = forward_matrix(L.sp, f.sp, f.sp->xi.data());
    f.T_backward = backward_matrix(L.sp, f.sp, f.T_forward);
  }
  search_edge(R.nodes, nodesID[0], nodesID[1], inv, pos, dir);
  R.edges[pos - 1] = f.id; f.quads[SLOT_RIGHT] = eR;
  R.quadPosition[pos - 1] = SLOT_RIGHT; R.edgesDirection[pos - 1] = dir; f.edgeLocation[SLOT_RIGHT] = pos;
  f.inverse = dir != FORWARD;
  init_storage(f.storage[SLOT_RIGHT], R.sp);
  if (R.N == f.N) f.transform[SLOT_RIGHT] = false;
  else {
    f.transform[SLOT_RIGHT] = true; f.NLow = R.N;
    f.T_forward = forward_matrix(R.sp, f.sp, f.sp->xi.data());
    f.T_backward = backward_matrix(R.sp, f.sp, f.T_forward);
  }
}

static void link_boundary(Oracle& o, Edge& f, int e) {
  Element& E = o.el[e];
  bool inv; int pos, dir;
  search_edge(E.nodes, f.nodes[0], f.nodes[1], inv, pos, dir);
  E.boundaryElement = true;
  E.edges[pos - 1] = f.id; f.quads[0] = e;
  E.edgesDirection[pos - 1] = FORWARD; E.quadPosition[pos - 1] = 0; f.edgeLocation[0] = pos;
  if (inv) edge_invert(o, f, pos == EBOTTOM || pos == ERIGHT);
  else if (pos == ETOP || pos == ELEFT) negate_normal(f);
  init_storage(f.storage[0], E.sp);
  f.transform[0] = f.transform[1] = false;
}

static void construct_mortars(Oracle& o, Edge& f, int N_N, int N_S) {
  f.N_N = N_N; f.N_S = N_S;
  f.spN = o.spectral(N_N); f.spS = o.spectral(N_S);
  const int PN = N_N + 1, PS = N_S + 1;
  if (f.kind == E_SUBDIV) {
    f.normal_N = {f.n[0], f.n[1]}; f.normal_S = {f.n[0], f.n[1]};
    f.dS_N = {0.5 * f.dS[0]}; f.dS_S = {0.5 * f.dS[0]};
  } else {
    f.normal_N.assign(2 * PN, 0.0); f.normal_S.assign(2 * PS, 0.0);
    f.dS_N.assign(PN, 0.0); f.dS_S.assign(PS, 0.0);
    double v[2];
    for (int p = 0; p < PN; ++p) { edge_evaluate_ds(f, 0.5 + 0.5 * f.spN->xi[p], v); f.normal_N[p] = v[0]; f.normal_N[PN + p] = v[1]; }
    for (int p = 0; p < PS; ++p) { edge_evaluate_ds(f, 0.5 * f.spS->xi[p], v); f.normal_S[p] = v[0]; f.normal_S[PS + p] = v[1]; }
    for (int p = 0; p < PN; ++p) {
      const double a = f.normal_N[p], b = f.normal_N[PN + p];
      f.dS_N[p] = 0.5 * std::sqrt(a * a + b * b);
      f.normal_N[p] = 0.5 * a / f.dS_N[p]; f.normal_N[PN + p] = 0.5 * b / f.dS_N[p];
    }
    for (int p = 0; p < PS; ++p) {
      const double a = f.normal_S[p], b = f.normal_S[PS + p];
      f.dS_S[p] = 0.5 * std::sqrt(a * a + b * b);
      f.normal_S[p] = 0.5 * a / f.dS_S[p]; f.normal_S[PS + p] = 0.5 * b / f.dS_S[p];
    }
  }
}

static void mortar_matrices(Oracle& o, Edge& f) {
  const Spectral* spL = f.storage[SLOT_LEFT].sp;
  const Spectral* spRN = f.storage[SLOT_RN].sp;
  const Spectral* spRS = f.storage[SLOT_RS].sp;
  const int PN = f.spN->P, PS = f.spS->P;
  std::vector<double> nodesS(PS), nodesN(PN);
  for (int p = 0; p < PS; ++p) nodesS[p] = 0.5 * f.spS->xi[p];
  for (int p = 0; p < PN; ++p) nodesN[p] = 0.5 + 0.5 * f.spN->xi[p];
  f.T_LS_FWD = forward_matrix(spL, f.spS, nodesS.data());
  f.T_LN_FWD = forward_matrix(spL, f.spN, nodesN.data());
  f.T_LS_BKW = backward_matrix(spL, f.spS, f.T_LS_FWD);
  f.T_LN_BKW = backward_matrix(spL, f.spN, f.T_LN_FWD);
  f.T_RS_FWD = forward_matrix(spRS, f.spS, f.spS->xi.data());
  f.T_RS_BKW = backward_matrix(spRS, f.spS, f.T_RS_FWD);
  f.T_RN_FWD = forward_matrix(spRN, f.spN, f.spN->xi.data());
  f.T_RN_BKW = backward_matrix(spRN, f.spN, f.T_RN_FWD);
  // The reference builds invert_N with the RIGHT_SOUTH degree; identical when both degrees agree.
  auto flip_fwd = [](std::vector<double>& T, int rows, int cols) {   // T * invert  (reverse columns)
    for (int r = 0; r < rows; ++r) std::reverse(T.begin() + r * cols, T.begin() + (r + 1) * cols);
  };
  auto flip_bkw = [](std::vector<double>& T, int rows, int cols) {   // invert * T  (reverse rows)
    for (int r = 0; r < rows / 2; ++r)
      for (int c = 0; c < cols; ++c) std::swap(T[r * cols + c], T[(rows - 1 - r) * cols + c]);
  };
  const Element& RS = o.el[f.quads[SLOT_RS]];
  const Element& RN = o.el[f.quads[SLOT_RN]];
  if (RS.edgesDirection[f.edgeLocation[SLOT_RS] - 1] == BACKWARD) {
    flip_fwd(f.T_RS_FWD, PS, spRS->P); flip_bkw(f.T_RS_BKW, spRS->P, PS);
  }
  if (RN.edgesDirection[f.edgeLocation[SLOT_RN] - 1] == BACKWARD) {
    if (spRN->N != spRS->N) throw std::runtime_error("mortar with unequal right-element degrees is not supported");
    flip_fwd(f.T_RN_FWD, PN, spRN->P); flip_bkw(f.T_RN_BKW, spRN->P, PN);
  }
}

static void link_subdivided(Oracle& o, Edge& f, int eL, int eR1, int eR2) {
  Element& L = o.el[eL];
  int nodesID[3] = {f.nodes[0], f.nodes[1], f.nodes[2]};
  bool inv; int pos, dir;
  search_edge(L.nodes, nodesID[0], nodesID[1], inv, pos, dir);
  L.edges[pos - 1] = f.id; f.quads[SLOT_LEFT] = eL;
  L.edgesDirection[pos - 1] = FORWARD; L.quadPosition[pos - 1] = SLOT_LEFT; f.edgeLocation[SLOT_LEFT] = pos;
  int eRN, eRS;
  if (inv) {
    eRN = eR1; eRS = eR2;
    edge_invert(o, f, pos == EBOTTOM || pos == ERIGHT);
    std::swap(nodesID[0], nodesID[1]);
  } else {
    eRN = eR2; eRS = eR1;
    if (pos == ETOP || pos == ELEFT) negate_normal(f);
  }
  init_storage(f.storage[SLOT_LEFT], L.sp);
  Element& RN = o.el[eRN];
  Element& RS = o.el[eRS];
  construct_mortars(o, f, std::max(L.N, RN.N), std::max(L.N, RS.N));
  search_edge(RN.nodes, nodesID[2], nodesID[1], inv, pos, dir);
  RN.edges[pos - 1] = f.id; f.quads[SLOT_RN] = eRN;
  RN.quadPosition[pos - 1] = SLOT_RN; RN.edgesDirection[pos - 1] = dir; f.edgeLocation[SLOT_RN] = pos;
  init_storage(f.storage[SLOT_RN], RN.sp);
  search_edge(RS.nodes, nodesID[0], nodesID[2], inv, pos, dir);
  RS.edges[pos - 1] = f.id; f.quads[SLOT_RS] = eRS;
  RS.quadPosition[pos - 1] = SLOT_RS; RS.edgesDirection[pos - 1] = dir; f.edgeLocation[SLOT_RS] = pos;
  init_storage(f.storage[SLOT_RS], RS.sp);
  mortar_matrices(o, f);
}

// ---------------------------------------------------------------- element mappings
static void set_mappings(Oracle& o, Element& e) {
  const int P = e.P, N = e.N;
  const std::vector<double>& xi = e.sp->xi;
  // X_edges[edge][(j*P+i)*2+d]
  std::vector<double> Xe(4 * P * P * 2, 0.0), dXe(4 * P * P * 2, 0.0);
  auto idx = [P](int edge, int i, int j, int d) { return ((size_t(edge - 1) * P + j) * P + i) * 2 + d; };
  for (int edge = 1; edge <= 4; ++edge) {
    const Edge& f = o.ed[e.edges[edge - 1]];
    const int dir = e.edgesDirection[edge - 1];
    const bool alongXi = (edge == EBOTTOM || edge == ETOP);
    for (int a = 0; a < P; ++a) {      // a = iXi for bottom/top, iEta for right/left
      double X[2], dX[2];
      if (f.kind == E_STRAIGHT || f.kind == E_CURVED) {
        edge_evaluate_x(o, f, xi[a], dir, X);
        edge_evaluate_dx(o, f, xi[a], dir, dX);
      } else if (f.kind == E_SUBDIV || f.kind == E_CURVED_SUBDIV) {
        const int qp = e.quadPosition[edge - 1];
        double v = 0, scal = 1;
        if (dir == FORWARD) {
          if (qp == SLOT_LEFT) { v = xi[a]; scal = 1.0; }
          else if (qp == SLOT_RN) { v = 0.5 + 0.5 * xi[a]; scal = 0.5; }
          else { v = 0.5 * xi[a]; scal = 0.5; }
        } else {
          if (qp == SLOT_RN) { v = 0.5 + 0.5 * xi[N - a]; scal = -0.5; }
          else { v = 0.5 * xi[N - a]; scal = -0.5; }
        }
        edge_evaluate_x(o, f, v, FORWARD, X);
        edge_evaluate_dx(o, f, v, FORWARD, dX);
        dX[0] *= scal; dX[1] *= scal;
      } else {   // boundary edges: nodal values
        const int ci = (dir == BACKWARD) ? N - a : a;
        X[0] = f.X[ci]; X[1] = f.X[P + ci];
        if (f.kind == E_STRAIGHT_BDRY) { dX[0] = dir * f.dX[0]; dX[1] = dir * f.dX[1]; }
        else { dX[0] = dir * f.dX[ci]; dX[1] = dir * f.dX[P + ci]; }
      }
      for (int b = 0; b < P; ++b) {
        const int i = alongXi ? a : b, j = alongXi ? b : a;
        for (int d = 0; d < 2; ++d) { Xe[idx(edge, i, j, d)] = X[d]; dXe[idx(edge, i, j, d)] = dX[d]; }
      }
    }
  }
  const double* n1 = &o.nodeX[2 * e.nodes[0]];
  const double* n2 = &o.nodeX[2 * e.nodes[1]];
  const double* n3 = &o.nodeX[2 * e.nodes[2]];
  const double* n4 = &o.nodeX[2 * e.nodes[3]];
  e.X.assign(P * P * 2, 0.0); e.Ja.assign(P * P * 4, 0.0); e.jac.assign(P * P, 0.0);
  for (int i = 0; i < P; ++i)
    for (int j = 0; j < P; ++j) {
      const double x = xi[i], y = xi[j];
      double dx[2][2];   // dx[d][0] = d/dxi, dx[d][1] = d/deta
      for (int d = 0; d < 2; ++d) {
        e.X[(j * P + i) * 2 + d] = (1.0 - y) * Xe[idx(EBOTTOM, i, j, d)] + x * Xe[idx(ERIGHT, i, j, d)] +
                                   y * Xe[idx(ETOP, i, j, d)] + (1.0 - x) * Xe[idx(ELEFT, i, j, d)]
                                   - n1[d] * (1.0 - x) * (1.0 - y) - n2[d] * x * (1.0 - y)
                                   - n3[d] * x * y - n4[d] * (1.0 - x) * y;
        dx[d][0] = (1.0 - y) * dXe[idx(EBOTTOM, i, j, d)] + Xe[idx(ERIGHT, i, j, d)] +
                   y * dXe[idx(ETOP, i, j, d)] - Xe[idx(ELEFT, i, j, d)]
                   + n1[d] * (1.0 - y) - n2[d] * (1.0 - y) - n3[d] * y + n4[d] * y;
        dx[d][1] = -Xe[idx(EBOTTOM, i, j, d)] + x * dXe[idx(ERIGHT, i, j, d)] +
                   Xe[idx(ETOP, i, j, d)] + (1.0 - x) * dXe[idx(ELEFT, i, j, d)]
                   + n1[d] * (1.0 - x) + n2[d] * x - n3[d] * x - n4[d] * (1.0 - x);
      }
      const int q = j * P + i;
      e.jac[q] = dx[0][0] * dx[1][1] - dx[0][1] * dx[1][0];
      e.Ja[q * 4 + 0] = dx[1][1];    // Ja(IX,IX) =  y_eta
      e.Ja[q * 4 + 1] = -dx[1][0];   // Ja(IX,IY) = -y_xi
      e.Ja[q * 4 + 2] = -dx[0][1];   // Ja(IY,IX) = -x_eta
      e.Ja[q * 4 + 3] = dx[0][0];    // Ja(IY,IY) =  x_xi
    }
}

void build_mesh(Oracle& o, const or_mesh& m) {
  const double Lref = o.ph.L;
  o.nodeX.assign(size_t(m.n_nodes) * 2, 0.0);
  for (int i = 0; i < 2 * m.n_nodes; ++i) o.nodeX[i] = m.points[i] / Lref;

  EdgeList L;
  compute_faces(m, L);
  merge_divided_faces(m, L);
  merge_divided_faces(m, L);
  std::vector<std::vector<int>> eoe;
  compute_element_of_edges(m, L, eoe);
  std::vector<int> marker(L.e.size(), 0);
  {
    std::unordered_map<uint64_t, int> pos;
    for (size_t i = 0; i < L.e.size(); ++i)
      if (L.e[i].N == 2) pos[EdgeList::key2(L.e[i].v[0], L.e[i].v[1])] = int(i);
    for (int b = 0; b < m.n_bdry_edges; ++b) {
      auto it = pos.find(EdgeList::key2(m.bdry_edges[2 * b], m.bdry_edges[2 * b + 1]));
      if (it == pos.end()) throw std::runtime_error("boundary edge not in mesh");
      marker[it->second] = m.bdry_marker[b];
    }
  }
  // curved edges: first list entry containing both curve points; orient coordinates
  std::vector<int> curveOfEdge(L.e.size(), -1);
  std::vector<std::vector<double>> cx(m.n_curved), cy(m.n_curved);
  for (int k = 0; k < m.n_curved; ++k) {
    const int a = m.curved_edges[2 * k], b = m.curved_edges[2 * k + 1];
    int pos = -1;
    for (size_t i = 0; i < L.e.size(); ++i)
      if (contains(L.e[i], a) && contains(L.e[i], b)) { pos = int(i); break; }
    if (pos < 0) throw std::runtime_error("curved edge not found");
    cx[k].assign(m.curve_x + size_t(k) * m.curve_np1, m.curve_x + size_t(k + 1) * m.curve_np1);
    cy[k].assign(m.curve_y + size_t(k) * m.curve_np1, m.curve_y + size_t(k + 1) * m.curve_np1);
    for (auto& v : cx[k]) v /= Lref;
    for (auto& v : cy[k]) v /= Lref;
    const bool inv = L.e[pos].v[1] == a && L.e[pos].v[0] == b;
    if (inv) {
      std::reverse(cx[k].begin(), cx[k].end());
      std::reverse(cy[k].begin(), cy[k].end());
    }
    if (curveOfEdge[pos] < 0) curveOfEdge[pos] = k;
    o.mf_curve_edge.push_back(pos + 1);
    o.mf_curve_inv.push_back(inv ? 1 : 0);
  }
  for (size_t i = 0; i < L.e.size(); ++i) {
    for (int k = 0; k < 3; ++k) o.mf_points.push_back(k < L.e[i].N ? L.e[i].v[k] : 0);
    for (int k = 0; k < 3; ++k) o.mf_elements.push_back(k < int(eoe[i].size()) ? eoe[i][k] : 0);
    o.mf_marker.push_back(marker[i]);
  }
  // elements
  o.el.resize(m.n_elements);
  int64_t off = 0;
  for (int e = 0; e < m.n_elements; ++e) {
    Element& E = o.el[e];
    E.id = e; E.N = m.poly_order[e]; E.P = E.N + 1; E.sp = o.spectral(E.N);
    for (int k = 0; k < 4; ++k) E.nodes[k] = m.quads[e * 4 + k] - 1;
    E.offset = off;
    off += int64_t(NCONS) * E.P * E.P;
  }
  o.ndof = off;
  // edges
  o.ed.resize(L.e.size());
  for (size_t i = 0; i < L.e.size(); ++i) {
    Edge& f = o.ed[i];
    f.id = int(i);
    const Entry& en = L.e[i];
    for (int k = 0; k < en.N; ++k) f.nodes.push_back(en.v[k] - 1);
    const auto& els = eoe[i];
    int N, NLow, NCurve;
    if (els.size() == 1) { N = o.el[els[0] - 1].N; NLow = N; NCurve = N; }
    else if (els.size() == 2) {
      N = std::max(o.el[els[0] - 1].N, o.el[els[1] - 1].N);
      NLow = std::min(o.el[els[0] - 1].N, o.el[els[1] - 1].N);
      NCurve = NLow > 1 ? NLow / 2 : NLow;
    } else {
      N = o.el[els[0] - 1].N;
      NLow = std::min({o.el[els[0] - 1].N, o.el[els[1] - 1].N, o.el[els[2] - 1].N});
      NCurve = NLow > 1 ? NLow / 2 : NLow;
    }
    f.N = N; f.NLow = NLow; f.NCurve = NCurve; f.sp = o.spectral(N);
    f.edgeType = marker[i];
    const bool curved = curveOfEdge[i] >= 0;
    if (f.edgeType == 0 && en.N == 2) f.kind = curved ? E_CURVED : E_STRAIGHT;
    else if (f.edgeType == 0 && en.N == 3) f.kind = curved ? E_CURVED_SUBDIV : E_SUBDIV;
    else f.kind = curved ? E_CURVED_BDRY : E_STRAIGHT_BDRY;
    if (curved) {
      const int k = curveOfEdge[i];
      edge_set_curve_curved(o, f, cx[k].data(), cy[k].data(), m.curve_np1 - 1);
    } else {
      edge_set_curve_straight(o, f);
    }
    if (els.size() == 3) {
      double X[2];
      edge_evaluate_x(o, f, 0.5, FORWARD, X);
      o.nodeX[2 * f.nodes[2]] = X[0]; o.nodeX[2 * f.nodes[2] + 1] = X[1];
    }
  }
  for (auto& f : o.ed) if (f.kind == E_STRAIGHT) edge_set_curve_straight(o, f);
  for (size_t i = 0; i < L.e.size(); ++i) {
    const auto& els = eoe[i];
    Edge& f = o.ed[i];
    if (els.size() == 1) link_boundary(o, f, els[0] - 1);
    else if (els.size() == 2) link_interior(o, f, els[0] - 1, els[1] - 1);
    else link_subdivided(o, f, els[0] - 1, els[1] - 1, els[2] - 1);
  }
  for (auto& E : o.el) {
    for (int k = 0; k < 4; ++k) if (E.edges[k] < 0) throw std::runtime_error("element with unlinked edge");
    set_mappings(o, E);
  }
  for (auto& E : o.el) {   // BilinearForm_F(jac, w, w) = w . (jac w)
    double s = 0;
    for (int i = 0; i < E.P; ++i) {
      double t = 0;
      for (int j = 0; j < E.P; ++j) t += E.jac[j * E.P + i] * E.sp->w[j];
      s += E.sp->w[i] * t;
    }
    E.volume = s;
  }
  for (auto& f : o.ed) {
    const int P = f.P();
    double A = 0;
    for (int p = 0; p < P; ++p) A += (f.straight_like() ? f.dS[0] : f.dS[p]) * f.sp->w[p];
    f.Area = A;
    if (f.is_bdry()) f.invh = A / o.el[f.quads[0]].volume;
    else if (f.is_subdiv())
      f.invh = A / std::min({o.el[f.quads[SLOT_LEFT]].volume, o.el[f.quads[SLOT_RN]].volume, o.el[f.quads[SLOT_RS]].volume});
    else f.invh = A / std::min(o.el[f.quads[SLOT_LEFT]].volume, o.el[f.quads[SLOT_RIGHT]].volume);
  }
}

}  // namespace orc
