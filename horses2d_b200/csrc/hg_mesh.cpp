// hg_mesh.cpp -- connectivity of a quad mesh file in O(E): the edge list, subdivided (hanging-node)
// edges, the elements of each edge, boundary markers and curved-edge assignment, with the same
// results as the reference's list-based construction (Mesh/MeshFile.f90:254-267 and 287-652:
// computeFaces, mergeDividedFaces twice, computeElementOfEdges, computeFaceMarkers,
// computeCurvedEdges), whose searches are linear in the list and make preprocessing O(E^2).
//
// The reference's IntegerArrayLinkedList fixes the conventions kept here:
//  * edges are listed in order of first appearance over the elements' faces (p1 p2, p2 p3, p3 p4,
//    p4 p1), stored with the orientation of that first appearance; lookups ignore orientation;
//  * a merged subdivided edge is removed from its place and appended at the end as
//    [long-edge ends as stored, middle node];
//  * "the first k entries containing a node" (SearchIfPresent) are taken in current list order.
// Here entries carry a creation sequence number, removed entries are marked dead, and every node
// keeps the ids of the entries containing it in creation order, so each of those searches costs
// the node's valence instead of the list length.
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>
#include <stdexcept>
#include <algorithm>

namespace {

struct Entry {
  int n = 2;        // 2 points, or 3 for a subdivided edge (middle node last)
  int v[3] = {0, 0, 0};
  bool boundary = false;
  bool alive = true;
};

inline uint64_t pair_key(int a, int b) {
  const uint32_t lo = uint32_t(std::min(a, b)), hi = uint32_t(std::max(a, b));
  return (uint64_t(lo) << 32) | hi;
}

struct EdgeList {
  std::vector<Entry> e;
  std::unordered_map<uint64_t, int> simple;      // sorted pair -> live 2-point entry
  std::vector<std::vector<int>> of_node;         // node -> entries containing it, creation order

  explicit EdgeList(int n_points) : of_node(size_t(n_points) + 1) {}

  int find2(int a, int b) const {
    auto it = simple.find(pair_key(a, b));
    return it == simple.end() ? -1 : it->second;
  }
  int add(int n, const int* v) {
    const int id = int(e.size());
    Entry en;
    en.n = n;
    for (int k = 0; k < n; ++k) en.v[k] = v[k];
    e.push_back(en);
    if (n == 2) simple.emplace(pair_key(v[0], v[1]), id);
    for (int k = 0; k < n; ++k) of_node[size_t(v[k])].push_back(id);
    return id;
  }
  void remove(int id) {
    Entry& en = e[size_t(id)];
    en.alive = false;
    if (en.n == 2) simple.erase(pair_key(en.v[0], en.v[1]));
  }
  // first `how_many` live entries containing node x, in list order
  int present(int x, int how_many, int* out) const {
    int c = 0;
    for (int id : of_node[size_t(x)]) {
      if (!e[size_t(id)].alive) continue;
      out[c++] = id;
      if (c == how_many) break;
    }
    return c;
  }
};

void merge_divided_faces(EdgeList& L, int n_points) {
  for (int X = 1; X <= n_points; ++X) {
    int edges[4];
    const int ne = L.present(X, 4, edges);
    if (ne >= 4 || ne < 3) continue;     // four edges: not a hanging node; fewer than three: merged
    bool bdry = false;
    for (int j = 0; j < 3; ++j) bdry = bdry || L.e[size_t(edges[j])].boundary;
    if (bdry) continue;
    int pts[3];
    for (int j = 0; j < 3; ++j) {
      const Entry& en = L.e[size_t(edges[j])];
      pts[j] = en.v[0] != X ? en.v[0] : en.v[1];
    }
    bool merged = false;
    for (int j = 0; j < 3 && !merged; ++j) {
      int neigh[8];
      const int nn = L.present(pts[j], 8, neigh);
      for (int k = 0; k < nn && !merged; ++k) {
        const Entry& en = L.e[size_t(neigh[k])];
        const int a = en.v[0], b = en.v[1];
        int point = -1;
        if (a != pts[j] && a != X) point = a;
        else if (b != pts[j] && b != X) point = b;
        if (point != pts[0] && point != pts[1] && point != pts[2]) continue;
        const int sub[3] = {a, b, X};
        const int r1 = L.find2(sub[0], sub[1]), r2 = L.find2(sub[0], sub[2]), r3 = L.find2(sub[1], sub[2]);
        if (r1 >= 0) L.remove(r1);
        if (r2 >= 0) L.remove(r2);
        if (r3 >= 0) L.remove(r3);
        L.add(3, sub);
        merged = true;
      }
    }
  }
}

}  // namespace

static std::string g_mesh_err;

extern "C" const char* hg_mesh_last_error() { return g_mesh_err.c_str(); }

extern "C" int hg_mesh_connectivity(int32_t n_points, int32_t n_elements, const int32_t* points_of_quads,
                                    int32_t n_bdry_edges, const int32_t* points_of_bdryedges,
                                    const int32_t* bdry_marker, int32_t n_curved, const int32_t* curved_edges_points,
                                    int32_t capacity, int32_t* n_edges, int32_t* points_of_edges,
                                    int32_t* elements_of_edges, int32_t* edge_marker, int32_t* curved_edges,
                                    int32_t* curve_inverted) {
  try {
    if (n_points < 1 || n_elements < 1 || !points_of_quads || !n_edges || !points_of_edges || !elements_of_edges ||
        !edge_marker || n_bdry_edges < 0 || (n_bdry_edges > 0 && (!points_of_bdryedges || !bdry_marker)) ||
        n_curved < 0 || (n_curved > 0 && (!curved_edges_points || !curved_edges || !curve_inverted)))
      throw std::runtime_error("bad mesh connectivity arguments");
    for (int64_t k = 0; k < int64_t(n_elements) * 4; ++k)
      if (points_of_quads[k] < 1 || points_of_quads[k] > n_points) throw std::runtime_error("quad point out of range");
    EdgeList L(n_points);
    L.e.reserve(size_t(n_elements) * 2 + 16);
    L.simple.reserve(size_t(n_elements) * 3);
    // computeFaces: faces of every element, first appearance kept
    for (int e = 0; e < n_elements; ++e) {
      const int32_t* q = points_of_quads + size_t(e) * 4;
      for (int f = 0; f < 4; ++f) {
        const int face[2] = {q[f], q[(f + 1) % 4]};
        if (L.find2(face[0], face[1]) < 0) L.add(2, face);
      }
    }
    // boundary attribute
    for (int b = 0; b < n_bdry_edges; ++b) {
      const int id = L.find2(points_of_bdryedges[2 * b], points_of_bdryedges[2 * b + 1]);
      if (id < 0) throw std::runtime_error("boundary edge " + std::to_string(b + 1) + " is no face of the mesh");
      L.e[size_t(id)].boundary = true;
    }
    merge_divided_faces(L, n_points);
    merge_divided_faces(L, n_points);
    // live entries in list order -> output positions
    std::vector<int> pos(L.e.size(), -1);
    int F = 0;
    for (size_t i = 0; i < L.e.size(); ++i)
      if (L.e[i].alive) pos[i] = F++;
    if (F > capacity) throw std::runtime_error("edge capacity too small: need " + std::to_string(F));
    // elements of each node (ascending), for computeElementOfEdges
    std::vector<std::vector<int>> el_of_node(size_t(n_points) + 1);
    for (int e = 0; e < n_elements; ++e)
      for (int k = 0; k < 4; ++k) {
        auto& v = el_of_node[size_t(points_of_quads[size_t(e) * 4 + k])];
        if (v.empty() || v.back() != e + 1) v.push_back(e + 1);
      }
    auto has = [&](int e, int x) {
      const int32_t* q = points_of_quads + size_t(e - 1) * 4;
      return q[0] == x || q[1] == x || q[2] == x || q[3] == x;
    };
    for (size_t i = 0; i < L.e.size(); ++i) {
      if (pos[i] < 0) continue;
      const Entry& en = L.e[i];
      const int p = pos[i];
      int32_t* pe = points_of_edges + size_t(p) * 3;
      int32_t* ee = elements_of_edges + size_t(p) * 3;
      pe[0] = en.v[0]; pe[1] = en.v[1]; pe[2] = en.n == 3 ? en.v[2] : 0;
      ee[0] = ee[1] = ee[2] = 0;
      edge_marker[p] = 0;
      if (en.n == 2) {
        // searchSimpleEdgeInElements: the first two elements (by id) holding both points
        int c = 0;
        for (int e : el_of_node[size_t(en.v[0])])
          if (has(e, en.v[1])) { ee[c++] = e; if (c == 2) break; }
      } else {
        // searchDividedEdgeInElements: ascending elements; (1,2) -> slot 1, else (1,3) -> 2, else (2,3) -> 3,
        // later matches overwrite, stop when all three slots are set
        std::vector<int> cand;
        for (int k = 0; k < 3; ++k) cand.insert(cand.end(), el_of_node[size_t(en.v[k])].begin(), el_of_node[size_t(en.v[k])].end());
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        int s[3] = {-1, -1, -1};
        for (int e : cand) {
          const bool h1 = has(e, en.v[0]), h2 = has(e, en.v[1]), h3 = has(e, en.v[2]);
          if (h1 && h2) s[0] = e;
          else if (h1 && h3) s[1] = e;
          else if (h2 && h3) s[2] = e;
          else continue;
          if (s[0] != -1 && s[1] != -1 && s[2] != -1) break;
        }
        for (int k = 0; k < 3; ++k) ee[k] = s[k] < 0 ? 0 : s[k];
      }
    }
    // computeFaceMarkers
    for (int b = 0; b < n_bdry_edges; ++b) {
      const int id = L.find2(points_of_bdryedges[2 * b], points_of_bdryedges[2 * b + 1]);
      if (id < 0 || pos[size_t(id)] < 0) throw std::runtime_error("boundary edge " + std::to_string(b + 1) + " was merged");
      edge_marker[pos[size_t(id)]] = bdry_marker[b];
    }
    // computeCurvedEdges: first listed edge holding both curve points; inverted when stored the other way
    for (int k = 0; k < n_curved; ++k) {
      const int a = curved_edges_points[2 * k], b = curved_edges_points[2 * k + 1];
      if (a < 1 || a > n_points || b < 1 || b > n_points) throw std::runtime_error("curve point out of range");
      int best = -1;
      for (int id : L.of_node[size_t(a)]) {
        const Entry& en = L.e[size_t(id)];
        if (!en.alive) continue;
        bool hb = false;
        for (int q = 0; q < en.n; ++q) hb = hb || en.v[q] == b;
        if (hb && (best < 0 || pos[size_t(id)] < pos[size_t(best)])) best = id;
      }
      if (best < 0) throw std::runtime_error("curved edge " + std::to_string(k + 1) + " is no edge of the mesh");
      const Entry& en = L.e[size_t(best)];
      curved_edges[k] = pos[size_t(best)] + 1;
      if (en.v[0] == a && en.v[1] == b) curve_inverted[k] = 0;
      else if (en.v[1] == a && en.v[0] == b) curve_inverted[k] = 1;
      else throw std::runtime_error("curved edge " + std::to_string(k + 1) + " does not match its edge's ends");
    }
    *n_edges = F;
    g_mesh_err.clear();
    return 0;
  } catch (const std::exception& ex) {
    g_mesh_err = ex.what();
    return 1;
  }
}
