"""Mesh generators in the reference's .HiOMesh layout.

The reference reads meshes written by its Matlab preprocessor
(Utils/MeshPreprocessor/Functions/MeshFile.m) into the NetCDF variables
``points`` [nodes][2], ``points_of_quads`` [elements][4] (1-based, counter-
clockwise), ``points_of_bdryedges`` [bdry][2], ``bdrymarker_of_edges`` [bdry] and,
for curved meshes, ``curvilinear_edges`` [curves][2] with ``x/y_curvilinear_edges``
[curves][Np1] sampled at Chebyshev-Gauss-Lobatto points (Mesh/MeshFile.f90:77-279,
Mesh/QuadElement_EdgeMappings.incf CurvedEdge_SetCurve).  The generators below
produce the same dictionaries (keys as in tests/golden/*.mesh.npz) for the
benchmark workloads: periodic Cartesian boxes and the cylinder O-grid.
"""
import numpy as np


def cartesian(nx, ny, x0, x1, y0, y1):
    """Uniform nx x ny quads on [x0,x1]x[y0,y1]; markers 1 bottom, 2 top, 3 left, 4 right."""
    xs = np.linspace(x0, x1, nx + 1)
    ys = np.linspace(y0, y1, ny + 1)
    X, Y = np.meshgrid(xs, ys)                       # [ny+1][nx+1]
    points = np.stack([X.ravel(), Y.ravel()], 1)
    nid = np.arange((nx + 1) * (ny + 1)).reshape(ny + 1, nx + 1) + 1
    quads = np.stack([nid[:-1, :-1], nid[:-1, 1:], nid[1:, 1:], nid[1:, :-1]], -1).reshape(-1, 4)
    bottom = np.stack([nid[0, :-1], nid[0, 1:]], 1)
    top = np.stack([nid[-1, 1:], nid[-1, :-1]], 1)
    left = np.stack([nid[1:, 0], nid[:-1, 0]], 1)
    right = np.stack([nid[:-1, -1], nid[1:, -1]], 1)
    be = np.concatenate([bottom, top, left, right])
    bm = np.concatenate([np.full(nx, 1), np.full(nx, 2), np.full(ny, 3), np.full(ny, 4)])
    return dict(points=points.astype(np.float64), quads=quads.astype(np.int32), bdry_edges=be.astype(np.int32),
                bdry_marker=bm.astype(np.int32), marker_names=np.array(["bottom", "top", "left", "right"]))


def box_descriptor(nx, ny, x0, x1, y0, y1, N, node_type, *, elem_offset=0, edge_offset=0, marker_offset=0):
    """Constructed-mesh descriptor (include/horses_gpu.h hg_mesh_desc) of a doubly periodic box.

    Geometry is what the reference's transfinite mapping gives for affine quads
    (QuadElement_SetMappings): x_xi = hx, y_eta = hy, Ja = [[hy, 0], [0, hx]],
    J = hx hy; straight edges carry unit normals outward from their LEFT element
    and dS = edge length.  Connectivity follows the reference's conventions:
    an interior edge's LEFT element is the first element (in element order) that
    owns it, sides are numbered EBOTTOM=1, ERIGHT=2, ETOP=3, ELEFT=4, and the
    bottom/top and left/right boundary edges are periodic partners (markers
    1/2 and 3/4).  Element e = j*nx + i (row-major, as ``cartesian``).
    ``N``: one order, or one per element (p-refinement): an edge then carries
    max(N_L, N_R) + 1 nodes, the reference's edge order; periodic partners must
    share an order.
    """
    from ._lib import nodes as lib_nodes
    hx, hy = (x1 - x0) / nx, (y1 - y0) / ny
    E = nx * ny
    Ne = np.broadcast_to(np.asarray(N, np.int32), (E,)).astype(np.int32)
    Pe = Ne + 1
    i = np.tile(np.arange(nx), ny)
    j = np.repeat(np.arange(ny), nx)
    ex0 = x0 + i * hx
    ey0 = y0 + j * hy
    # nodes in (eta, xi) order, elements one after the other (Storage%Q offsets)
    n0 = np.concatenate([[0], np.cumsum(Pe * Pe)])
    nodes = int(n0[-1])
    xn, yn = np.empty(nodes), np.empty(nodes)
    for Nk in np.unique(Ne):
        xi, _ = lib_nodes(int(Nk), node_type)
        XI, ETA = np.meshgrid(xi, xi)                   # [eta][xi]
        el = np.nonzero(Ne == Nk)[0]
        idx = (n0[el][:, None] + np.arange((Nk + 1) ** 2)[None, :]).ravel()
        xn[idx] = (ex0[el][:, None] + hx * XI.ravel()[None, :]).ravel()
        yn[idx] = (ey0[el][:, None] + hy * ETA.ravel()[None, :]).ravel()
    x = np.stack([xn, yn], -1).reshape(-1)
    Ja = np.zeros((nodes, 4))
    Ja[:, 0] = hy
    Ja[:, 3] = hx
    jac = np.full(nodes, hx * hy)
    verts = np.stack([np.stack([ex0, ey0], 1), np.stack([ex0 + hx, ey0], 1), np.stack([ex0 + hx, ey0 + hy], 1),
                      np.stack([ex0, ey0 + hy], 1)], 1).reshape(-1)
    eid = (j * nx + i).reshape(ny, nx) + elem_offset
    edges_elem, edges_side, marker, nrm, dS = [], [], [], [], []

    def add(L, sL, R, sR, n_, d_, mk):
        edges_elem.append(np.stack([L, R], 1))
        edges_side.append(np.stack([np.full_like(L, sL), np.full_like(L, sR)], 1))
        marker.append(np.full(L.shape, mk))
        nrm.append(np.tile(np.asarray(n_, float), (L.size, 1)))
        dS.append(np.full(L.size, d_))

    none = lambda a: np.full_like(a, -1)   # noqa: E731
    # interior vertical edges: LEFT (i, j) side ERIGHT, RIGHT (i+1, j) side ELEFT, normal +x
    add(eid[:, :-1].ravel(), 2, eid[:, 1:].ravel(), 4, (1.0, 0.0), hy, 0)
    # interior horizontal edges: LEFT (i, j) side ETOP, RIGHT (i, j+1) side EBOTTOM, normal +y
    add(eid[:-1, :].ravel(), 3, eid[1:, :].ravel(), 1, (0.0, 1.0), hx, 0)
    nint = sum(a.shape[0] for a in edges_elem)
    b_bot, b_top, b_lft, b_rgt = eid[0, :], eid[-1, :], eid[:, 0], eid[:, -1]
    add(b_bot, 1, none(b_bot), 0, (0.0, -1.0), hx, marker_offset + 1)
    add(b_top, 3, none(b_top), 0, (0.0, 1.0), hx, marker_offset + 2)
    add(b_lft, 4, none(b_lft), 0, (-1.0, 0.0), hy, marker_offset + 3)
    add(b_rgt, 2, none(b_rgt), 0, (1.0, 0.0), hy, marker_offset + 4)
    F = nint + 2 * nx + 2 * ny
    partner = np.full(F, -1, np.int64)
    o = nint
    partner[o:o + nx] = np.arange(o + nx, o + 2 * nx) + edge_offset
    partner[o + nx:o + 2 * nx] = np.arange(o, o + nx) + edge_offset
    o += 2 * nx
    partner[o:o + ny] = np.arange(o + ny, o + 2 * ny) + edge_offset
    partner[o + ny:o + 2 * ny] = np.arange(o, o + ny) + edge_offset
    ee = np.concatenate(edges_elem)
    # nodes per edge: the higher order of its elements
    loc = ee - elem_offset
    PEd = np.where(loc[:, 1] >= 0, np.maximum(Pe[loc[:, 0]], Pe[np.maximum(loc[:, 1], 0)]), Pe[loc[:, 0]])
    # invh = Area / min(adjacent volumes) (QuadMesh_Construct.incf:270-303): 1/hx across x, 1/hy across y
    invh = np.concatenate([np.full(ny * (nx - 1), 1.0 / hx), np.full(nx * (ny - 1), 1.0 / hy),
                           np.full(2 * nx, 1.0 / hy), np.full(2 * ny, 1.0 / hx)])
    return dict(N=Ne.copy(), Ja=Ja.reshape(-1), jac=jac, x=x, volume=np.full(E, hx * hy),
                vertices=verts, edge_elem=ee.reshape(-1).astype(np.int32),
                edge_side=np.concatenate(edges_side).reshape(-1).astype(np.int32),
                edge_inverse=np.zeros(F, np.int32), edge_marker=np.concatenate(marker).astype(np.int32),
                edge_n=np.repeat(np.concatenate(nrm), PEd, axis=0).reshape(-1),
                edge_dS=np.repeat(np.concatenate(dS), PEd),
                periodic_partner=partner.astype(np.int32),
                edge_invh=invh)


def _same(a, b):
    """Spectral_Auxiliars almostEqual: |a-b| <= 2 eps max(|a|,|b|) (absolute 2 eps at zero)."""
    eps = np.finfo(float).eps
    if a == 0.0 or b == 0.0:
        return abs(a - b) <= 2.0 * eps
    return abs(b - a) <= 2.0 * eps * max(abs(a), abs(b))


def _bary(x):
    w = np.ones_like(x)
    for j in range(len(x)):
        for k in range(len(x)):
            if k != j:
                w[j] *= x[j] - x[k]
    return 1.0 / w


def _interp(old, new):
    """Barycentric interpolation matrix T[new, old] (exact rows where nodes coincide)."""
    wb = _bary(old)
    T = np.zeros((len(new), len(old)))
    for k, x in enumerate(new):
        d = x - old
        hit = np.abs(d) <= 2.0 * np.finfo(float).eps * np.maximum(np.abs(x), np.abs(old))
        if np.any(hit):
            T[k, np.argmax(hit)] = 1.0
        else:
            t = wb / d
            T[k] = t / t.sum()
    return T


def build_descriptor(m, N, node_type, *, reynolds_length=1.0, periodic_pairs=()):
    """Constructed-mesh descriptor (include/horses_gpu.h hg_mesh_desc) from .HiOMesh arrays.

    Conforming meshes with one polynomial order.  Restates the reference's
    construction (Mesh/MeshFile.f90 computeFaces / computeElementOfEdges,
    Mesh/QuadMesh_Construct.incf, Mesh/QuadElement_EdgeMappings.incf,
    Mesh/QuadElement_EdgeProcedures.incf Edge_LinkWithElements / Edge_Invert,
    Mesh/QuadElement_QuadMappings.incf QuadElement_SetMappings) with hash-based
    connectivity:
      * edges numbered by first appearance over elements and their faces
        (p1p2, p2p3, p3p4, p4p1); LEFT = first owner, RIGHT = second;
      * curved edges re-interpolated from their Chebyshev-Gauss-Lobatto samples at
        order N/2 (interior) or N (boundary), then at the edge nodes;
      * normals and dS per edge node, outward from LEFT, in LEFT's local order;
        ``inverse`` when RIGHT runs the other way;
      * transfinite element mappings, Ja = [[y_eta, -y_xi], [-x_eta, x_xi]].
    ``periodic_pairs``: [(marker_a, marker_b, coord)] boundary zones linked as the
    reference's Zone_LinkPeriodicZones does (coord 0: match x, 1: match y).
    """
    from ._lib import nodes as lib_nodes
    P = N + 1
    xi, w = lib_nodes(N, node_type)
    D = np.zeros((P, P))
    wb = _bary(xi)
    for i in range(P):
        for j in range(P):
            if j != i:
                D[i, j] = wb[j] / (wb[i] * (xi[i] - xi[j]))
        D[i, i] = -D[i].sum() + D[i, i]
    X = np.asarray(m["points"], float) / reynolds_length
    quads = np.asarray(m["quads"], np.int64) - 1
    E = quads.shape[0]
    # ---- connectivity
    edge_of, enodes, left, lside, right, rside = {}, [], [], [], [], []
    for e in range(E):
        for f in range(4):
            a, b = quads[e, f], quads[e, (f + 1) % 4]
            key = (min(a, b), max(a, b))
            if key not in edge_of:
                edge_of[key] = len(enodes)
                enodes.append((a, b))
                left.append(e); lside.append(f + 1); right.append(-1); rside.append(0)
            else:
                k = edge_of[key]
                if right[k] != -1:
                    raise ValueError("edge shared by more than two elements (non-conforming mesh)")
                right[k] = e; rside[k] = f + 1
    F = len(enodes)
    marker = np.zeros(F, np.int32)
    for (a, b), mk in zip(np.asarray(m["bdry_edges"], np.int64) - 1, np.asarray(m["bdry_marker"])):
        marker[edge_of[(min(a, b), max(a, b))]] = mk
    for k in range(F):
        if (right[k] < 0) != (marker[k] != 0):
            raise ValueError("boundary edges and element connectivity disagree (hanging nodes are not supported)")
    curve = {}
    if "curved_edges" in m and len(m["curved_edges"]):
        ce = np.asarray(m["curved_edges"], np.int64) - 1
        for c, (a, b) in enumerate(ce):
            k = edge_of[(min(a, b), max(a, b))]
            if k in curve:
                continue
            cx = np.asarray(m["curve_x"][c], float) / reynolds_length
            cy = np.asarray(m["curve_y"][c], float) / reynolds_length
            if (a, b) != tuple(enodes[k]):
                cx, cy = cx[::-1], cy[::-1]
            curve[k] = (cx, cy)
    # ---- edge geometry in stored order, then oriented to LEFT
    eX = np.zeros((F, P, 2)); edX = np.zeros((F, P, 2)); en = np.zeros((F, P, 2)); edS = np.zeros((F, P))
    straight = np.ones(F, bool)
    for k, (a, b) in enumerate(enodes):
        if k in curve:
            straight[k] = False
            cx, cy = curve[k]
            order = len(cx) - 1
            nc = N if marker[k] != 0 else (N // 2 if N > 1 else N)
            cgl = 0.5 + 0.5 * np.cos(np.pi * (order - np.arange(order + 1)) / order)
            cgli = 0.5 + 0.5 * np.cos(np.pi * (nc - np.arange(nc + 1)) / nc)
            T1 = _interp(cgl, cgli)
            T2 = _interp(cgli, xi)
            pts = T2 @ (T1 @ np.stack([cx, cy], 1))
            dX = D @ pts
            eX[k], edX[k] = pts, dX
            edS[k] = np.sqrt((dX ** 2).sum(1))
            en[k] = np.stack([dX[:, 1], -dX[:, 0]], 1) / edS[k][:, None]
        else:
            na, nb = X[a], X[b]
            eX[k] = na[None] * (1.0 - xi)[:, None] + nb[None] * xi[:, None]
            d = nb - na
            edX[k] = d
            L = np.sqrt(d[1] ** 2 + d[0] ** 2)
            edS[k] = L
            en[k] = np.array([d[1], -d[0]]) / L
    nodes_lp = [tuple(enodes[k]) for k in range(F)]
    for k in range(F):                         # LEFT side TOP/LEFT runs against the local coordinate
        if lside[k] in (3, 4):
            eX[k] = eX[k][::-1]; edX[k] = -edX[k][::-1]; edS[k] = edS[k][::-1]; en[k] = en[k][::-1]
            nodes_lp[k] = nodes_lp[k][::-1]
    inverse = np.zeros(F, np.int32)
    for k in range(F):
        if right[k] >= 0:
            e, s = right[k], rside[k] - 1
            p0, p1 = quads[e, s], quads[e, (s + 1) % 4]
            rp = (p0, p1) if s in (0, 1) else (p1, p0)
            inverse[k] = int(rp != nodes_lp[k])
    # ---- periodic partners (Zone_LinkPeriodicZones)
    partner = np.full(F, -1, np.int32)
    for ma, mb, coord in periodic_pairs:
        ea = [k for k in range(F) if marker[k] == ma]
        eb = [k for k in range(F) if marker[k] == mb]
        used = set()
        for k1 in ea:
            a1, b1 = X[nodes_lp[k1][0], coord], X[nodes_lp[k1][1], coord]
            for k2 in eb:
                if k2 in used:
                    continue
                a2, b2 = X[nodes_lp[k2][0], coord], X[nodes_lp[k2][1], coord]
                if (_same(a1, a2) and _same(b1, b2)) or (_same(a1, b2) and _same(b1, a2)):
                    used.add(k2)
                    partner[k1], partner[k2] = k2, k1
                    inv = int(np.dot(edX[k1][0], edX[k2][0]) < 0.0)
                    inverse[k1] = inverse[k2] = inv
                    break
    # ---- element mappings (transfinite)
    elem_edges = {}
    for k in range(F):
        elem_edges[(left[k], lside[k])] = (k, 1)
        if right[k] >= 0:
            elem_edges[(right[k], rside[k])] = (k, -1 if inverse[k] else 1)
    Ja = np.zeros((E, P, P, 4)); jac = np.zeros((E, P, P)); xn = np.zeros((E, P, P, 2))
    XI, ETA = np.meshgrid(xi, xi)            # [j][i]
    for e in range(E):
        Xe = np.zeros((4, P, P, 2)); dXe = np.zeros((4, P, P, 2))
        for side in range(1, 5):
            k, dr = elem_edges[(e, side)]
            cx = xi if dr == 1 else 1.0 - xi
            if marker[k] != 0:
                idx = np.arange(P) if dr == 1 else np.arange(P)[::-1]
                Xs, dXs = eX[k][idx], dr * (edX[k][idx] if not straight[k] else np.tile(edX[k][0], (P, 1)))
            elif straight[k]:
                na, nb = X[nodes_lp[k][0]], X[nodes_lp[k][1]]
                Xs = na[None] * (1.0 - cx)[:, None] + nb[None] * cx[:, None]
                dXs = np.tile(dr * (nb - na), (P, 1))
            else:
                T = _interp(xi, cx)
                Xs, dXs = T @ eX[k], dr * (T @ edX[k])
            if side in (1, 3):                    # along xi: value depends on i
                Xe[side - 1] = Xs[None, :, :].repeat(P, 0)
                dXe[side - 1] = dXs[None, :, :].repeat(P, 0)
            else:                                 # along eta: value depends on j
                Xe[side - 1] = Xs[:, None, :].repeat(P, 1)
                dXe[side - 1] = dXs[:, None, :].repeat(P, 1)
        n1, n2, n3, n4 = (X[quads[e, q]] for q in range(4))
        x_, y_ = XI[..., None], ETA[..., None]
        Xm = ((1 - y_) * Xe[0] + x_ * Xe[1] + y_ * Xe[2] + (1 - x_) * Xe[3]
              - n1 * (1 - x_) * (1 - y_) - n2 * x_ * (1 - y_) - n3 * x_ * y_ - n4 * (1 - x_) * y_)
        dxi = ((1 - y_) * dXe[0] + Xe[1] + y_ * dXe[2] - Xe[3] + n1 * (1 - y_) - n2 * (1 - y_) - n3 * y_ + n4 * y_)
        deta = (-Xe[0] + x_ * dXe[1] + Xe[2] + (1 - x_) * dXe[3] + n1 * (1 - x_) + n2 * x_ - n3 * x_ - n4 * (1 - x_))
        jac[e] = dxi[..., 0] * deta[..., 1] - deta[..., 0] * dxi[..., 1]
        Ja[e, ..., 0] = deta[..., 1]
        Ja[e, ..., 1] = -dxi[..., 1]
        Ja[e, ..., 2] = -deta[..., 0]
        Ja[e, ..., 3] = dxi[..., 0]
        xn[e] = Xm
    vol = np.einsum("eji,j,i->e", jac, w, w)
    area = (edS * w[None, :]).sum(1)
    invh = np.zeros(F)
    for k in range(F):
        vmin = vol[left[k]] if right[k] < 0 else min(vol[left[k]], vol[right[k]])
        invh[k] = area[k] / vmin
    return dict(N=np.full(E, N, np.int32), Ja=Ja.reshape(-1), jac=jac.reshape(-1), x=xn.reshape(-1),
                volume=vol, vertices=X[quads].reshape(-1),
                edge_elem=np.stack([left, right], 1).reshape(-1).astype(np.int32),
                edge_side=np.stack([lside, rside], 1).reshape(-1).astype(np.int32),
                edge_inverse=inverse, edge_marker=marker, edge_n=en.reshape(-1), edge_dS=edS.reshape(-1),
                periodic_partner=partner, edge_invh=invh)


def concat_descriptors(descs):
    """Pack independent meshes into one element list (disjoint union, ensemble runs)."""
    out = {}
    for k in descs[0]:
        out[k] = np.concatenate([d[k] for d in descs])
    return out


def periodic_bcs_cartesian():
    """Zone list (markers 1..4) pairing bottom/top (y) and left/right (x), as the reference's case files do."""
    return [dict(type=1, periodic_dir=2, connected_marker=2), dict(type=1, periodic_dir=2, connected_marker=1),
            dict(type=1, periodic_dir=1, connected_marker=4), dict(type=1, periodic_dir=1, connected_marker=3)]


def ogrid(n_radial, n_azimuthal, r0, r1, stretch, np1=11):
    """O-grid around a circle of radius r0 out to r1 with geometric radial stretching.

    Every azimuthal arc is a curved edge sampled at ``np1`` Chebyshev-Gauss-Lobatto
    points.  Markers: 1 wall (r = r0), 2 far field (r = r1).
    """
    # radial stations with geometric growth, scaled to end exactly at r1
    w = stretch ** np.arange(n_radial)
    r = r0 + (r1 - r0) * np.concatenate([[0.0], np.cumsum(w)]) / w.sum()
    th = 2.0 * np.pi * np.arange(n_azimuthal) / n_azimuthal
    R, T = np.meshgrid(r, th, indexing="ij")          # [nr+1][nt]
    points = np.stack([(R * np.cos(T)).ravel(), (R * np.sin(T)).ravel()], 1)
    nid = np.arange((n_radial + 1) * n_azimuthal).reshape(n_radial + 1, n_azimuthal) + 1
    nxt = np.roll(nid, -1, axis=1)
    # counter-clockwise quads: (r_i, th_j) -> (r_i+1, th_j) -> (r_i+1, th_j+1) -> (r_i, th_j+1)
    quads = np.stack([nid[:-1], nid[1:], nxt[1:], nxt[:-1]], -1).reshape(-1, 4)
    wall = np.stack([nxt[0], nid[0]], 1)
    far = np.stack([nid[-1], nxt[-1]], 1)
    be = np.concatenate([wall, far])
    bm = np.concatenate([np.full(n_azimuthal, 1), np.full(n_azimuthal, 2)])
    # curved (azimuthal) edges on every radial station
    cgl = 0.5 - 0.5 * np.cos(np.pi * np.arange(np1) / (np1 - 1))
    ce, cx, cy = [], [], []
    for i in range(n_radial + 1):
        for j in range(n_azimuthal):
            a, b = nid[i, j], nxt[i, j]
            ta = th[j]
            tb = ta + 2.0 * np.pi / n_azimuthal
            tt = ta + (tb - ta) * cgl
            ce.append((a, b))
            cx.append(r[i] * np.cos(tt))
            cy.append(r[i] * np.sin(tt))
    return dict(points=points.astype(np.float64), quads=quads.astype(np.int32), bdry_edges=be.astype(np.int32),
                bdry_marker=bm.astype(np.int32), marker_names=np.array(["wall", "farfield"]),
                curved_edges=np.array(ce, np.int32), curve_x=np.array(cx), curve_y=np.array(cy))


def locate(desc, points, node_type, tol=1e-12, max_iter=30):
    """Element (0-based) and reference coordinates (xi, eta) in [0,1]^2 of physical points, for probes
    (the reference locates a probe once, at monitor construction).  The element map is the degree-N
    interpolant of the descriptor's node coordinates (the transfinite map itself on straight-sided
    elements); candidates are the elements whose bounding box (nodes and vertices, widened by a tenth)
    holds the point, and the map is inverted by Newton's method.  Returns (elements [n] int32, xi_eta [n, 2]); raises ValueError for a
    point outside the mesh."""
    from ._lib import nodes as lib_nodes
    pts = np.asarray(points, dtype=float).reshape(-1, 2)
    N = int(np.asarray(desc["N"])[0])
    P = N + 1
    xi, _ = lib_nodes(N, node_type)
    bw = np.array([1.0 / np.prod([xi[j] - xi[k] for k in range(P) if k != j]) for j in range(P)])
    X = np.asarray(desc["x"], dtype=float).reshape(-1, P * P, 2)
    V = np.asarray(desc["vertices"], dtype=float).reshape(-1, 4, 2)
    lo, hi = np.minimum(X.min(1), V.min(1)), np.maximum(X.max(1), V.max(1))
    pad = 0.1 * (hi - lo).max(1, keepdims=True)     # curved sides may bulge past nodes and vertices

    def basis(x):
        d = x - xi
        hit = np.abs(d) <= 1e-15
        if hit.any():
            l = hit.astype(float)
            # derivative at a node: l_j'(x_i) = D(i, j)
            i = int(np.argmax(hit))
            dl = np.array([(bw[j] / bw[i]) / (xi[i] - xi[j]) if j != i else 0.0 for j in range(P)])
            dl[i] = -dl.sum()
            return l, dl
        t = bw / d
        s = t.sum()
        l = t / s
        dt = -bw / d ** 2
        dl = (dt * s - t * dt.sum()) / s ** 2
        return l, dl

    elements, coords = np.zeros(len(pts), np.int32), np.zeros((len(pts), 2))
    for k, p in enumerate(pts):
        cand = np.nonzero(np.all(lo - pad <= p, 1) & np.all(p <= hi + pad, 1))[0]
        for e in cand:
            G = X[e].reshape(P, P, 2)          # [eta][xi][d]
            s = np.array([0.5, 0.5])
            for _ in range(max_iter):
                lx, dlx = basis(s[0])
                ly, dly = basis(s[1])
                f = np.einsum("j,i,jid->d", ly, lx, G) - p
                J = np.stack([np.einsum("j,i,jid->d", ly, dlx, G), np.einsum("j,i,jid->d", dly, lx, G)], 1)
                ds = np.linalg.solve(J, -f)
                s = np.clip(s + ds, -0.5, 1.5)
                if np.abs(ds).max() < tol:
                    break
            if np.all(s >= -1e-10) and np.all(s <= 1.0 + 1e-10):
                elements[k], coords[k] = e, np.clip(s, 0.0, 1.0)
                break
        else:
            raise ValueError(f"point {tuple(p)} is outside the mesh")
    return elements, coords


def connectivity(m):
    """Mesh-file connectivity through the library's O(E) builder (hg_mesh_connectivity), for a mesh dict
    with points, quads (1-based point ids), bdry_edges, bdry_marker and optional curved_edges: the
    reference's lists (1-based, list order) as dict(points_of_edges [F,3], elements_of_edges [F,3],
    edge_marker [F], curved_edges [C], curve_inverted [C])."""
    import ctypes as C
    from . import _lib as L
    lib = L.load()
    quads = np.ascontiguousarray(m["quads"], dtype=np.int32).reshape(-1, 4)
    be = np.ascontiguousarray(m["bdry_edges"], dtype=np.int32).reshape(-1, 2)
    bm = np.ascontiguousarray(m["bdry_marker"], dtype=np.int32).ravel()
    ce = np.ascontiguousarray(m.get("curved_edges", np.zeros((0, 2))), dtype=np.int32).reshape(-1, 2)
    n_pts = int(np.asarray(m["points"]).reshape(-1, 2).shape[0])
    cap = 4 * quads.shape[0]
    nE = C.c_int32(0)
    pts, els = np.zeros((cap, 3), np.int32), np.zeros((cap, 3), np.int32)
    mk = np.zeros(cap, np.int32)
    cedge, cinv = np.zeros(max(len(ce), 1), np.int32), np.zeros(max(len(ce), 1), np.int32)
    p = lambda a: a.ctypes.data_as(L.I32P)   # noqa: E731
    rc = lib.hg_mesh_connectivity(n_pts, quads.shape[0], p(quads), be.shape[0], p(be), p(bm), len(ce), p(ce), cap,
                                  C.byref(nE), p(pts), p(els), p(mk), p(cedge), p(cinv))
    if rc != 0:
        raise ValueError(lib.hg_mesh_last_error().decode())
    F = nE.value
    return dict(points_of_edges=pts[:F], elements_of_edges=els[:F], edge_marker=mk[:F],
                curved_edges=cedge[:len(ce)], curve_inverted=cinv[:len(ce)])
