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
    """
    from ._lib import nodes as lib_nodes
    P = N + 1
    xi, _ = lib_nodes(N, node_type)
    hx, hy = (x1 - x0) / nx, (y1 - y0) / ny
    E = nx * ny
    i = np.tile(np.arange(nx), ny)
    j = np.repeat(np.arange(ny), nx)
    ex0 = x0 + i * hx
    ey0 = y0 + j * hy
    # nodes in (eta, xi) order
    XI, ETA = np.meshgrid(xi, xi)                       # [eta][xi]
    xn = ex0[:, None] + hx * XI.ravel()[None, :]
    yn = ey0[:, None] + hy * ETA.ravel()[None, :]
    x = np.stack([xn, yn], -1).reshape(-1)
    Ja = np.zeros((E, P * P, 4))
    Ja[:, :, 0] = hy
    Ja[:, :, 3] = hx
    jac = np.full(E * P * P, hx * hy)
    verts = np.stack([np.stack([ex0, ey0], 1), np.stack([ex0 + hx, ey0], 1), np.stack([ex0 + hx, ey0 + hy], 1),
                      np.stack([ex0, ey0 + hy], 1)], 1).reshape(-1)
    eid = (j * nx + i).reshape(ny, nx) + elem_offset
    edges_elem, edges_side, marker, nrm, dS, partner = [], [], [], [], [], []

    def add(L, sL, R, sR, n_, d_, mk):
        edges_elem.append(np.stack([L, R], 1))
        edges_side.append(np.stack([np.full_like(L, sL), np.full_like(L, sR)], 1))
        marker.append(np.full(L.shape, mk))
        nrm.append(np.tile(np.asarray(n_, float), (L.size, P, 1)))
        dS.append(np.full((L.size, P), d_))

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
    return dict(N=np.full(E, N, np.int32), Ja=Ja.reshape(-1), jac=jac, x=x, volume=np.full(E, hx * hy),
                vertices=verts, edge_elem=ee.reshape(-1).astype(np.int32),
                edge_side=np.concatenate(edges_side).reshape(-1).astype(np.int32),
                edge_inverse=np.zeros(F, np.int32), edge_marker=np.concatenate(marker).astype(np.int32),
                edge_n=np.concatenate(nrm).reshape(-1), edge_dS=np.concatenate(dS).reshape(-1),
                periodic_partner=partner.astype(np.int32),
                edge_invh=np.full(F, 0.0))


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
