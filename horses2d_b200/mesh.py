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
