"""Host-side mesh builders of the package against the oracle's reference-faithful construction (CPU)."""
import numpy as np
import pytest

from oracle import oracle as O
from horses2d_b200 import mesh as hmesh, lib


def side_table(d):
    """Per element-side view of an edge-centric descriptor: neighbour, orientation, normals, dS."""
    E = len(d["N"])
    F = len(d["edge_marker"])
    tab = {}
    # nodes per edge: the higher order of its elements
    ee = np.asarray(d["edge_elem"]).reshape(-1, 2)
    PE = np.where(ee[:, 1] >= 0, np.maximum(d["N"][ee[:, 0]], d["N"][np.maximum(ee[:, 1], 0)]), d["N"][ee[:, 0]]) + 1
    off = np.concatenate([[0], np.cumsum(PE)])
    assert off[-1] * 2 == len(d["edge_n"]) and off[-1] == len(d["edge_dS"])
    n = [d["edge_n"][2 * off[f]:2 * off[f + 1]].reshape(-1, 2) for f in range(F)]
    dS = [d["edge_dS"][off[f]:off[f + 1]] for f in range(F)]
    for f in range(F):
        L, R = d["edge_elem"][2 * f], d["edge_elem"][2 * f + 1]
        sL, sR = d["edge_side"][2 * f], d["edge_side"][2 * f + 1]
        inv = bool(d["edge_inverse"][f])
        if d["edge_marker"][f] == 0:
            tab[(L, sL)] = ("L", R, sR, inv, n[f], dS[f])
            tab[(R, sR)] = ("R", L, sL, inv, n[f][::-1] if inv else n[f], dS[f][::-1] if inv else dS[f])
        else:
            p = d["periodic_partner"][f]
            tab[(L, sL)] = ("B", d["edge_elem"][2 * p] if p >= 0 else -1, d["edge_side"][2 * p] if p >= 0 else 0,
                            inv, n[f], dS[f])
    assert len(tab) == 4 * E
    return tab


@pytest.mark.parametrize("nodes,N", [(O.LGL, 4), (O.LG, 3), (O.LG, "mixed"), (O.LGL, "mixed")])
def test_box_descriptor_matches_reference_construction(nodes, N):
    nx, ny = 5, 4
    if isinstance(N, str):   # a p-refined band (orders 3 / 5), periodic partners sharing an order
        N = np.where(np.tile(np.arange(nx), ny) % 2 == 1, 5, 3).astype(np.int32)
    m = hmesh.cartesian(nx, ny, -5.0, 5.0, -2.0, 3.0)
    orc = O.Oracle(m, N, nodes=nodes, bcs=hmesh.periodic_bcs_cartesian())
    ref = orc.export_mesh()
    ours = hmesh.box_descriptor(nx, ny, -5.0, 5.0, -2.0, 3.0, N, nodes)
    for k in ("Ja", "jac", "x", "volume", "vertices"):
        np.testing.assert_allclose(ours[k], ref[k], rtol=1e-13, atol=1e-13)
    ta, tb = side_table(ours), side_table(ref)
    for key, va in ta.items():
        vb = tb[key]
        assert va[:4] == vb[:4], key
        np.testing.assert_allclose(va[4], vb[4], atol=1e-15)
        np.testing.assert_allclose(va[5], vb[5], rtol=1e-14)


def test_library_nodes_match_oracle():
    for nodes in (O.LG, O.LGL):
        for N in range(1, 9):
            xi, w = lib.nodes(N, nodes)
            orc = O.Oracle(hmesh.cartesian(1, 1, 0.0, 1.0, 0.0, 1.0), N, nodes=nodes,
                           bcs=hmesh.periodic_bcs_cartesian())
            X = orc.coords()[:N + 1, 0]
            np.testing.assert_allclose(xi, X, rtol=0, atol=1e-15)
            assert abs(w.sum() - 1.0) < 1e-15


@pytest.mark.parametrize("case", ["cylinder", "ogrid", "periodic"])
def test_general_builder_matches_reference_construction(case):
    """build_descriptor (curved edges, LEFT/RIGHT orientation, periodic pairing) vs the oracle's mesh export."""
    from cases_util import load_mesh
    if case == "cylinder":
        m, N, nodes, pp = load_mesh("CylinderBench"), 5, O.LGL, ()
        bcs = [dict(type=O.BC_DIRICHLET)] * 4 + [dict(type=O.BC_EULERWALL)]
    elif case == "ogrid":
        m, N, nodes, pp = hmesh.ogrid(6, 12, 0.5, 10.0, 1.2), 3, O.LG, ()
        bcs = [dict(type=O.BC_EULERWALL), dict(type=O.BC_DIRICHLET)]
    else:
        m, N, nodes, pp = load_mesh("VortexTransportCase"), 4, O.LGL, [(1, 2, 0), (3, 4, 1)]
        bcs = hmesh.periodic_bcs_cartesian()
    ref = O.Oracle(m, N, nodes=nodes, bcs=bcs, mach=0.3).export_mesh()
    ours = hmesh.build_descriptor(m, N, nodes, periodic_pairs=pp)
    for k in ("Ja", "jac", "x", "volume", "vertices", "edge_invh"):
        scale = max(1.0, float(np.max(np.abs(ref[k]))))
        np.testing.assert_allclose(ours[k], ref[k], rtol=0, atol=1e-13 * scale, err_msg=k)
    ta, tb = side_table(ours), side_table(ref)
    for key, va in ta.items():
        vb = tb[key]
        assert va[:4] == vb[:4], key
        np.testing.assert_allclose(va[4], vb[4], atol=1e-13)
        np.testing.assert_allclose(va[5], vb[5], rtol=1e-13)


@pytest.mark.parametrize("kind", ["box", "ogrid"])
def test_locate_points_for_probes(kind):
    """mesh.locate recovers element and reference coordinates of points placed at known nodes (Gauss
    nodes are interior, so the element is unique), on a box and on a curved O-grid."""
    import horses2d_b200 as hg
    N = 4
    if kind == "box":
        d = hmesh.box_descriptor(5, 4, -1.0, 1.5, 0.0, 2.0, N, hg.NODES_LG)
    else:
        d = hmesh.build_descriptor(hmesh.ogrid(4, 12, 0.5, 3.0, 1.2), N, hg.NODES_LG)
    xi, _ = hg.lib.nodes(N, hg.NODES_LG)
    X = np.asarray(d["x"]).reshape(-1, (N + 1) ** 2, 2)
    rng = np.random.default_rng(3)
    picks = [(int(e), int(i), int(j)) for e, i, j in zip(rng.integers(0, X.shape[0], 12), rng.integers(0, N + 1, 12),
                                                          rng.integers(0, N + 1, 12))]
    pts = np.array([X[e, j * (N + 1) + i] for e, i, j in picks])
    el, xe = hmesh.locate(d, pts, hg.NODES_LG)
    for (e, i, j), ek, (a, b) in zip(picks, el, xe):
        assert ek == e
        assert abs(a - xi[i]) < 1e-10 and abs(b - xi[j]) < 1e-10
    with pytest.raises(ValueError):
        hmesh.locate(d, [[100.0, 100.0]], hg.NODES_LG)


@pytest.mark.parametrize("name", ["VortexTransportBench", "VortexTransportCase", "CylinderBench", "RampBench",
                                  "CouetteBench", "ShockWave"])
def test_library_connectivity_matches_mesh_file_construction(name):
    """hg_mesh_connectivity (O(E), C++ in the library) gives the lists of the reference's MeshFile
    construction -- edge order and orientation, subdivided (hanging-node) edges, elements of each
    edge, markers, curved-edge assignment and orientation -- as the oracle restates it, on every
    reference mesh the tests carry (the VortexTransport meshes have hanging nodes, the cylinder
    curved edges)."""
    from cases_util import load_mesh
    from oracle import oracle as O
    m = load_mesh(name)
    n_markers = int(np.max(m["bdry_marker"]))
    orc = O.Oracle(m, 2, nodes=O.LG, riemann=O.ROE, mach=0.3, bcs=[dict(type=O.BC_EULERWALL)] * n_markers)
    n_curved = int(np.asarray(m.get("curved_edges", np.zeros((0, 2)))).reshape(-1, 2).shape[0])
    pts, els, mk, ce, ci = orc.mesh_lists(n_curved)
    c = hmesh.connectivity(m)
    np.testing.assert_array_equal(c["points_of_edges"], pts)
    np.testing.assert_array_equal(c["elements_of_edges"], els)
    np.testing.assert_array_equal(c["edge_marker"], mk)
    np.testing.assert_array_equal(c["curved_edges"], ce)
    np.testing.assert_array_equal(c["curve_inverted"], ci)
    if name == "VortexTransportBench":
        assert np.any(pts[:, 2] > 0)            # hanging nodes merged into subdivided edges


def test_library_connectivity_scales_linearly():
    """A 1024 x 1024 quad mesh (the Kelvin-Helmholtz workload's size) is connected in seconds."""
    import time
    n = 1024
    ij = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1) + 1
    quads = np.stack([ij[:-1, :-1], ij[:-1, 1:], ij[1:, 1:], ij[1:, :-1]], -1).reshape(-1, 4)
    sides = [np.stack([ij[0, :-1], ij[0, 1:]], 1), np.stack([ij[-1, :-1], ij[-1, 1:]], 1),
             np.stack([ij[:-1, 0], ij[1:, 0]], 1), np.stack([ij[:-1, -1], ij[1:, -1]], 1)]
    m = dict(points=np.zeros(((n + 1) ** 2, 2)), quads=quads, bdry_edges=np.concatenate(sides),
             bdry_marker=np.repeat(np.arange(1, 5, dtype=np.int32), n))
    t0 = time.perf_counter()
    c = hmesh.connectivity(m)
    el = time.perf_counter() - t0
    assert len(c["edge_marker"]) == 2 * n * (n + 1) and int((c["edge_marker"] == 3).sum()) == n
    assert np.all(c["elements_of_edges"][c["edge_marker"] == 0][:, 1] > 0)
    assert el < 20.0
