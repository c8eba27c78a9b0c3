"""ctypes wrapper of the CPU FP64 oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the HORSES2D residual and time integrator in C++
(``oracle/*.cpp``).  Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` import this module, and only as the checker.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

BC_PERIODIC, BC_DIRICHLET, BC_EULERWALL, BC_VISCOUSWALL, BC_FARFIELD, BC_PRESSUREOUTLET = 1, 2, 3, 4, 5, 6
BC_NEWDIRICHLET = 7
ROE, HLL, EXACT, LXF, INTERIOR = 0, 1, 2, 3, -1
LG, LGL = 1, 2
EULER, RK3, RK5 = 0, 1, 2
BR1, IP = 0, 1
AV_NONE, AV_LAPLACIAN, AV_PHYSICAL = 0, 1, 2
IND_JUMPS, IND_MODAL, IND_EXTERNAL = 0, 1, 2


class OrBC(C.Structure):
    _fields_ = [("type", C.c_int), ("riemann", C.c_int), ("periodic_dir", C.c_int), ("connected_marker", C.c_int),
                ("pressure", C.c_double), ("temperature", C.c_double), ("mach", C.c_double), ("aoa_deg", C.c_double),
                ("wall_type", C.c_int), ("wall_T", C.c_double), ("wall_v", C.c_double * 2), ("outflow_type", C.c_int),
                ("nd_mode", C.c_int), ("nd_outflow_total", C.c_int)]


class OrCase(C.Structure):
    _fields_ = [("nodes", C.c_int), ("riemann", C.c_int), ("navier_stokes", C.c_int), ("viscous", C.c_int),
                ("ip_method", C.c_int), ("sigma0_ip", C.c_double), ("sigma1_ip", C.c_double),
                ("mach", C.c_double), ("reynolds", C.c_double), ("prandtl", C.c_double),
                ("pressure_ref", C.c_double), ("temperature_ref", C.c_double), ("reynolds_length", C.c_double),
                ("n_markers", C.c_int), ("bcs", C.POINTER(OrBC)), ("av_type", C.c_int), ("av_intensity", C.c_double),
                ("av_indicator", C.c_int), ("av_s0", C.c_double), ("av_kappa", C.c_double)]


class OrMesh(C.Structure):
    _fields_ = [("n_nodes", C.c_int), ("n_elements", C.c_int), ("n_bdry_edges", C.c_int),
                ("points", C.POINTER(C.c_double)), ("quads", C.POINTER(C.c_int)),
                ("bdry_edges", C.POINTER(C.c_int)), ("bdry_marker", C.POINTER(C.c_int)),
                ("n_curved", C.c_int), ("curve_np1", C.c_int), ("curved_edges", C.POINTER(C.c_int)),
                ("curve_x", C.POINTER(C.c_double)), ("curve_y", C.POINTER(C.c_double)),
                ("poly_order", C.POINTER(C.c_int))]


_lib = None


def build():
    """Compile the oracle with its Makefile (gcc, no CUDA)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, dp, ip, d, i = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_double, C.c_int
        L.or_create.restype = vp
        L.or_create.argtypes = [C.POINTER(OrCase), C.POINTER(OrMesh), C.c_char_p, i]
        L.or_destroy.argtypes = [vp]
        L.or_ndof.restype = C.c_int64
        L.or_ndof.argtypes = [vp]
        for name in ("or_n_elements", "or_n_edges"):
            getattr(L, name).restype = i
            getattr(L, name).argtypes = [vp]
        L.or_element_orders.argtypes = [vp, ip]
        for name in ("or_node_coords", "or_set_state", "or_get_state", "or_get_qdot"):
            getattr(L, name).argtypes = [vp, dp]
        L.or_time_derivative.argtypes = [vp, d]
        L.or_time_step.argtypes = [vp, i, d, d]
        L.or_estimate_dt.restype = d
        L.or_estimate_dt.argtypes = [vp, d, d]
        L.or_residuals.argtypes = [vp, dp]
        L.or_integrate.restype = i
        L.or_integrate.argtypes = [vp, i, i, d, d, i, d, d, d, dp]
        L.or_ref_values.argtypes = [vp, dp]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_set_av_g.argtypes = [vp, dp]
        L.or_set_minmax_nan.argtypes = [C.c_int]
        L.or_zone_state.argtypes = [vp, C.c_int, dp]
        L.or_av_viscosity.argtypes = [vp, dp]
        L.or_element_geometry.argtypes = [vp, dp, dp, dp]
        L.or_edge_count_by_type.restype = i
        L.or_edge_count_by_type.argtypes = [vp, i]
        L.or_export_mesh.restype = i
        L.or_export_mesh.argtypes = [vp, ip, dp, dp, dp, dp, dp, ip, ip, ip, ip, dp, dp, ip, dp, ip, ip, ip, dp, dp, dp]
        L.or_export_sizes.restype = None
        L.or_export_sizes.argtypes = [vp, ip]
        L.or_mesh_lists.restype = i
        L.or_mesh_lists.argtypes = [vp, ip, ip, ip, ip, ip]
        L.or_probe.restype = i
        L.or_probe.argtypes = [vp, i, C.c_double, C.c_double, dp]
        L.or_surface_integrals.restype = i
        L.or_surface_integrals.argtypes = [vp, i, dp]
        L.or_zone_edge_nodes.restype = i
        L.or_zone_edge_nodes.argtypes = [vp, i, dp]
        L.or_set_zone_state.argtypes = [vp, i, dp]
        _lib = L
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Oracle:
    """One oracle instance: mesh + physics + state, mirroring a DGSEM_t run."""

    def __init__(self, mesh, poly_order, *, nodes=LGL, riemann=ROE, mach=0.5, reynolds=0.0, prandtl=0.72,
                 pressure_ref=101325.0, temperature_ref=273.15, reynolds_length=1.0, bcs=(), navier_stokes=0,
                 viscous=BR1, ip_method=0, sigma0_ip=1.0, sigma1_ip=0.0, av_type=0, av_intensity=1.0, av_indicator=0, av_s0=None,
                 av_kappa=1.0):
        self._keep = []
        m = OrMesh()
        pts = np.ascontiguousarray(mesh["points"], dtype=np.float64)
        quads = np.ascontiguousarray(mesh["quads"], dtype=np.int32)
        be = np.ascontiguousarray(mesh["bdry_edges"], dtype=np.int32).reshape(-1, 2)
        bm = np.ascontiguousarray(mesh["bdry_marker"], dtype=np.int32)
        order = np.ascontiguousarray(np.broadcast_to(np.asarray(poly_order, dtype=np.int32), (quads.shape[0],)))
        self._keep += [pts, quads, be, bm, order]
        m.n_nodes, m.n_elements, m.n_bdry_edges = pts.shape[0], quads.shape[0], be.shape[0]
        m.points, m.quads = _p(pts, C.c_double), _p(quads, C.c_int)
        m.bdry_edges, m.bdry_marker = _p(be, C.c_int), _p(bm, C.c_int)
        m.poly_order = _p(order, C.c_int)
        if "curved_edges" in mesh and len(mesh["curved_edges"]):
            ce = np.ascontiguousarray(mesh["curved_edges"], dtype=np.int32)
            cx = np.ascontiguousarray(mesh["curve_x"], dtype=np.float64)
            cy = np.ascontiguousarray(mesh["curve_y"], dtype=np.float64)
            self._keep += [ce, cx, cy]
            m.n_curved, m.curve_np1 = ce.shape[0], cx.shape[1]
            m.curved_edges, m.curve_x, m.curve_y = _p(ce, C.c_int), _p(cx, C.c_double), _p(cy, C.c_double)
        else:
            m.n_curved, m.curve_np1 = 0, 0
        bc_arr = (OrBC * max(1, len(bcs)))()
        for k, b in enumerate(bcs):
            bb = bc_arr[k]
            bb.type = b["type"]
            bb.riemann = b.get("riemann", INTERIOR)
            bb.periodic_dir = b.get("periodic_dir", 0)
            bb.connected_marker = b.get("connected_marker", 0)
            bb.pressure = b.get("pressure", -1.0)
            bb.temperature = b.get("temperature", -1.0)
            bb.mach = b.get("mach", -1.0)
            bb.aoa_deg = b.get("aoa_deg", 0.0)
            bb.wall_type = b.get("wall_type", 2)
            bb.wall_T = b.get("wall_T", temperature_ref)
            wv = b.get("wall_v", (0.0, 0.0))
            bb.wall_v[0], bb.wall_v[1] = wv[0], wv[1]
            bb.outflow_type = b.get("outflow_type", 1)
            bb.nd_mode = b.get("mode", 0)
            bb.nd_outflow_total = b.get("outflow_total", 0)
        self._keep.append(bc_arr)
        c = OrCase(nodes=nodes, riemann=riemann, navier_stokes=navier_stokes, viscous=viscous, ip_method=ip_method,
                   sigma0_ip=sigma0_ip, sigma1_ip=sigma1_ip, mach=mach, reynolds=reynolds, prandtl=prandtl,
                   pressure_ref=pressure_ref, temperature_ref=temperature_ref, reynolds_length=reynolds_length,
                   n_markers=len(bcs), bcs=C.cast(bc_arr, C.POINTER(OrBC)), av_type=av_type,
                   av_intensity=av_intensity, av_indicator=av_indicator,
                   av_s0=(np.log10(1.0 / (int(np.max(poly_order)) + 1) ** 4) if av_s0 is None else av_s0),
                   av_kappa=av_kappa)
        err = C.create_string_buffer(512)
        self.h = lib().or_create(C.byref(c), C.byref(m), err, 512)
        if not self.h:
            raise RuntimeError("oracle: " + err.value.decode())
        self.ndof = lib().or_ndof(self.h)
        self.n_elements = lib().or_n_elements(self.h)
        self.orders = np.zeros(self.n_elements, dtype=np.int32)
        lib().or_element_orders(self.h, _p(self.orders, C.c_int))
        rv = np.zeros(8)
        lib().or_ref_values(self.h, _p(rv, C.c_double))
        self.ref = dict(rho=rv[0], a=rv[1], p=rv[2], V=rv[3], T=rv[4], L=rv[5], mu=rv[6], invSqrtGammaMach=rv[7])

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    def coords(self):
        X = np.zeros((self.ndof // 4, 2))
        lib().or_node_coords(self.h, _p(X, C.c_double))
        return X

    def set_state(self, Q):
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        assert Q.size == self.ndof
        lib().or_set_state(self.h, _p(Q, C.c_double))

    def state(self):
        Q = np.zeros(self.ndof)
        lib().or_get_state(self.h, _p(Q, C.c_double))
        return Q

    def qdot(self):
        Q = np.zeros(self.ndof)
        lib().or_get_qdot(self.h, _p(Q, C.c_double))
        return Q

    def time_derivative(self, t=0.0):
        lib().or_time_derivative(self.h, t)
        return self.qdot()

    def time_step(self, scheme, t, dt):
        lib().or_time_step(self.h, scheme, t, dt)

    def estimate_dt(self, cfl, dt_cap):
        return lib().or_estimate_dt(self.h, cfl, dt_cap)

    def residuals(self):
        r = np.zeros(4)
        lib().or_residuals(self.h, _p(r, C.c_double))
        return r

    def zone_state(self, zone):
        """Dimensionless state of zone `zone` (1-based marker) as the oracle built it."""
        q = np.zeros(4)
        lib().or_zone_state(self.h, zone, _p(q, C.c_double))
        return q

    def set_av_g(self, G):
        """Per-element indicator G used by av_indicator=IND_EXTERNAL."""
        G = np.ascontiguousarray(G, dtype=np.float64)
        lib().or_set_av_g(self.h, _p(G, C.c_double))

    def av_viscosity(self):
        """Element artificial viscosity computed by the last time derivative."""
        mu = np.zeros(self.n_elements)
        lib().or_av_viscosity(self.h, _p(mu, C.c_double))
        return mu

    def integrate(self, scheme, *, transient=True, t0=0.0, t_end=1.0, max_iter=1000, cfl=0.1, dt_cap=0.01,
                  residual_target=1e-12):
        t = C.c_double(0.0)
        it = lib().or_integrate(self.h, scheme, 1 if transient else 0, t0, t_end, max_iter, cfl, dt_cap,
                                residual_target, C.byref(t))
        return it, t.value

    def geometry(self):
        n = self.ndof // 4
        Ja, jac, vol = np.zeros((n, 2, 2)), np.zeros(n), np.zeros(self.n_elements)
        lib().or_element_geometry(self.h, _p(Ja, C.c_double), _p(jac, C.c_double), _p(vol, C.c_double))
        return Ja, jac, vol

    def edge_count(self, kind):
        return lib().or_edge_count_by_type(self.h, kind)

    def zone_edge_nodes(self, zone):
        n = lib().or_zone_edge_nodes(self.h, zone, None)
        X = np.zeros((n, 2))
        lib().or_zone_edge_nodes(self.h, zone, _p(X, C.c_double))
        return X

    def surface_integrals(self, zone):
        """Dimensionless surface integrals of zone `zone` over the traces of the last residual
        evaluation: dict(surface, pressure, pressure_force (2), viscous_force (2), mass_flow, flow)."""
        out = np.zeros(8)
        if lib().or_surface_integrals(self.h, zone, _p(out, C.c_double)) != 0:
            raise ValueError(f"unknown zone {zone}")
        return dict(surface=out[0], pressure=out[1], pressure_force=out[2:4].copy(), viscous_force=out[4:6].copy(),
                    mass_flow=out[6], flow=out[7])

    def mesh_lists(self, n_curved):
        """(points [F,3], elements [F,3], marker [F], curve_edge [n_curved], curve_inv [n_curved]) of the
        mesh file as the reference's MeshFile builds them (1-based, list order)."""
        F = lib().or_mesh_lists(self.h, None, None, None, None, None)
        pts, els = np.zeros((F, 3), np.int32), np.zeros((F, 3), np.int32)
        mk, ce, ci = np.zeros(F, np.int32), np.zeros(max(n_curved, 1), np.int32), np.zeros(max(n_curved, 1), np.int32)
        lib().or_mesh_lists(self.h, _p(pts, C.c_int), _p(els, C.c_int), _p(mk, C.c_int), _p(ce, C.c_int),
                            _p(ci, C.c_int))
        return pts, els, mk, ce[:n_curved], ci[:n_curved]

    def probe(self, e, xi, eta):
        out = np.zeros(4)
        if lib().or_probe(self.h, int(e), float(xi), float(eta), _p(out, C.c_double)) != 0:
            raise ValueError(f"unknown element {e}")
        return out

    def set_zone_state(self, zone, uB):
        uB = np.ascontiguousarray(uB, dtype=np.float64)
        lib().or_set_zone_state(self.h, zone, _p(uB, C.c_double))

    def export_mesh(self):
        """The constructed mesh flattened like include/horses_gpu.h hg_mesh_desc (subdivided edges as
        the mortar list)."""
        E, n = self.n_elements, self.ndof // 4
        sz = np.zeros(4, np.int32)
        lib().or_export_sizes(self.h, _p(sz, C.c_int))
        F, FN, M, MN = (int(v) for v in sz)
        d = dict(N=np.zeros(E, np.int32), Ja=np.zeros(4 * n), jac=np.zeros(n), x=np.zeros(2 * n), volume=np.zeros(E),
                 vertices=np.zeros(8 * E), edge_elem=np.zeros(2 * F, np.int32), edge_side=np.zeros(2 * F, np.int32),
                 edge_inverse=np.zeros(F, np.int32), edge_marker=np.zeros(F, np.int32), edge_n=np.zeros(2 * FN),
                 edge_dS=np.zeros(FN), periodic_partner=np.zeros(F, np.int32), edge_invh=np.zeros(F),
                 mortar_elem=np.zeros(3 * M, np.int32), mortar_side=np.zeros(3 * M, np.int32),
                 mortar_flip=np.zeros(2 * M, np.int32), mortar_n=np.zeros(2 * MN), mortar_dS=np.zeros(MN),
                 mortar_invh=np.zeros(M))
        ip_, dp_ = C.c_int, C.c_double
        lib().or_export_mesh(self.h, *[_p(d[k], ip_ if d[k].dtype == np.int32 else dp_) for k in
                                       ("N", "Ja", "jac", "x", "volume", "vertices", "edge_elem", "edge_side",
                                        "edge_inverse", "edge_marker", "edge_n", "edge_dS", "periodic_partner",
                                        "edge_invh", "mortar_elem", "mortar_side", "mortar_flip", "mortar_n",
                                        "mortar_dS", "mortar_invh")])
        return d
