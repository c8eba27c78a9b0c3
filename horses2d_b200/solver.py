"""Host-side mirror of the reference's time-derivative and time-scheme interface.

``GpuDGSEM`` wraps one libhorsesgpu context.  Its methods correspond to the
reference procedures a HORSES2D driver calls on the hot path:

=========================================  =====================================================
reference (Solver/src/...)                 here
=========================================  =====================================================
DGSpatial_computeTimeDerivative            ``compute_time_derivative(t)``
 (Approximation/DGSpatialDiscretizationMethods.f90:94-116)
TimeScheme / TimeIntegrator_WilliamsonRK3  ``time_step(scheme, t, dt)``
 (Approximation/DGTimeIntegrator.f90:71-83, 263-365)
TimeIntegrator_EstimateTimeStep            ``estimate_time_step(cfl, dt_cap)``
 (DGTimeIntegrator.f90:462-511)
Mesh_ComputeResiduals                      ``residuals()``
 (Mesh/QuadMesh_Auxiliars.incf:22-38)
Storage%Q read/write (Generic/Storage.f90)  ``set_state(Q)`` / ``state()``
=========================================  =====================================================

Errors raise ``HorsesGpuError`` carrying the library's message (the reference
stops the program instead).
"""
import ctypes as C
import os

import numpy as np

from . import _lib as L
from . import restart


class HorsesGpuError(RuntimeError):
    """An error status of the library; `status` is its code (L.STATUS_CRASHED: the stepped state is no
    longer physical)."""
    status = 1

    pass


def _arr(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class GpuDGSEM:
    """One mesh + physics + resident state on the GPU."""

    def __init__(self, mesh, *, mach, node_type=L.NODES_LGL, riemann=L.ROE, bcs=(), precision=L.PREC_FP64,
                 reynolds=0.0, prandtl=0.72, navier_stokes=0, viscous=L.BR1, ip_method=L.SIPG, sigma0_ip=1.0,
                 pressure_ref=101325.0, temperature_ref=273.15, reynolds_length=1.0, gamma=1.4, av_type=L.AV_NONE,
                 av_intensity=1.0):
        lib = L.load()
        self._keep = []
        md = L.MeshDesc()
        md.n_elements = int(len(mesh["N"]))
        md.n_edges = int(len(mesh["edge_marker"]))

        def put(field, key, dtype, ctype, optional=False):
            if key not in mesh or mesh[key] is None:
                if not optional:
                    raise HorsesGpuError(f"mesh descriptor lacks '{key}'")
                setattr(md, field, C.cast(None, C.POINTER(ctype)))
                return
            a = _arr(mesh[key], dtype)
            self._keep.append(a)
            setattr(md, field, a.ctypes.data_as(C.POINTER(ctype)))

        put("N", "N", np.int32, C.c_int32)
        put("Ja", "Ja", np.float64, C.c_double)
        put("jac", "jac", np.float64, C.c_double)
        put("x", "x", np.float64, C.c_double, True)
        put("volume", "volume", np.float64, C.c_double, True)
        put("vertices", "vertices", np.float64, C.c_double, True)
        put("edge_elem", "edge_elem", np.int32, C.c_int32)
        put("edge_side", "edge_side", np.int32, C.c_int32)
        put("edge_inverse", "edge_inverse", np.int32, C.c_int32)
        put("edge_marker", "edge_marker", np.int32, C.c_int32)
        put("edge_n", "edge_n", np.float64, C.c_double)
        put("edge_dS", "edge_dS", np.float64, C.c_double)
        put("periodic_partner", "periodic_partner", np.int32, C.c_int32, True)
        put("edge_invh", "edge_invh", np.float64, C.c_double, True)
        md.n_mortars = int(len(np.asarray(mesh.get("mortar_elem", ()))) // 3)
        for f, dt, ct in (("mortar_elem", np.int32, C.c_int32), ("mortar_side", np.int32, C.c_int32),
                          ("mortar_flip", np.int32, C.c_int32), ("mortar_n", np.float64, C.c_double),
                          ("mortar_dS", np.float64, C.c_double), ("mortar_invh", np.float64, C.c_double)):
            put(f, f, dt, ct, True)
        ph = L.PhysicsDesc(node_type=node_type, riemann=riemann, navier_stokes=navier_stokes, viscous=viscous,
                           ip_method=ip_method, sigma0_ip=sigma0_ip, mach=mach, reynolds=reynolds,
                           prandtl=prandtl, pressure_ref=pressure_ref, temperature_ref=temperature_ref, reynolds_length=reynolds_length, gamma=gamma,
                           gas_R=287.15, av_type=av_type, av_intensity=av_intensity)
        barr = (L.BCDesc * max(1, len(bcs)))()
        for k, b in enumerate(bcs):
            barr[k].type = b["type"]
            barr[k].riemann = b.get("riemann", L.INTERIOR)
            st = b.get("state", (0.0, 0.0, 0.0, 0.0))
            for i in range(4):
                barr[k].state[i] = st[i]
            barr[k].wall_T = b.get("wall_T", 1.0)
            wv = b.get("wall_v", (0.0, 0.0))
            barr[k].wall_v[0], barr[k].wall_v[1] = wv[0], wv[1]
            barr[k].wall_type = b.get("wall_type", 2)
            barr[k].outflow_type = b.get("outflow_type", 1)
            barr[k].nd_mode = b.get("mode", 0)
            barr[k].nd_outflow_total = b.get("outflow_total", 0)
        self._keep.append(barr)
        h = C.c_void_p()
        rc = lib.hg_create(C.byref(md), C.byref(ph), barr, len(bcs), precision, C.byref(h))
        if rc != 0:
            raise HorsesGpuError(lib.hg_last_error(None).decode())
        self._h = h
        self._lib = lib
        self.ndof = lib.hg_ndof(h)
        self.precision = precision

    def _check(self, rc):
        if rc != 0:
            err = HorsesGpuError(self._lib.hg_last_error(self._h).decode())
            err.status = rc
            raise err

    def close(self):
        if getattr(self, "_h", None):
            self._lib.hg_destroy(self._h)
            self._h = None

    __del__ = close

    # --- Storage%Q ---------------------------------------------------------
    def set_state(self, Q):
        Q = _arr(Q, np.float64).ravel()
        self._check(self._lib.hg_set_state(self._h, Q.ctypes.data_as(L.F64P), Q.size))

    def state(self, out=None):
        """Storage%Q of the resident state; `out` (contiguous float64, e.g. a pinned host buffer)
        receives it instead of a new array."""
        Q = np.empty(self.ndof) if out is None else out
        if Q.dtype != np.float64 or Q.size != self.ndof or not Q.flags.c_contiguous:
            raise HorsesGpuError("state buffer must be contiguous float64 of ndof values")
        self._check(self._lib.hg_get_state(self._h, Q.ctypes.data_as(L.F64P), Q.size))
        return Q

    # --- hot path ----------------------------------------------------------
    def compute_time_derivative(self, t=0.0, return_qdot=True):
        if return_qdot:
            out = np.empty(self.ndof)
            self._check(self._lib.hg_time_derivative(self._h, t, out.ctypes.data_as(L.F64P)))
            return out
        self._check(self._lib.hg_time_derivative(self._h, t, None))
        return None

    def time_step(self, scheme, t, dt):
        self._check(self._lib.hg_time_step(self._h, scheme, t, dt))

    def time_steps(self, scheme, n_steps, t0, dt):
        self._check(self._lib.hg_time_steps(self._h, scheme, n_steps, t0, dt))

    def residuals(self):
        r = np.zeros(4)
        self._check(self._lib.hg_residuals(self._h, r.ctypes.data_as(L.F64P)))
        return r

    def health(self):
        """(bits, element) of the device health word: HEALTH_* bits (0: clean) and one offending
        element (-1 when clean)."""
        b, e = C.c_int32(0), C.c_int32(-1)
        self._check(self._lib.hg_health(self._h, C.byref(b), C.byref(e)))
        return b.value, e.value

    def set_health_policy(self, fatal_bits):
        """HEALTH_* bits that make the step calls fail (default HEALTH_NONFINITE)."""
        self._check(self._lib.hg_set_health_policy(self._h, fatal_bits))

    def estimate_time_step(self, cfl, dt_cap):
        d = C.c_double(0.0)
        self._check(self._lib.hg_estimate_dt(self._h, cfl, dt_cap, C.byref(d)))
        return d.value

    def integrate(self, scheme, *, transient, t0, t_end, max_iter, cfl, dt_cap, residual_target=0.0,
                  estimate_interval=100, initial_iteration=0, autosave_interval=0, solution_file=None):
        """The reference's integration loop (Approximation/DGTimeIntegrator.f90:173-247) around the
        library's steps: dt from EstimateTimeStep, re-estimated every `estimate_interval` iterations;
        transient mode clips the last step to end exactly at t_end; steady mode stops when the largest
        residual falls below residual_target.  The host replays the loop's time arithmetic exactly and
        issues runs of ordinary transient steps through the multi-step call.  Iterations are numbered
        from initial_iteration + 1 (the iteration a restart file holds); with autosave_interval > 0 a
        restart file named after solution_file is written every that many iterations, and with a
        solution_file the final state is saved there.  Returns (last iteration, t)."""
        def same(a, b):   # the reference's almost-equal test of the final time
            eps = np.finfo(float).eps
            if a == 0.0 or b == 0.0:
                return abs(a - b) <= 2.0 * eps
            return abs(b - a) <= 2.0 * eps * max(abs(a), abs(b))

        t = t0
        dt = self.estimate_time_step(cfl, dt_cap)
        pending, t_first = 0, t0      # ordinary steps of the current dt not yet issued

        def flush():
            nonlocal pending
            if pending:
                self.time_steps(scheme, pending, t_first, dt)
                pending = 0

        it = initial_iteration
        for it in range(initial_iteration + 1, initial_iteration + max_iter + 1):
            if transient and t + dt >= t_end:
                flush()
                dt = t_end - t
                self.time_step(scheme, t, dt)
            elif transient:
                if pending == 0:
                    t_first = t
                pending += 1
            else:
                self.time_step(scheme, t, dt)
            t = t + dt
            if transient and same(t, t_end):
                break
            if autosave_interval > 0 and solution_file and it % autosave_interval == 0:
                flush()
                self.save_restart(restart.autosave_name(solution_file, it), t, it, wait=False)
            if it % estimate_interval == 0:
                flush()
                dt = self.estimate_time_step(cfl, dt_cap)
            if not transient and np.max(np.abs(self.residuals())) < residual_target:
                break
        flush()
        self.restart_wait()
        if solution_file:
            self.save_restart(solution_file, t, it)
        return it, t

    # --- restart files (*.HiORst) --------------------------------------------
    def save_restart(self, path, t, iteration, wait=True):
        """The resident state, t and iter to a restart file (TimeIntegrator_Autosave).  wait=False
        returns at once: the state is copied on the stream and a host thread writes the file while
        stepping goes on (restart_wait() or the next save waits for it)."""
        if not wait:
            self._check(self._lib.hg_save_restart_async(self._h, os.fsencode(path), float(t), int(iteration)))
            return
        self._check(self._lib.hg_restart_wait(self._h))
        if self._lib.hg_save_restart(self._h, os.fsencode(path), float(t), int(iteration)) != 0:
            raise OSError(self._lib.hg_restart_last_error().decode())

    def restart_wait(self):
        """Wait for an asynchronous restart write; raises its error, if any."""
        self._check(self._lib.hg_restart_wait(self._h))

    def load_restart(self, path):
        """A restart file into the resident state (DGSEM_loadRestartFile); returns (t, iter)."""
        t, it = C.c_double(0.0), C.c_int32(0)
        if self._lib.hg_load_restart(self._h, os.fsencode(path), C.byref(t), C.byref(it)) != 0:
            raise OSError(self._lib.hg_restart_last_error().decode())
        return t.value, it.value

    # --- plumbing ----------------------------------------------------------
    def set_stream(self, cuda_stream_handle):
        self._check(self._lib.hg_set_stream(self._h, C.c_void_p(cuda_stream_handle)))

    def synchronize(self):
        self._check(self._lib.hg_synchronize(self._h))

    def device_state_ptr(self):
        return self._lib.hg_device_state(self._h)

    def launch_count(self):
        return self._lib.hg_launch_count(self._h)

    def profile(self, enable=True):
        """Start (clearing the totals) or stop per-kernel CUDA-event timing."""
        self._check(self._lib.hg_profile(self._h, 1 if enable else 0))

    def kernel_times(self):
        """{kernel class: (total ms, launches)} since profile(True)."""
        n = len(L.KERNEL_KINDS)
        ms, cnt = (C.c_double * n)(), (C.c_int64 * n)()
        self._check(self._lib.hg_kernel_times(self._h, ms, cnt, n))
        return {k: (ms[i], cnt[i]) for i, k in enumerate(L.KERNEL_KINDS)}

    # --- shock sensor of the artificial dissipation -------------------------
    def set_sensor(self, kind, s0=float("nan"), kappa=float("nan"), mlp=None, lo=None, hi=None):
        """Indicator that sets the artificial viscosity: L.SENSOR_JUMPS (reference), _MODAL, _LEARNED."""
        def f32(a, n):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float32).ravel()
            if a.size != n:
                raise HorsesGpuError(f"expected {n} values, got {a.size}")
            self._keep.append(a)
            return a.ctypes.data_as(L.F32P)
        self._check(self._lib.hg_set_sensor(self._h, kind, s0, kappa, f32(mlp, L.MLP_PARAMS),
                                            f32(lo, L.SENSOR_FEATURES), f32(hi, L.SENSOR_FEATURES)))

    def sensor_eval(self):
        """(features [n_el,16] float32, out [n_el,4]: modal G, learned G, OOD flag, G in use)."""
        n = self.info()["n_elements"]
        f = np.zeros((n, L.SENSOR_FEATURES), np.float32)
        o = np.zeros((n, 4))
        self._check(self._lib.hg_sensor_eval(self._h, f.ctypes.data_as(L.F32P), o.ctypes.data_as(L.F64P)))
        return f, o

    def set_boundary_state(self, zone, uB):
        """Per-node states of Dirichlet zone `zone` (1-based marker): the reference's boundary-condition
        function evaluated at the zone's edge nodes, [edges x (N+1)] x 4 in mesh edge order."""
        uB = np.ascontiguousarray(uB, dtype=np.float64).ravel()
        self._check(self._lib.hg_set_boundary_state(self._h, int(zone), uB.ctypes.data_as(L.F64P), uB.size))

    def surface_integrals(self, zone):
        """Dimensionless surface integrals of zone `zone` over the traces of the last residual evaluation:
        dict(surface, pressure, pressure_force (2), viscous_force (2), mass_flow, flow)."""
        out = np.zeros(8)
        self._check(self._lib.hg_surface_integrals(self._h, int(zone), out.ctypes.data_as(L.F64P)))
        return dict(surface=out[0], pressure=out[1], pressure_force=out[2:4].copy(), viscous_force=out[4:6].copy(),
                    mass_flow=out[6], flow=out[7])

    def probes(self, elements, xi_eta):
        """Resident state [n, 4] at probe points given by element (0-based) and reference coordinates [n, 2]
        in [0,1] (mesh.locate turns physical points into these)."""
        el = np.ascontiguousarray(elements, dtype=np.int32).ravel()
        xe = np.ascontiguousarray(xi_eta, dtype=np.float64).reshape(-1, 2)
        if xe.shape[0] != el.size:
            raise HorsesGpuError("one (xi, eta) pair per probe")
        out = np.zeros((el.size, 4))
        self._check(self._lib.hg_probes(self._h, el.size, el.ctypes.data_as(L.I32P), xe.ctypes.data_as(L.F64P),
                                        out.ctypes.data_as(L.F64P)))
        return out

    def autotune(self, trials=10):
        """Time the elements-per-CTA variants on the resident state (RK3 steps with dt = 0; the state is
        kept) and keep the fastest: {"chosen": variant, "ms": [ms per step per variant -- per residual
        evaluation on a mixed-order mesh], "tiling": get_tiling()}."""
        ch = C.c_int32(0)
        ms = np.zeros(L.TILINGS)
        self._check(self._lib.hg_autotune(self._h, int(trials), C.byref(ch), ms.ctypes.data_as(L.F64P)))
        return {"chosen": ch.value, "ms": ms.tolist(), "tiling": self.get_tiling()}

    def set_tiling(self, variant):
        self._check(self._lib.hg_set_tiling(self._h, int(variant)))

    def get_tiling(self):
        """{variant, elements per CTA, threads per CTA} of the stage kernels."""
        out = (C.c_int32 * 3)()
        self._check(self._lib.hg_get_tiling(self._h, out))
        return dict(variant=out[0], elements_per_cta=out[1], threads_per_cta=out[2])

    def element_viscosity(self):
        n = self.info()["n_elements"]
        mu = np.zeros(n)
        self._check(self._lib.hg_element_viscosity(self._h, mu.ctypes.data_as(L.F64P)))
        return mu

    def info(self):
        """{N, n_elements, affine, precision} of the context."""
        out = (C.c_int32 * 4)()
        self._check(self._lib.hg_info(self._h, out))
        return dict(N=out[0], n_elements=out[1], affine=bool(out[2]), precision=out[3])


class GpuGroup:
    """Independent contexts stepped together by one CUDA graph (hg_group_*): an ensemble packed into
    one GpuDGSEM per polynomial order.  The members must share one stream and have their state set."""

    def __init__(self, members):
        self.members = list(members)   # keeps the contexts alive while the group exists
        lib = L.load()
        arr = (C.c_void_p * len(self.members))(*[m._h.value for m in self.members])
        h = C.c_void_p()
        if lib.hg_group_create(arr, len(self.members), C.byref(h)) != 0:
            raise HorsesGpuError(lib.hg_group_last_error(None).decode())
        self._h = h
        self._lib = lib

    def time_steps(self, scheme, n_steps, t0, dt):
        if self._lib.hg_group_time_steps(self._h, int(scheme), int(n_steps), float(t0), float(dt)) != 0:
            raise HorsesGpuError(self._lib.hg_group_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.hg_group_destroy(self._h)
            self._h = None

    __del__ = close
