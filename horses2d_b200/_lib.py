"""ctypes binding of libhorsesgpu.so (C ABI declared in include/horses_gpu.h).

The shared library is built in-tree by ``horses2d_b200.build`` (nvcc, sm_100a).
There is no CPU fallback: if the library or a Blackwell GPU is missing, calls
raise.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhorsesgpu.so")

NODES_LG, NODES_LGL = 1, 2
ROE, HLL, EXACT, LXF, INTERIOR = 0, 1, 2, 3, -1
SCHEME_EULER, SCHEME_RK3, SCHEME_RK5 = 0, 1, 2
PREC_FP64, PREC_FP32 = 0, 1
BR1, IP = 0, 1
SIPG, NIPG, IIPG = 0, 1, 2
BC_PERIODIC, BC_DIRICHLET, BC_EULERWALL, BC_VISCOUSWALL, BC_FARFIELD, BC_PRESSUREOUTLET = 1, 2, 3, 4, 5, 6
BC_NEWDIRICHLET = 7
AV_NONE, AV_LAPLACIAN, AV_PHYSICAL = 0, 1, 2
STATUS_CRASHED = 2
HEALTH_NONFINITE, HEALTH_DENSITY, HEALTH_PRESSURE = 1, 2, 4

I32P = C.POINTER(C.c_int32)
F64P = C.POINTER(C.c_double)


class PhysicsDesc(C.Structure):
    _fields_ = [("node_type", C.c_int32), ("riemann", C.c_int32), ("navier_stokes", C.c_int32),
                ("viscous", C.c_int32), ("ip_method", C.c_int32), ("sigma0_ip", C.c_double),
                ("mach", C.c_double), ("reynolds", C.c_double), ("prandtl", C.c_double),
                ("pressure_ref", C.c_double), ("temperature_ref", C.c_double), ("reynolds_length", C.c_double),
                ("gamma", C.c_double), ("gas_R", C.c_double), ("av_type", C.c_int32), ("av_intensity", C.c_double)]


class BCDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("riemann", C.c_int32), ("state", C.c_double * 4), ("wall_T", C.c_double),
                ("wall_v", C.c_double * 2), ("wall_type", C.c_int32), ("outflow_type", C.c_int32),
                ("nd_mode", C.c_int32), ("nd_outflow_total", C.c_int32)]


class MeshDesc(C.Structure):
    _fields_ = [("n_elements", C.c_int32), ("n_edges", C.c_int32), ("N", I32P), ("Ja", F64P), ("jac", F64P),
                ("x", F64P), ("volume", F64P), ("vertices", F64P), ("edge_elem", I32P), ("edge_side", I32P),
                ("edge_inverse", I32P), ("edge_marker", I32P), ("edge_n", F64P), ("edge_dS", F64P),
                ("periodic_partner", I32P), ("edge_invh", F64P), ("n_mortars", C.c_int32),
                ("mortar_elem", I32P), ("mortar_side", I32P), ("mortar_flip", I32P), ("mortar_n", F64P),
                ("mortar_dS", F64P), ("mortar_invh", F64P)]


_lib = None
EXPORTED = ("hg_create", "hg_destroy", "hg_last_error", "hg_set_state", "hg_get_state", "hg_ndof",
            "hg_time_derivative", "hg_time_step", "hg_time_steps", "hg_residuals", "hg_estimate_dt",
            "hg_set_stream", "hg_synchronize", "hg_device_state", "hg_launch_count", "hg_nodes", "hg_info",
            "hg_profile", "hg_kernel_times", "hg_residuals_noalloc", "hg_set_sensor", "hg_sensor_eval",
            "hg_element_viscosity", "hg_mlp_forward", "hg_mlp_grad", "hg_mlp_train", "hg_set_boundary_state",
            "hg_autotune", "hg_set_tiling", "hg_get_tiling", "hg_group_create", "hg_group_destroy",
            "hg_group_time_steps", "hg_group_last_error", "hg_surface_integrals", "hg_probes",
            "hg_mesh_connectivity", "hg_mesh_last_error", "hg_write_restart", "hg_read_restart",
            "hg_save_restart", "hg_load_restart", "hg_restart_last_error", "hg_save_restart_async",
            "hg_restart_wait", "hg_health", "hg_set_health_policy")
SENSOR_JUMPS, SENSOR_MODAL, SENSOR_LEARNED = 0, 1, 2
SENSOR_FEATURES, MLP_PARAMS = 16, 1633
F32P = C.POINTER(C.c_float)
KERNEL_KINDS = ("stage", "gradient", "trace", "reduce", "speed", "face_flux", "mortar")
TILINGS = 2


def load():
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m horses2d_b200.build` "
                           "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.hg_create.restype = C.c_int
    L.hg_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(PhysicsDesc), C.POINTER(BCDesc), C.c_int32, C.c_int32,
                            C.POINTER(vp)]
    L.hg_destroy.argtypes = [vp]
    L.hg_last_error.restype = C.c_char_p
    L.hg_last_error.argtypes = [vp]
    L.hg_set_state.argtypes = [vp, F64P, C.c_int64]
    L.hg_get_state.argtypes = [vp, F64P, C.c_int64]
    L.hg_ndof.restype = C.c_int64
    L.hg_ndof.argtypes = [vp]
    L.hg_time_derivative.argtypes = [vp, C.c_double, F64P]
    L.hg_time_step.argtypes = [vp, C.c_int32, C.c_double, C.c_double]
    L.hg_time_steps.argtypes = [vp, C.c_int32, C.c_int32, C.c_double, C.c_double]
    L.hg_residuals.argtypes = [vp, F64P]
    L.hg_estimate_dt.argtypes = [vp, C.c_double, C.c_double, F64P]
    L.hg_set_stream.argtypes = [vp, vp]
    L.hg_synchronize.argtypes = [vp]
    L.hg_health.argtypes = [vp, I32P, I32P]
    L.hg_set_health_policy.argtypes = [vp, C.c_int32]
    L.hg_device_state.restype = C.c_void_p
    L.hg_device_state.argtypes = [vp]
    L.hg_launch_count.restype = C.c_int64
    L.hg_launch_count.argtypes = [vp]
    L.hg_nodes.argtypes = [C.c_int32, C.c_int32, F64P, F64P]
    L.hg_info.argtypes = [vp, I32P]
    L.hg_profile.argtypes = [vp, C.c_int32]
    L.hg_kernel_times.argtypes = [vp, F64P, C.POINTER(C.c_int64), C.c_int32]
    f32p = C.POINTER(C.c_float)
    L.hg_set_sensor.argtypes = [vp, C.c_int32, C.c_double, C.c_double, f32p, f32p, f32p]
    L.hg_sensor_eval.argtypes = [vp, f32p, F64P]
    L.hg_element_viscosity.argtypes = [vp, F64P]
    L.hg_set_boundary_state.argtypes = [vp, C.c_int32, F64P, C.c_int64]
    L.hg_autotune.argtypes = [vp, C.c_int32, I32P, F64P]
    L.hg_surface_integrals.argtypes = [vp, C.c_int32, F64P]
    L.hg_probes.argtypes = [vp, C.c_int32, I32P, F64P, F64P]
    L.hg_mesh_connectivity.argtypes = [C.c_int32, C.c_int32, I32P, C.c_int32, I32P, I32P, C.c_int32, I32P, C.c_int32,
                                       I32P, I32P, I32P, I32P, I32P, I32P]
    L.hg_mesh_last_error.argtypes = []
    L.hg_mesh_last_error.restype = C.c_char_p
    L.hg_write_restart.argtypes = [C.c_char_p, C.c_double, C.c_int32, F64P, C.c_int64, C.c_int32, C.c_int32]
    L.hg_read_restart.argtypes = [C.c_char_p, F64P, I32P, F64P, C.c_int64, C.POINTER(C.c_int64)]
    L.hg_save_restart.argtypes = [vp, C.c_char_p, C.c_double, C.c_int32]
    L.hg_load_restart.argtypes = [vp, C.c_char_p, F64P, I32P]
    L.hg_restart_last_error.argtypes = []
    L.hg_restart_last_error.restype = C.c_char_p
    L.hg_save_restart_async.argtypes = [vp, C.c_char_p, C.c_double, C.c_int32]
    L.hg_restart_wait.argtypes = [vp]
    L.hg_set_tiling.argtypes = [vp, C.c_int32]
    L.hg_get_tiling.argtypes = [vp, I32P]
    L.hg_group_create.argtypes = [C.POINTER(vp), C.c_int32, C.POINTER(vp)]
    L.hg_group_destroy.argtypes = [vp]
    L.hg_group_destroy.restype = None
    L.hg_group_time_steps.argtypes = [vp, C.c_int32, C.c_int32, C.c_double, C.c_double]
    L.hg_group_last_error.argtypes = [vp]
    L.hg_group_last_error.restype = C.c_char_p
    L.hg_mlp_forward.argtypes = [f32p, f32p, C.c_int64, f32p]
    L.hg_mlp_grad.argtypes = [f32p, f32p, f32p, f32p, C.c_int64, F64P, f32p]
    L.hg_mlp_train.argtypes = [f32p, f32p, f32p, f32p, C.c_int64, C.c_int32, C.c_int32, C.c_double, C.c_uint64, F64P]
    _lib = L
    return L


def nodes(N, node_type):
    """The library's interpolation nodes and weights on [0,1] for order N."""
    import numpy as np
    xi, w = np.zeros(N + 1), np.zeros(N + 1)
    if load().hg_nodes(N, node_type, xi.ctypes.data_as(F64P), w.ctypes.data_as(F64P)) != 0:
        raise RuntimeError(load().hg_last_error(None).decode())
    return xi, w
