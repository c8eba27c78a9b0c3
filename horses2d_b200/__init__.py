"""horses2d_b200 -- B200-native DGSEM residual and Runge-Kutta stepper for HORSES2D.

The hot path (``DGSpatial_computeTimeDerivative`` + the low-storage RK schemes of
the reference) runs as hand-written sm_100a CUDA kernels in ``libhorsesgpu.so``,
reached through the C ABI in ``include/horses_gpu.h``.  This package holds the
CUDA sources (``csrc/``), the Python mirror of the reference interface
(``solver.GpuDGSEM``) and host-side mesh builders (``mesh``).
"""
from . import _lib as lib  # noqa: F401
from . import restart  # noqa: F401
from .solver import GpuDGSEM, GpuGroup, HorsesGpuError  # noqa: F401
from ._lib import (NODES_LG, NODES_LGL, ROE, HLL, EXACT, LXF, INTERIOR, SCHEME_EULER, SCHEME_RK3,  # noqa: F401
                   SCHEME_RK5, PREC_FP64, PREC_FP32, BC_PERIODIC, BC_DIRICHLET, BC_EULERWALL, BC_VISCOUSWALL,
                   BC_FARFIELD, BC_PRESSUREOUTLET, BC_NEWDIRICHLET, BR1, IP, SIPG, NIPG, IIPG,
                   AV_NONE, AV_LAPLACIAN, AV_PHYSICAL, SENSOR_JUMPS, SENSOR_MODAL, SENSOR_LEARNED,
                   STATUS_CRASHED, HEALTH_NONFINITE, HEALTH_DENSITY, HEALTH_PRESSURE)
