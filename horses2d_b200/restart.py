"""Restart files (*.HiORst) through the library's NetCDF-classic reader and writer.

``write`` produces the file the reference's TimeIntegrator_Autosave writes
(Solver/src/Approximation/DGTimeIntegrator.f90:413-454): dimensions one, NDOF, N,
NCONS, no_of_elements and variables t, Q, iter.  ``read`` returns what
DGSEM_loadRestartFile (Solver/src/Approximation/DGSEM_class.f90:263-291) takes
from it.  Q is Storage%Q, the state layout of ``GpuDGSEM.set_state``.
"""
import ctypes as C
import os

import numpy as np

from . import _lib as L


def autosave_name(solution_file, iteration):
    """Name of an intermediate restart file: the solution file's name up to '.HiORst', then
    '_<iter>.HiORst' (the reference's Autosave without an explicit file name, lines 431-435)."""
    pos = solution_file.find(".HiORst")
    stem = solution_file if pos < 0 else solution_file[:pos]
    return f"{stem}_{int(iteration)}.HiORst"


def write(path, t, iteration, Q, N, n_elements):
    lib = L.load()
    Q = np.ascontiguousarray(Q, dtype=np.float64).ravel()
    rc = lib.hg_write_restart(os.fsencode(path), float(t), int(iteration), Q.ctypes.data_as(L.F64P), Q.size, int(N),
                              int(n_elements))
    if rc != 0:
        raise OSError(lib.hg_restart_last_error().decode())


def read(path):
    """(t, iter, Q) of a restart file."""
    lib = L.load()
    n = C.c_int64(0)
    if lib.hg_read_restart(os.fsencode(path), None, None, None, 0, C.byref(n)) != 0:
        raise OSError(lib.hg_restart_last_error().decode())
    Q = np.empty(n.value)
    t, it = C.c_double(0.0), C.c_int32(0)
    if lib.hg_read_restart(os.fsencode(path), C.byref(t), C.byref(it), Q.ctypes.data_as(L.F64P), Q.size, None) != 0:
        raise OSError(lib.hg_restart_last_error().decode())
    return t.value, it.value, Q
