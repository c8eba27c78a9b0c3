"""hg_residuals_noalloc (fixed device scratch, no allocation) against hg_residuals on the same QDot.

Collected last on purpose: it must pass alone and after every other GPU test in one process.
"""
import ctypes as C

import numpy as np
import pytest

import horses2d_b200 as hg
from horses2d_b200 import mesh as hmesh, cases

pytestmark = pytest.mark.gpu

MAX_NDOF = 536870912


def noalloc():
    f = hg.lib.load().hg_residuals_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.POINTER(C.c_double)]
    return f


def call(f, ptr, ndof, stream):
    out = (C.c_double * 4)()
    rc = f(C.c_void_p(ptr), ndof, C.c_void_p(stream), out)
    return rc, np.array(out[:])


def vortex_context(n, N, seed):
    d = hmesh.box_descriptor(n, n, -5.0, 5.0, -5.0, 5.0, N, hg.NODES_LGL)
    x = d["x"].reshape(-1, 2)
    rng = np.random.default_rng(seed)
    Q = cases.isentropic_vortex(x[:, 0], x[:, 1], mach=0.5).ravel()
    Q *= 1.0 + 0.01 * rng.standard_normal(Q.shape)
    g = hg.GpuDGSEM(d, mach=0.5, node_type=hg.NODES_LGL, riemann=hg.ROE, bcs=[dict(type=hg.BC_PERIODIC)] * 4)
    g.set_state(Q)
    return g


def test_two_calls_in_a_row_match_hg_residuals():
    import torch
    f = noalloc()
    stream = torch.cuda.current_stream().cuda_stream
    ga, gb = vortex_context(12, 4, 1), vortex_context(40, 5, 2)     # 1 block and several blocks of scratch
    qa, qb = ga.compute_time_derivative(0.0), gb.compute_time_derivative(0.0)
    ra, rb = ga.residuals(), gb.residuals()                            # the existing entry point
    da, db = torch.from_numpy(qa).cuda(), torch.from_numpy(qb).cuda()
    torch.cuda.synchronize()
    for _ in range(2):
        rc, oa = call(f, da.data_ptr(), da.numel(), stream)
        assert rc == 0 and np.array_equal(oa, ra)
        rc, ob = call(f, db.data_ptr(), db.numel(), stream)
        assert rc == 0 and np.array_equal(ob, rb)


def test_calls_on_a_non_default_stream():
    """The input is written on a fresh stream and the calls run on that stream: the partial and reduce
    passes stay ordered after the write and before the read-back, and the result equals hg_residuals'."""
    import torch
    f = noalloc()
    g = vortex_context(24, 5, 4)
    q = g.compute_time_derivative(0.0)
    r = g.residuals()
    src = torch.from_numpy(q).pin_memory()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        d = torch.empty(q.size, dtype=torch.float64, device="cuda")
        d.copy_(src, non_blocking=True)
        for _ in range(2):
            rc, out = call(f, d.data_ptr(), d.numel(), s.cuda_stream)
            assert rc == 0 and np.array_equal(out, r)


def test_ragged_sizes_and_nan():
    import torch
    f = noalloc()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(3)
    for n_nodes in (1, 255, 8192, 8193, 3 * 8192 + 5):
        x = rng.standard_normal(4 * n_nodes)
        d = torch.from_numpy(x).cuda()
        torch.cuda.synchronize()
        rc, out = call(f, d.data_ptr(), d.numel(), stream)
        assert rc == 0
        assert np.array_equal(out, np.abs(x.reshape(-1, 4)).max(0))
    x[4 * 7 + 2] = np.nan
    d = torch.from_numpy(x).cuda()
    torch.cuda.synchronize()
    rc, out = call(f, d.data_ptr(), d.numel(), stream)
    assert rc == 0 and np.isnan(out[2]) and np.all(np.isfinite(out[[0, 1, 3]]))


def test_rejects_sizes_beyond_the_scratch_and_bad_arguments():
    import torch
    f = noalloc()
    d = torch.zeros(64, dtype=torch.float64, device="cuda")
    p = d.data_ptr()
    assert call(f, p, MAX_NDOF + 4, 0)[0] == 1        # above the scratch limit: rejected before any launch
    assert call(f, p, 6, 0)[0] == 1                   # not whole nodes
    assert call(f, p, 0, 0)[0] == 1
    assert call(f, 0, 8, 0)[0] == 1                   # null
    assert call(f, p + 8, 8, 0)[0] == 1               # not 32-byte aligned
    assert call(f, p, 64, 0)[0] == 0
