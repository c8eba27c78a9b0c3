"""Restart files (*.HiORst): the library's NetCDF-classic writer and reader against the reference's
files (Solver/src/Approximation/DGTimeIntegrator.f90:413-454 writes them, DGSEM_class.f90:263-291
reads them) and against scipy's independent NetCDF reader."""
import hashlib
import os

import numpy as np
import pytest
from scipy.io import netcdf_file

from horses2d_b200 import restart

HERE = os.path.dirname(os.path.abspath(__file__))
# sha256 of TestCases/SupersonicTests/ShockWave/RESULTS/InitialConditionP5.HiORst (295140 bytes), the
# reference's restart fixture whose t, iter and Q tests/golden/ShockWaveP5.rst.npz holds
REF_SHA256 = "8f8a1043e841ee0473ab8df13c3fd49fd3e6abe1b128b9b561964a8e3daba586"
# the reference tree (HORSES2D_REF, optional): when set, the written bytes are also compared with the file
REF_FILE = (os.path.join(os.environ["HORSES2D_REF"], "TestCases/SupersonicTests/ShockWave/RESULTS/InitialConditionP5.HiORst")
            if os.environ.get("HORSES2D_REF") else None)


def fixture():
    z = np.load(os.path.join(HERE, "golden", "ShockWaveP5.rst.npz"))
    return float(z["t"][0]), int(z["iter"][0]), z["Q"].astype(np.float64)


def test_writer_reproduces_reference_file_bytes(tmp_path):
    t, it, Q = fixture()
    p = tmp_path / "InitialConditionP5.HiORst"
    restart.write(p, t, it, Q, N=5, n_elements=256)
    data = p.read_bytes()
    assert len(data) == 295140
    assert hashlib.sha256(data).hexdigest() == REF_SHA256
    if REF_FILE and os.path.exists(REF_FILE):
        with open(REF_FILE, "rb") as f:
            assert f.read() == data


def test_reader_on_reference_fixture(tmp_path):
    t, it, Q = fixture()
    src = REF_FILE
    if not (src and os.path.exists(src)):
        src = tmp_path / "rst.HiORst"
        restart.write(src, t, it, Q, N=5, n_elements=256)
    t2, it2, Q2 = restart.read(src)
    assert t2 == t and it2 == it
    assert np.array_equal(Q2, Q)


def test_round_trip_and_scipy_reads_it(tmp_path):
    rng = np.random.default_rng(7)
    N, E = 3, 37
    Q = rng.standard_normal(E * (N + 1) ** 2 * 4) * 1e3
    Q[5] = np.inf
    Q[6] = -0.0
    p = tmp_path / "a.HiORst"
    restart.write(p, 12.375, 4242, Q, N=N, n_elements=E)
    t, it, Q2 = restart.read(p)
    assert (t, it) == (12.375, 4242)
    assert np.array_equal(Q2, Q) and np.signbit(Q2[6])
    f = netcdf_file(p, "r", mmap=False)
    try:
        assert f.dimensions == {"one": 1, "NDOF": Q.size, "N": N, "NCONS": 4, "no_of_elements": E}
        assert float(f.variables["t"].data[0]) == 12.375
        assert int(f.variables["iter"].data[0]) == 4242
        assert np.array_equal(f.variables["Q"].data.astype(np.float64), Q)
    finally:
        f.close()


@pytest.mark.parametrize("version", [1, 2])
def test_reader_accepts_other_classic_layouts(tmp_path, version):
    """Variables in another order, attributes and (CDF-2) 64-bit offsets: any classic file holding t, Q, iter."""
    Q = np.arange(64, dtype=np.float64) / 7.0
    p = tmp_path / "b.HiORst"
    f = netcdf_file(p, "w", version=version)
    f.title = "written by scipy"
    f.createDimension("NDOF", Q.size)
    f.createDimension("one", 1)
    vi = f.createVariable("iter", "i4", ("one",))
    vi[:] = 17
    vi.units = "iterations"
    vq = f.createVariable("Q", "f8", ("NDOF",))
    vq[:] = Q
    vt = f.createVariable("t", "f8", ("one",))
    vt[:] = 0.5
    f.close()
    t, it, Q2 = restart.read(p)
    assert (t, it) == (0.5, 17) and np.array_equal(Q2, Q)


def test_reader_errors(tmp_path):
    with pytest.raises(OSError, match="cannot open"):
        restart.read(tmp_path / "missing.HiORst")
    bad = tmp_path / "bad.HiORst"
    bad.write_bytes(b"HDF\x89 not netcdf")
    with pytest.raises(OSError, match="classic"):
        restart.read(bad)
    good = tmp_path / "good.HiORst"
    restart.write(good, 0.0, 0, np.ones(16), N=1, n_elements=1)
    trunc = tmp_path / "trunc.HiORst"
    trunc.write_bytes(good.read_bytes()[:150])
    with pytest.raises(OSError, match="truncated"):
        restart.read(trunc)
    nov = tmp_path / "nov.HiORst"
    f = netcdf_file(nov, "w")
    f.createDimension("one", 1)
    f.createVariable("t", "f8", ("one",))[:] = 1.0
    f.close()
    with pytest.raises(OSError, match="no variable Q"):
        restart.read(nov)
    with pytest.raises(OSError, match="bad restart arguments"):
        restart.write(tmp_path / "x.HiORst", 0.0, 0, np.ones(6), N=1, n_elements=1)


def test_autosave_name():
    assert restart.autosave_name("RESULTS/Cylinder.HiORst", 500) == "RESULTS/Cylinder_500.HiORst"
    assert restart.autosave_name("out", 3) == "out_3.HiORst"
