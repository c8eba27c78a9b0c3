"""The C-ABI library loads without a GPU and exports every function include/horses_gpu.h declares (CPU)."""
import ctypes as C
import os
import re
import subprocess

from horses2d_b200 import lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "horses_gpu.h")


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    return sorted(set(re.findall(r"\b(hg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    L = lib.load()
    names = declared_functions()
    assert "hg_create" in names and "hg_time_step" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert set(declared_functions()) <= set(lib.EXPORTED)


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """Sizes and field offsets of the descriptors as gcc lays them out, against the ctypes mirrors."""
    structs = {"hg_physics_desc": lib.PhysicsDesc, "hg_bc_desc": lib.BCDesc, "hg_mesh_desc": lib.MeshDesc}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "horses_gpu.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(ln.split()[:2]): int(ln.split()[2]) for ln in out if ln}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_mixed_order_descriptor_validation():
    """Mixed orders are checked before any device call: Euler orders above 12 are refused with the
    reason (CPU; the oracle's export gives the descriptor)."""
    import numpy as np
    import pytest
    import horses2d_b200 as hg
    from horses2d_b200 import mesh as hmesh
    from oracle import oracle as O
    m = hmesh.cartesian(3, 3, -1.0, 1.0, -1.0, 1.0)
    orc = O.Oracle(m, np.array([2, 3, 2, 3, 2, 3, 2, 3, 2]), nodes=O.LG, riemann=O.ROE, mach=0.5,
                   bcs=hmesh.periodic_bcs_cartesian())
    d = orc.export_mesh()
    assert len(d["edge_n"]) == 2 * sum(max(d["N"][a], d["N"][b] if b >= 0 else 0) + 1
                                       for a, b in d["edge_elem"].reshape(-1, 2))
    d13 = dict(d, N=np.where(d["N"] == 3, 13, d["N"]).astype(np.int32))
    with pytest.raises(hg.HorsesGpuError, match="1..12"):
        hg.GpuDGSEM(d13, mach=0.5, bcs=[dict(type=hg.BC_PERIODIC)] * 4)
