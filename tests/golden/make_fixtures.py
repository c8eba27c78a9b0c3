"""Generate the committed golden fixtures from the HORSES2D reference tree.

Run once in a container that has the reference checked out, with ``HORSES2D_REF``
set to the root of that tree (the script refuses to run without it).  Outputs, next to
this script:

* ``<name>.mesh.npz`` -- the .HiOMesh NetCDF variables (points, quads, boundary
  edges/markers, curved edges, p-refinement zones) of the meshes the reference's
  regression cases use;
* ``ShockWaveP5.rst.npz`` -- the reference restart fixture
  ``TestCases/SupersonicTests/ShockWave/RESULTS/InitialConditionP5.HiORst`` (t, iter, Q);
* ``benchmarks.json`` -- the expected values the reference's benchmark
  ``ProblemFile.f90`` plugins assert in their ``Finalize`` (iteration counts,
  max-norm errors, residuals, lift/drag), parsed from those sources.

Nothing at test time reads the reference tree; only these files.
"""
import json
import os
import re
import sys

import numpy as np
from scipy.io import netcdf_file

REF = os.environ.get("HORSES2D_REF")
HERE = os.path.dirname(os.path.abspath(__file__))

MESHES = {
    "VortexTransportBench": "TestCases/Benchmark/Simulations/VortexTransport/MESH/VortexTransport.HiOMesh",
    "CouetteBench": "TestCases/Benchmark/Simulations/Couette/MESH/Couette.HiOMesh",
    "CylinderBench": "TestCases/Benchmark/Simulations/CylinderRe100/MESH/Cylinder.HiOMesh",
    "RampBench": "TestCases/Benchmark/Simulations/Ramp/MESH/Ramp.HiOMesh",
    "ShockWave": "TestCases/SupersonicTests/ShockWave/MESH/ShockWave.HiOMesh",
    "VortexTransportCase": "TestCases/Cases/VortexTransport/MESH/VortexTransport.HiOMesh",
    "CylinderInflation": "TestCases/Benchmark/Simulations/CylinderRe1000/MESH/CylinderInflation.HiOMesh",
}

PLUGINS = {
    "VortexTransport": "TestCases/Benchmark/Simulations/VortexTransport/SETUP/ProblemFile.f90",
    "Couette": "TestCases/Benchmark/Simulations/Couette/SETUP/ProblemFile.f90",
    "CylinderRe100": "TestCases/Benchmark/Simulations/CylinderRe100/SETUP/ProblemFile.f90",
    "CylinderRe1000": "TestCases/Benchmark/Simulations/CylinderRe1000/SETUP/ProblemFile.f90",
    "CylinderMach2": "TestCases/Benchmark/Simulations/CylinderMach2/SETUP/ProblemFile.f90",
    "Ramp": "TestCases/Benchmark/Simulations/Ramp/SETUP/ProblemFile.f90",
}


def read_mesh(path):
    nc = netcdf_file(path, "r", mmap=False)
    v = nc.variables
    out = {
        "points": np.asarray(v["points"].data, dtype=np.float64),
        "quads": np.asarray(v["points_of_quads"].data, dtype=np.int32),
        "bdry_edges": np.asarray(v["points_of_bdryedges"].data, dtype=np.int32),
        "bdry_marker": np.asarray(v["bdrymarker_of_edges"].data, dtype=np.int32),
    }
    names = []
    k = 1
    while f"marker{k}" in v:
        names.append(v[f"marker{k}"].data.tobytes().decode().strip())
        k += 1
    out["marker_names"] = np.array(names)
    if "curvilinear_edges" in v:
        out["curved_edges"] = np.asarray(v["curvilinear_edges"].data, dtype=np.int32)
        out["curve_x"] = np.asarray(v["x_curvilinear_edges"].data, dtype=np.float64)
        out["curve_y"] = np.asarray(v["y_curvilinear_edges"].data, dtype=np.float64)
    if "pRefinement_zones" in v:
        out["p_zones"] = np.asarray(v["pRefinement_zones"].data, dtype=np.int32)
    nc.close()
    return out


def parse_plugin(path):
    src = open(path).read()
    num = r"([-+]?\d+\.\d+E[-+]?\d+)_RP"
    res = {}
    for key in ("expectedIter", "finalIteration"):
        m = re.search(key + r"\s*=\s*(\d+)", src)
        if m:
            res["expected_iter"] = int(m.group(1))
    for key in ("expectedErrors", "expectedResiduals", "residuals"):
        m = re.search(r"\b" + key + r"\((?:NCONS|4)\)\s*&?\s*=\s*&?\s*\[([^\]]*)\]", src, re.S)
        if m:
            res[key] = [float(x) for x in re.findall(r"[-+]?\d+\.\d+E[-+]?\d+", m.group(1))]
    for key in ("expectedCl", "expectedCd", "cl", "cd"):
        m = re.search(r"\b" + key + r"\s*=\s*" + num, src)
        if m:
            res[key] = float(m.group(1))
    return res


def main():
    if not REF:
        sys.stderr.write("set HORSES2D_REF to the root of the HORSES2D reference tree\n")
        return 2
    for name, rel in MESHES.items():
        d = read_mesh(os.path.join(REF, rel))
        np.savez_compressed(os.path.join(HERE, f"{name}.mesh.npz"), **d)
        print(name, d["quads"].shape)
    rst = netcdf_file(os.path.join(REF, "TestCases/SupersonicTests/ShockWave/RESULTS/InitialConditionP5.HiORst"),
                      "r", mmap=False)
    np.savez_compressed(os.path.join(HERE, "ShockWaveP5.rst.npz"),
                        t=np.asarray(rst.variables["t"].data, dtype=np.float64),
                        iter=np.asarray(rst.variables["iter"].data),
                        Q=np.asarray(rst.variables["Q"].data, dtype=np.float64))
    rst.close()
    bench = {k: parse_plugin(os.path.join(REF, v)) for k, v in PLUGINS.items()}
    with open(os.path.join(HERE, "benchmarks.json"), "w") as f:
        json.dump(bench, f, indent=1, sort_keys=True)
    print(json.dumps(bench, indent=1))


if __name__ == "__main__":
    sys.exit(main())
