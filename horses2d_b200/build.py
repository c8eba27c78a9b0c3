"""Build libhorsesgpu.so in-tree with nvcc for sm_100a.

    python -m horses2d_b200.build [--force] [-v]

Each translation unit compiles to an object under ``_build/`` in parallel (the kernel
instantiations are split by precision and polynomial order), then nvcc links the shared library.
"""
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "libhorsesgpu.so")
OBJ_DIR = os.path.join(HERE, "_build")
SOURCES = ["csrc/hg_api.cu", "csrc/hg_spectral.cpp", "csrc/hg_noalloc.cu", "csrc/hg_mlp.cu", "csrc/hg_exact.cu", "csrc/hg_monitors.cu",
           "csrc/hg_mesh.cpp", "csrc/hg_restart.cpp", "csrc/hg_mortar.cu", "csrc/hg_autosave.cu",
           "csrc/hg_inst_euler_hi.cu", "csrc/hg_inst_euler_hi_t1.cu", "csrc/hg_inst_ns_hi.cu",
           "csrc/hg_inst_euler.cu", "csrc/hg_inst_euler_t1.cu",
           "csrc/hg_inst_euler32_hi.cu", "csrc/hg_inst_euler32_hi_t1.cu", "csrc/hg_inst_ns32_hi.cu",
           "csrc/hg_inst_euler32.cu", "csrc/hg_inst_euler32_t1.cu",
           "csrc/hg_inst_sensor.cu"] + \
    [f"csrc/hg_inst_ns{prec}{part}{t}.cu" for t in ("", "_t1") for prec in ("64", "32") for part in "abcd"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]
# FP32 stage kernels: quotients and square roots with the approximate (about 1-2 ulp) forms instead of
# the correctly rounded instruction sequences.  Only the FP32 instantiation units get it: the FP64
# kernels keep IEEE division and square root, which their bitwise parity with the oracle needs.
FP32_FLAGS = ["-prec-div=false", "-prec-sqrt=false"]


def flags_of(src):
    b = os.path.basename(src)
    return NVCC_FLAGS + (FP32_FLAGS if b.startswith("hg_inst_ns32") or b.startswith("hg_inst_euler32") else [])


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def headers():
    return glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + glob.glob(os.path.join(HERE, "csrc", "*.h")) + \
        [os.path.join(HERE, "..", "include", "horses_gpu.h")]


def obj_path(src):
    return os.path.join(OBJ_DIR, os.path.splitext(os.path.basename(src))[0] + ".o")


def stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(not os.path.exists(d) or os.path.getmtime(d) > t for d in deps)


def up_to_date():
    objs = [obj_path(s) for s in SOURCES]
    hdr = headers()
    return not stale(OUT, objs) and not any(stale(obj_path(s), [os.path.join(HERE, s)] + hdr) for s in SOURCES)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return OUT
    os.makedirs(OBJ_DIR, exist_ok=True)
    hdr = headers()
    todo = [s for s in SOURCES if force or stale(obj_path(s), [os.path.join(HERE, s)] + hdr)]

    def compile_one(src):
        cmd = [nvcc()] + flags_of(src) + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj_path(src)]
        r = subprocess.run(cmd, cwd=HERE, capture_output=True, text=True)
        return src, r

    with ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 4) or 1) as ex:
        results = list(ex.map(compile_one, todo))
    failed = False
    for src, r in results:
        if verbose or r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            sys.stderr.write(f"nvcc failed on {src}\n")
            failed = True
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc")
    subprocess.run([nvcc()] + ARCH + ["-shared", "-o", OUT] + [obj_path(s) for s in SOURCES], cwd=HERE, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
