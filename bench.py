"""Benchmark of the B200 DGSEM residual + Williamson RK3 stepper (DOF-stage updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--precision fp32|fp64]
    python bench.py --impl reference ...      # CPU arm: the oracle restatement on all host cores

One "step" is one Williamson RK3 time step (3 residual evaluations + updates)
over the whole workload.  DOF-stage updates/s = NDOF * 3 * K / time, NDOF =
size(Storage%Q) = 4 x nodes (the reference's DOF count, DGSEM_class.f90:337-340).

Workloads (synthetic inputs with the configurations' shapes; seeds fixed):
  cylinder : (default) Navier-Stokes past a circular cylinder, Re 100, M 0.2, Pr 0.72,
             O-grid 64 radial x 128 azimuthal curved quads, r 0.5 -> 30, radial
             stretching 1.05, N = 5, Legendre-Gauss nodes, BR1, Roe, adiabatic viscous
             wall, far-field zone; uniform free stream + 1e-3 N(0,1) per DOF (seed
             20261203); NDOF 1,179,648; CFL 0.05 (the reference's time-step estimate is
             inviscid only; with the near-wall elements at Re 100, N = 5 the viscous limit
             makes CFL 0.2 unstable, for the oracle as for the kernels).  FP64 plain; the
             FP32-bulk path is timed in the same run and its density error after the K
             steps is reported.
  vortex16 : the reference-runnable case: 16 x 16 periodic vortex, N = 4, LGL, Roe, FP64.
  ensemble : 512 periodic isentropic-vortex instances on [-5,5]^2, n x n elements with
             n ~ U{8..48}, N ~ U{3..7}, vortex centre ~ U[-2,2]^2, beta ~ U[2,6],
             M 0.5 at 45 deg, LGL nodes, Roe, packed by polynomial order into one
             element list per order; FP32 bulk with FP64 state accumulator by default.
  box512   : one 512 x 512 periodic vortex box, N = 4, LGL, Roe, FP64 (profiling case).
  shock    : the learned-sensor case: [0,10] x [0,1], 512 x 64 elements, N = 3, Mach-3 normal shock
             with an upstream entropy wave (amplitude 0.2), HLL, Re = 0, Laplacian artificial
             dissipation; the sensor network is first trained on the GPU on 2 x 100 solver snapshots
             (shock position +-0.5, amplitude 0.1-0.3, seed 20261203); value = FP32 bulk + learned
             sensor, beside the plain FP64 path with the modal-decay sensor.
  kh       : doubly periodic Kelvin-Helmholtz shear layer on [0,1]^2, 1024 x 1024 elements, N = 7
             (NDOF 268,435,456), Re 1e4, M 0.3, tanh layers of thickness 0.01 with a seeded 4-mode
             perturbation of amplitude 1e-2, SIPG (sigma0 10), Roe, Laplacian artificial viscosity
             driven by the learned sensor (trained as for `shock`; out-of-distribution elements use
             the modal indicator); FP32 bulk + learned beside FP64 + modal.  --kh-n sets the size.
  prefine  : p-refined periodic vortex box (as the reference's VortexTransport p-zones): 384 x 384
             elements on [-5,5]^2, N = 7 in the central 192 x 192 square and N = 5 around it
             (edges between the two orders through the mortar kernel), Legendre-Gauss, Roe, FP64,
             CFL 0.3 (with Legendre-Gauss nodes RK3 at CFL 0.4 is unstable, for the oracle as for the kernels).
Multi-GPU: independent replicas (the workload does not exchange data), weak scaling.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 20261203
L2_BYTES = 126 * 2 ** 20
KH_DT_COEF = 0.05   # kh workload: dt = 0.05 / n^2 (half the measured interior-penalty stability limit)
CONFIGS = ("cylinder", "vortex16", "ensemble", "box512", "shock", "kh", "prefine")


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------------------- workloads
def ensemble_spec(seed=SEED, n_inst=512):
    rng = np.random.default_rng(seed)
    inst = []
    for _ in range(n_inst):
        n = int(rng.integers(8, 49))
        N = int(rng.choice([3, 4, 5, 6, 7]))
        xc, yc = rng.uniform(-2.0, 2.0, 2)
        beta = float(rng.uniform(2.0, 6.0))
        inst.append(dict(n=n, N=N, xc=float(xc), yc=float(yc), beta=beta))
    return inst


def cylinder_mesh():
    from horses2d_b200 import mesh as hmesh
    return hmesh.ogrid(64, 128, 0.5, 30.0, 1.05)


def freestream(mach, gamma=1.4):
    """Dimensionless uniform state (rho = p = 1, u = sqrt(gamma) M)."""
    u = np.sqrt(gamma) * mach
    return np.array([1.0, u, 0.0, 1.0 / (gamma - 1.0) + 0.5 * u * u])


def cylinder_state(n_nodes, seed=SEED):
    rng = np.random.default_rng(seed)
    return (np.tile(freestream(0.2), n_nodes) + 1e-3 * rng.standard_normal(4 * n_nodes))


def prefine_orders(n):
    """Orders of the p-refined box: 7 in the central n/2 x n/2 square, 5 elsewhere (row-major)."""
    i = np.tile(np.arange(n), n)
    j = np.repeat(np.arange(n), n)
    inner = (i >= n // 4) & (i < n - n // 4) & (j >= n // 4) & (j < n - n // 4)
    return np.where(inner, 7, 5).astype(np.int32)


def build_parts(config):
    """[(descriptor, Q0, N, n_instances, solver kwargs, cfl)] -- one GPU context each."""
    from horses2d_b200 import mesh as hmesh, cases
    import horses2d_b200 as hg
    if config == "prefine":
        n = 384
        desc = hmesh.box_descriptor(n, n, -5.0, 5.0, -5.0, 5.0, prefine_orders(n), hg.NODES_LG)
        x = desc["x"].reshape(-1, 2)
        Q0 = cases.isentropic_vortex(x[:, 0], x[:, 1], mach=0.5, beta=5.0).ravel()
        kw = dict(mach=0.5, node_type=hg.NODES_LG, riemann=hg.ROE, bcs=[dict(type=hg.BC_PERIODIC)] * 4)
        # CFL 0.1: at 0.3 the 384^2 box (192^2 too) goes non-finite within 40 steps -- on the oracle as on
        # the device (at 48^2 and 96^2 it stays finite); at 0.1 the oracle stays finite over 250 steps,
        # more than the 200 between the load warm-up's restarts
        return [(desc, Q0, "5/7", 1, kw, 0.1)]
    if config == "cylinder":
        N = 5
        desc = hmesh.build_descriptor(cylinder_mesh(), N, hg.NODES_LG)
        q = freestream(0.2)
        kw = dict(mach=0.2, reynolds=100.0, prandtl=0.72, navier_stokes=1, viscous=hg.BR1, node_type=hg.NODES_LG,
                  riemann=hg.ROE, bcs=[dict(type=hg.BC_VISCOUSWALL, wall_type=2),
                                       dict(type=hg.BC_FARFIELD, state=q)])
        return [(desc, cylinder_state(len(desc["N"]) * (N + 1) ** 2), N, 1, kw, 0.05)]
    if config == "vortex16":
        inst = [dict(n=16, N=4, xc=0.0, yc=0.0, beta=5.0)]
    elif config == "box512":
        inst = [dict(n=512, N=4, xc=0.0, yc=0.0, beta=5.0)]
    elif config == "ensemble":
        inst = ensemble_spec()
    else:
        raise SystemExit(f"unknown config {config}")
    kw = dict(mach=0.5, node_type=hg.NODES_LGL, riemann=hg.ROE, bcs=[dict(type=hg.BC_PERIODIC)] * 4)
    parts = []
    for N in sorted({i["N"] for i in inst}):
        descs, qs = [], []
        eo = fo = 0
        for it in (i for i in inst if i["N"] == N):
            d = hmesh.box_descriptor(it["n"], it["n"], -5.0, 5.0, -5.0, 5.0, N, hg.NODES_LGL,
                                     elem_offset=eo, edge_offset=fo)
            x = d["x"].reshape(-1, 2)
            qs.append(cases.isentropic_vortex(x[:, 0], x[:, 1], mach=0.5, beta=it["beta"], xc=it["xc"], yc=it["yc"]))
            eo += len(d["N"])
            fo += len(d["edge_marker"])
            descs.append(d)
        parts.append((hmesh.concat_descriptors(descs), np.concatenate(qs).ravel(), N,
                      sum(1 for i in inst if i["N"] == N), kw, 0.4))
    return parts


def step_bytes_per_dof_stage(fp32, affine, br1):
    """Algorithmic DRAM bytes per DOF-stage of a Williamson RK3 step with fused stages: the state Q read
    and written in FP64 every stage (16 B), the RK register G written every stage and read in stages 2-3
    (sG = 4 or 8 B: 5/3 sG), the volume metrics Ja, 1/J on curved meshes (5 values per node: 1.25 sG;
    0 on affine meshes, whose metrics are per element), and with BR1 the lifted gradient written and read
    back (8 values per node: 4 sG).  Interior-penalty gradients are element-local (0).  Face traces and
    nodal matrices count 0 (cache-resident).  FP64: 29.33 affine, +10 curved, +32 BR1."""
    sg = 4.0 if fp32 else 8.0
    return 16.0 + sg * 5.0 / 3.0 + (0.0 if affine else 1.25 * sg) + (4.0 * sg if br1 else 0.0)


def stage_kernel_bytes_per_dof(fp32, affine, br1):
    """The share of those bytes that the stage kernel moves: all of them except, with BR1, the gradient
    write (2 sG), which the gradient kernel makes."""
    return step_bytes_per_dof_stage(fp32, affine, br1) - ((8.0 if fp32 else 16.0) if br1 else 0.0)


def roofline_from_split(split, split_steps, ms_step, ndof, fp32, affine, br1, peak, peak_kind, traffic_name=None,
                        ns=True):
    """Roofline of the dominant kernel (the stage kernel) from the timed region: its average launch time
    is its share of the per-kernel event times (library timing mode, `split`) times the timed
    milliseconds per step, divided by its launches per step; achieved = its algorithmic bytes per launch
    over that time.  Also the whole step's algorithmic bytes over the timed step."""
    total = sum(v[0] for v in split.values()) or 1.0
    share = {k: round(v[0] / total, 4) for k, v in split.items() if v[1]}
    st_ms, st_n = split["stage"]
    per_step = st_n / split_steps
    avg_s = (st_ms / total) * ms_step * 1e-3 / per_step
    dof_per_launch = ndof * 3.0 / per_step
    kbpd = stage_kernel_bytes_per_dof(fp32, affine, br1)
    achieved = kbpd * dof_per_launch / avg_s / 1e9
    traffic = None
    if traffic_name:
        tpath = os.path.join(ROOT, "profiles", f"{traffic_name}.traffic.json")
        if os.path.exists(tpath):
            try:
                traffic = json.load(open(tpath))["bytes_per_dof"] * dof_per_launch
            except Exception:
                traffic = None
    sbpd = step_bytes_per_dof_stage(fp32, affine, br1)
    step_ach = sbpd * ndof * 3.0 / (ms_step * 1e-3) / 1e9
    kernel = {"bound": "hbm", "kernel": "ns_stage_kernel" if ns else "stage_kernel",
              "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
              "peak_source": peak_kind, "algorithmic_bytes_per_dof": kbpd, "avg_launch_us": avg_s * 1e6,
              "launch_time_from": "kernel share of the library's per-launch events x timed ms per step"}
    step = {"algorithmic_bytes_per_dof_stage": sbpd, "achieved": step_ach, "frac": step_ach / peak}
    return {"kernel": kernel, "step": step, "share": share}


def kh_dt(n):
    """Time step of the kh workload at n x n elements: half the measured interior-penalty limit
    (the reference's estimate is inviscid only; measured on the oracle, dt_max ~ 0.1 / n^2)."""
    return KH_DT_COEF / n ** 2


KH_PHYSICS = ("Navier-Stokes, Re 1e4, M 0.3, Pr 0.72, periodic, SIPG (sigma0 10), Roe, Laplacian artificial "
              "viscosity")


def workload_ndof(name, args):
    """NDOF = 4 x nodes of a workload, from its definition (no device needed)."""
    if name == "kh":
        return 4 * args.kh_n ** 2 * 64
    if name == "cylinder":
        return 4 * 64 * 128 * 36
    if name == "shock":
        return 4 * 512 * 64 * 16
    if name == "vortex16":
        return 4 * 16 * 16 * 25
    if name == "box512":
        return 4 * 512 * 512 * 25
    if name == "prefine":
        return int(4 * np.sum((prefine_orders(384) + 1) ** 2))
    return int(sum(4 * it["n"] ** 2 * (it["N"] + 1) ** 2 for it in ensemble_spec()))


def workload_config(name, args, world):
    """The `config` object of a workload: what is run, identical in both arms (measured quantities and
    the autotuner's choice go elsewhere in the line)."""
    ndof = workload_ndof(name, args)
    par = f"replicas x{world}"
    l2 = ("256 MB buffer written between timed steps (outside the step events)" if ndof * 8 * 3 < 2 * L2_BYTES
          else "inputs larger than L2")
    if name == "kh":
        n = args.kh_n
        return {"workload": "kh", "ndof": ndof, "mesh": f"{n}x{n}", "N": 7, "nodes": "Legendre-Gauss",
                "precision": "fp64", "physics": KH_PHYSICS, "sensor": "modal decay (the plain method)",
                "dt": kh_dt(n), "scheme": "Williamson RK3", "l2": l2, "parallelism": par}
    if name == "shock":
        return {"workload": "shock", "ndof": ndof, "mesh": "512x64", "N": 3, "nodes": "Legendre-Gauss",
                "precision": "fp32", "physics": "Navier-Stokes build at Re 0, Mach-3 shock, HLL, SIPG, Laplacian "
                "artificial viscosity", "sensor": "learned (MLP 16-32-32-1) with modal fallback",
                "scheme": "Williamson RK3", "l2": l2, "parallelism": par}
    prec = args.precision or ("fp32" if name == "ensemble" else "fp64")
    orders = {"cylinder": [5], "vortex16": [4], "box512": [4], "prefine": ["5/7"],
              "ensemble": [3, 4, 5, 6, 7]}[name]
    return {"workload": name, "ndof": ndof, "precision": prec, "orders": orders,
            "instances": 512 if name == "ensemble" else 1, "scheme": "Williamson RK3", "l2": l2,
            "parallelism": par}


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, max clock, throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(k)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------- CPU (oracle) timing
class CpuArm:
    """Oracle restatement timed on the host cores on a bounded sample of the workload.

    cylinder: the full workload on one oracle whose element loops run on all host
    threads (OpenMP, face loops serial, as the reference's own parallel build).
    Vortex workloads: instances stepped concurrently, one single-threaded oracle per
    host thread (the ctypes calls release the GIL)."""

    def __init__(self, config, threads=None):
        from oracle import oracle as O
        from horses2d_b200 import mesh as hmesh, cases
        self.O = O
        self.config = config
        self.threads = threads or os.cpu_count() or 1
        self.steps_done = []
        if config == "shock":
            from horses2d_b200 import sensor as S
            O.lib().or_set_threads(self.threads)
            (r1, u1, p1), (r2, u2, p2) = S.rankine_hugoniot(3.0)
            bcs = [dict(type=O.BC_EULERWALL), dict(type=O.BC_EULERWALL), dict(type=O.BC_DIRICHLET),
                   dict(type=O.BC_NEWDIRICHLET, pressure=101325.0 * p2, temperature=273.15 * p2 / r2,
                        mach=u2 / np.sqrt(1.4 * p2 / r2))]
            o = O.Oracle(hmesh.cartesian(512, 64, 0.0, 10.0, 0.0, 1.0), 3, nodes=O.LG, riemann=O.HLL, mach=3.0,
                         reynolds=0.0, navier_stokes=1, viscous=O.IP, ip_method=0, sigma0_ip=10.0, bcs=bcs,
                         av_type=O.AV_LAPLACIAN, av_intensity=1.0, av_indicator=O.IND_MODAL)
            x = o.coords()[:, 0]
            up = x < 5.0
            o.set_state(S.conservative(np.where(up, 1.0 + 0.2 * np.sin(5.0 * x), r2), np.where(up, u1, u2),
                                       np.where(up, 1.0, p2)).ravel())
            self.orcs = [(o, o.estimate_dt(0.1, 1.0))]
            return
        if config == "kh":
            # bounded sample: 128 x 128 elements of the 1024 x 1024 workload, same order and physics
            O.lib().or_set_threads(self.threads)
            o = O.Oracle(hmesh.cartesian(128, 128, 0.0, 1.0, 0.0, 1.0), 7, nodes=O.LG, riemann=O.ROE, mach=0.3,
                         reynolds=1.0e4, navier_stokes=1, viscous=O.IP, ip_method=0, sigma0_ip=10.0,
                         bcs=hmesh.periodic_bcs_cartesian(), av_type=O.AV_LAPLACIAN, av_intensity=1.0,
                         av_indicator=O.IND_MODAL)
            X = o.coords()
            o.set_state(cases.kelvin_helmholtz(X[:, 0], X[:, 1], seed=SEED).ravel())
            self.orcs = [(o, min(o.estimate_dt(0.2, 1.0), KH_DT_COEF / 128 ** 2))]
            return
        if config == "cylinder":
            O.lib().or_set_threads(self.threads)
            o = O.Oracle(cylinder_mesh(), 5, nodes=O.LG, riemann=O.ROE, mach=0.2, reynolds=100.0, prandtl=0.72,
                         navier_stokes=1, viscous=O.BR1,
                         bcs=[dict(type=O.BC_VISCOUSWALL, wall_type=2), dict(type=O.BC_FARFIELD)])
            o.set_state(cylinder_state(o.ndof // 4))
            self.orcs = [(o, o.estimate_dt(0.05, 1.0))]
            return
        if config == "prefine":
            # bounded sample: one 48 x 48 box with the same order layout per host thread
            self.inst = [dict(n=48, N="5/7")] * self.threads
            self.orcs = []
            for _ in self.inst:
                o = O.Oracle(hmesh.cartesian(48, 48, -5.0, 5.0, -5.0, 5.0), prefine_orders(48), nodes=O.LG,
                             riemann=O.ROE, mach=0.5, bcs=hmesh.periodic_bcs_cartesian())
                X = o.coords()
                o.set_state(cases.isentropic_vortex(X[:, 0], X[:, 1], mach=0.5, beta=5.0).ravel())
                self.orcs.append((o, o.estimate_dt(0.1, 1.0)))
            return
        inst = ensemble_spec() if config == "ensemble" else [dict(n=16, N=4, xc=0.0, yc=0.0, beta=5.0)]
        if config == "box512":
            inst = [dict(n=64, N=4, xc=0.0, yc=0.0, beta=5.0)]
        self.inst = inst[:self.threads] if config == "ensemble" else inst * self.threads
        self.orcs = []
        for it in self.inst:
            o = O.Oracle(hmesh.cartesian(it["n"], it["n"], -5.0, 5.0, -5.0, 5.0), it["N"], nodes=O.LGL,
                         riemann=O.ROE, mach=0.5, bcs=hmesh.periodic_bcs_cartesian())
            X = o.coords()
            o.set_state(cases.isentropic_vortex(X[:, 0], X[:, 1], beta=it["beta"], xc=it["xc"],
                                                yc=it["yc"]).ravel())
            self.orcs.append((o, o.estimate_dt(0.4, 1.0)))

    def _run(self, arg, budget_s, single):
        O = self.O
        if single:
            O.lib().or_set_threads(1)
        o, dt = arg
        t0 = time.perf_counter()
        steps = 0
        while time.perf_counter() - t0 < budget_s or steps == 0:
            o.time_step(O.RK3, steps * dt, dt)
            steps += 1
        return o.ndof * 3 * steps, time.perf_counter() - t0, steps

    def sample(self, budget_s):
        """(DOF-stage/s, cores, description) of ~budget_s seconds of RK3 steps."""
        from concurrent.futures import ThreadPoolExecutor
        if self.config in ("cylinder", "shock", "kh"):
            n, el, steps = self._run(self.orcs[0], budget_s, False)
            what = ("scaled: 128 x 128 elements of the 1024 x 1024 kh workload (the rate per DOF-stage "
                    "does not depend on the element count)" if self.config == "kh"
                    else f"full {self.config} workload")
            return (n / el, self.threads, f"{what} (NDOF {self.orcs[0][0].ndof}), {steps} RK3 "
                    f"steps in {el:.1f} s, OpenMP element loops on {self.threads} threads, FP64"
                    + (", modal-decay sensor" if self.config in ("shock", "kh") else ""))
        with ThreadPoolExecutor(max_workers=self.threads) as ex:
            res = list(ex.map(lambda a: self._run(a, budget_s, True), self.orcs))
        rate = sum(r[0] / r[1] for r in res)
        desc = ", ".join(f"{it['n']}x{it['n']} N={it['N']}" for it in self.inst[:4])
        return rate, self.threads, (f"{len(self.inst)} instance(s) ({desc}{', ...' if len(self.inst) > 4 else ''}),"
                                    f" RK3 steps for ~{budget_s:.0f} s each, one single-threaded oracle per host "
                                    "thread")


def run_reference(args, rank, world):
    if rank != 0:
        return
    arm = CpuArm(args.config)
    per_step_rates = []
    cores = 0
    sample = ""
    for s in range(args.warmup + args.steps):
        rate, cores, sample = arm.sample(3.0)
        if s >= args.warmup:
            per_step_rates.append(rate)
    value = float(np.mean(per_step_rates))
    line = {"impl": "reference", "metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.config, args, world),
            "cpu_baseline": {"value": value, "unit": "DOF-stage/s", "cores": cores, "kind": "port",
                             "sample": f"each step: {sample}"},
            "e2e": {"value": value, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Fortran needs gfortran + NetCDF-Fortran (absent); its C++ FP64 restatement is timed"}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU arm
def make_contexts(parts, prec, stream):
    import torch
    import horses2d_b200 as hg
    ctxs = []
    for desc, Q0, N, ninst, kw, cfl in parts:
        g = hg.GpuDGSEM(desc, precision=prec, **kw)
        g.set_stream(stream.cuda_stream)
        Qh = torch.from_numpy(Q0).pin_memory()
        g.set_state(Qh.numpy())
        tune = g.autotune(trials=10)     # elements-per-CTA variant, timed on this workload's state
        ctxs.append(dict(g=g, Qh=Qh, N=N, ninst=ninst, cfl=cfl, tune=tune))
    return ctxs


def bucket_launch_cost(prec, stream, dt, steps=200):
    """Measured cost of running the ensemble as one context per order: the same group graph (five
    contexts, one stage launch each per RK stage, the contexts on forked streams) with each context cut
    to one 2 x 2-element instance, so that the kernels do almost no work, against one context alone
    (three launches per step, what one kernel over all orders would launch).  ms per step of each."""
    import torch
    import horses2d_b200 as hg
    from horses2d_b200 import mesh as hmesh, cases
    kw = dict(mach=0.5, node_type=hg.NODES_LGL, riemann=hg.ROE, bcs=[dict(type=hg.BC_PERIODIC)] * 4)
    gs = []
    for N in (3, 4, 5, 6, 7):
        d = hmesh.box_descriptor(2, 2, -5.0, 5.0, -5.0, 5.0, N, hg.NODES_LGL)
        x = d["x"].reshape(-1, 2)
        g = hg.GpuDGSEM(d, precision=prec, **kw)
        g.set_stream(stream.cuda_stream)
        g.set_state(cases.isentropic_vortex(x[:, 0], x[:, 1], mach=0.5, beta=0.0).ravel())   # the uniform stream
        gs.append(g)

    def timed(run):
        run(3)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    group = hg.GpuGroup(gs)
    ms5 = timed(lambda n: group.time_steps(hg.SCHEME_RK3, n, 0.0, dt))
    group.close()
    ms1 = timed(lambda n: gs[2].time_steps(hg.SCHEME_RK3, n, 0.0, dt))
    for g in gs:
        g.close()
    return {"five_orders_ms_per_step": ms5, "one_order_ms_per_step": ms1, "launches_per_step": [15, 3],
            "sample": "one 2x2-element instance of the uniform stream per order (kernels with almost no work), "
                      "group graph vs one context alone"}


def tiling_summary(ctxs):
    """Autotuner outcome per context: elements per CTA chosen and ms per residual of each variant."""
    return [{"N": c["N"], "elements_per_cta": c["tune"]["tiling"]["elements_per_cta"],
             "threads_per_cta": c["tune"]["tiling"]["threads_per_cta"],
             "ms_per_variant": [round(x, 5) for x in c["tune"]["ms"]]} for c in ctxs]


class L2Flush:
    """Writes a 256 MB device buffer (twice the 126 MB L2) between timed steps."""

    def __init__(self, enabled):
        import torch
        self.buf = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device="cuda") if enabled else None
        self.val = 0

    def __call__(self, stream):
        import torch
        if self.buf is not None:
            self.val ^= 1
            with torch.cuda.stream(stream):
                self.buf.fill_(self.val)


def device_timed(ctxs, steps, warmup, dt, stream, world, dist, flush, min_load_s=0.0):
    """Warm-up (at least `warmup` steps and, when asked, at least `min_load_s` seconds of load so
    that the clock sampler sees the GPU busy), then K steps, each between its own events on the
    launching stream with the L2 flush (if any) outside the events; barrier + sync on both sides.
    Returns (ms, launches)."""
    import torch
    import horses2d_b200 as hg

    def step(s):
        for c in ctxs:
            c["g"].time_step(hg.SCHEME_RK3, s * dt, dt)

    def restart():
        for c in ctxs:
            c["g"].set_state(c["Qh"].numpy())

    t0 = time.perf_counter()
    s = 0
    while s < warmup or time.perf_counter() - t0 < min_load_s:
        if s and s % 200 == 0:   # a long load warm-up restarts from the workload's state: the physics stays that of the workload
            restart()
        flush(stream)
        step(s)
        s += 1
        if s % 16 == 0:
            torch.cuda.synchronize()
    restart()                    # the timed steps start from the workload's initial state
    torch.cuda.synchronize()
    group = hg.GpuGroup([c["g"] for c in ctxs]) if (flush.buf is None and len(ctxs) > 1) else None

    def multi(n, t):
        """n steps through the library's multi-step call: CUDA graphs of step pairs (one graph for all
        contexts of a multi-context workload, whose members then run concurrently)."""
        if group is not None:
            group.time_steps(hg.SCHEME_RK3, n, t, dt)
        else:
            for c in ctxs:
                c["g"].time_steps(hg.SCHEME_RK3, n, t, dt)

    if flush.buf is None:
        multi(3, s * dt)   # captures the step-pair graph(s) outside the timed region
        s += 3
        torch.cuda.synchronize()
    launches0 = sum(c["g"].launch_count() for c in ctxs)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if flush.buf is None:
        # inputs larger than L2: the K steps run back to back between one pair of events
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        multi(steps, s * dt)
        ev1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        n_launch = sum(c["g"].launch_count() for c in ctxs) - launches0
        if group is not None:
            group.close()
        return ev0.elapsed_time(ev1), n_launch
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush(stream)
        evs[k][0].record(stream)
        step(s + k)
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    return sum(a.elapsed_time(b) for a, b in evs), sum(c["g"].launch_count() for c in ctxs) - launches0


def max_over_ranks(values, world, dist, device="cuda"):
    """Per-rank timings (ms) reduced to the job's: every rank gets the max over ranks (the slowest
    replica sets the whole job's time)."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def kernel_split(ctxs, steps, dt, stream, flush):
    """Per-kernel CUDA-event times over `steps` further steps (library timing mode)."""
    import torch
    import horses2d_b200 as hg
    for c in ctxs:
        c["g"].profile(True)
    for s in range(steps):
        flush(stream)
        for c in ctxs:
            c["g"].time_step(hg.SCHEME_RK3, s * dt, dt)
    tot = {}
    for c in ctxs:
        for k, (ms, n) in c["g"].kernel_times().items():
            a = tot.setdefault(k, [0.0, 0])
            a[0] += ms
            a[1] += n
        c["g"].profile(False)
    torch.cuda.synchronize()
    return tot


def run_shock(args, rank, world, local, dist):
    """The learned-sensor workload: train, then time FP32 + learned beside FP64 + modal."""
    import torch
    import horses2d_b200 as hg
    from horses2d_b200 import sensor as S
    nx, ny, N = 512, 64, 3
    t0 = time.perf_counter()
    params, lo, hi, info = S.train_two_rounds(100, SEED, nx=nx, ny=ny, N=N, steps=100, epochs=30, batch=4096)
    train_s = time.perf_counter() - t0
    desc, kw = S.shock_case(nx, ny, N)
    x_shock = S.snap_to_face(5.0, nx)
    Q0 = S.shock_state(desc, x_shock, 0.2)
    stream = torch.cuda.Stream()
    parts = [(desc, Q0, N, 1, kw, 0.1)]

    def ctx(prec, learned):
        c = make_contexts(parts, prec, stream)
        if learned:
            c[0]["g"].set_sensor(hg.SENSOR_LEARNED, mlp=params, lo=lo, hi=hi)
        else:
            c[0]["g"].set_sensor(hg.SENSOR_MODAL)
        c[0]["tune"] = c[0]["g"].autotune(trials=10)    # again, with the sensor that will run
        return c

    c32, c64 = ctx(hg.PREC_FP32, True), ctx(hg.PREC_FP64, False)
    ndof = c32[0]["g"].ndof
    dt = info["dt"]
    flush = L2Flush(ndof * 8 * 3 < 2 * L2_BYTES)
    clocks = ClockSampler(local)
    clocks.start()
    ms32, launches = device_timed(c32, args.steps, args.warmup, dt, stream, world, dist, flush, min_load_s=2.0)
    clk = clocks.stop()
    ms64, _ = device_timed(c64, args.steps, args.warmup, dt, stream, world, dist, flush)
    split = kernel_split(c32, max(3, min(args.steps, 10)), dt, stream, flush)
    # accuracy: FP32 + learned against FP64 + learned from the same state, and the sensors' statistics
    c64l = ctx(hg.PREC_FP64, True)
    steps_acc = 200
    for c in (c32[0], c64[0], c64l[0]):
        c["g"].set_state(Q0)
        c["g"].time_steps(hg.SCHEME_RK3, steps_acc, 0.0, dt)
    Q32, Q64, Q64l = (c["g"].state() for c in (c32[0], c64[0], c64l[0]))
    rho_err = float(np.linalg.norm(Q32[0::4] - Q64l[0::4]) / np.linalg.norm(Q64l[0::4]))
    _, out32 = c32[0]["g"].sensor_eval()
    _, out64 = c64[0]["g"].sensor_eval()
    m_learned = S.shock_metrics(Q32, out32[:, 3], nx, ny, x_shock)
    m_modal = S.shock_metrics(Q64, out64[:, 3], nx, ny, x_shock)
    # end to end through the public API with host buffers (FP32 + learned)
    g = c32[0]["g"]
    Qpin = torch.empty(g.ndof, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    g.set_state(c32[0]["Qh"].numpy())
    res = np.zeros(4)
    for s in range(args.steps):
        g.time_step(hg.SCHEME_RK3, s * dt, dt)
        res = np.maximum(res, g.residuals())
    Qe = g.state(out=Qpin.numpy())
    e2e_ms = (time.perf_counter() - t1) * 1e3
    if not (np.all(np.isfinite(Qe)) and np.all(np.isfinite(res))):
        raise SystemExit("non-finite state after the timed steps")
    ms32, ms64, e2e_ms = max_over_ranks([ms32, ms64, e2e_ms], world, dist)
    value = ndof * 3 * args.steps * world / (ms32 * 1e-3)
    value64 = ndof * 3 * args.steps * world / (ms64 * 1e-3)
    peak, peak_kind = peaks()
    split_steps = max(3, min(args.steps, 10))
    roof = roofline_from_split(split, split_steps, ms32 / args.steps, ndof, True, True, False, peak, peak_kind,
                               "ns_stage_kernel_shock_fp32")
    line = {"metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64acc", "data": "synthetic",
            "config": workload_config("shock", args, world), "tiling": tiling_summary(c32),
            "e2e": {"value": ndof * 3 * args.steps * world / (e2e_ms * 1e-3), "unit": "DOF-stage/s",
                    "h2d_bytes_per_step": ndof * 8 / args.steps, "d2h_bytes_per_step": 32 + ndof * 8 / args.steps},
            "gpu_launches": launches,
            "roofline": roof["kernel"], "step_roofline": roof["step"], "kernel_share": roof["share"],
            "fp64_plain_modal": {"value": value64, "ms_per_step": ms64 / args.steps, "speedup_fp32_learned": ms64 / ms32},
            "accuracy": {"rel_l2_density_fp32_vs_fp64_after_200_steps": rho_err},
            "sensor": {"training_s": train_s, "samples": info["samples"], "snapshots": 200,
                       "final_loss": info["loss_round2"][-1], "learned": m_learned, "modal": m_modal,
                       "troubled_cell_disagreement": S.disagreement(out32[:, 0], out32[:, 3]),
                       "ood_elements": int(out32[:, 2].sum())},
            "clocks": clk}
    if rank == 0 and not args.no_cpu_baseline:
        rate, cores, sample = CpuArm("shock").sample(12.0)
        line["cpu_baseline"] = {"value": rate, "unit": "DOF-stage/s", "cores": cores, "kind": "port", "sample": sample}
    line["node_stage_per_s"] = line["value"] / 4.0   # DOF-stage/s over the 4 variables of a node
    if rank == 0:
        print(json.dumps(line), flush=True)
    for c in c32 + c64 + c64l:
        c["g"].close()
    if world > 1:
        dist.destroy_process_group()


def kh_state_pinned(n, N, xi, seed):
    """The kh initial state (cases.kelvin_helmholtz at the box's nodes) in pinned host memory: the
    separable factors are evaluated on the host and multiplied out on the device (input preparation,
    outside every timed region), then copied once into the pinned buffer that the e2e leg uploads."""
    import torch
    from horses2d_b200 import cases
    rho_y, u_y, damp_y, vx = (torch.from_numpy(a).cuda() for a in cases.kelvin_helmholtz_factors(n, N, xi, seed=seed))
    P = N + 1
    rho = rho_y[:, None, :, None].expand(n, n, P, P)
    uu = u_y[:, None, :, None].expand(n, n, P, P)
    v = vx[None, :, None, :] * damp_y[:, None, :, None]
    Q = torch.empty((n, n, P, P, 4), dtype=torch.float64, device="cuda")
    Q[..., 0] = rho
    Q[..., 1] = rho * uu
    Q[..., 2] = rho * v
    Q[..., 3] = 1.0 / 0.4 + 0.5 * rho * (uu * uu + v * v)
    host = torch.empty(Q.numel(), dtype=torch.float64).pin_memory()
    host.copy_(Q.reshape(-1))
    del Q, v
    torch.cuda.synchronize()
    return host


def kh_kwargs(hg):
    return dict(mach=0.3, reynolds=1.0e4, navier_stokes=1, viscous=hg.IP, ip_method=hg.SIPG, sigma0_ip=10.0,
                node_type=hg.NODES_LG, riemann=hg.ROE, av_type=hg.AV_LAPLACIAN, av_intensity=1.0,
                bcs=[dict(type=hg.BC_PERIODIC)] * 4)


def kh_accuracy(params, lo, hi, n=32, steps=100):
    """Density error of the device paths against the FP64 oracle on a bounded sample of the kh workload
    (n x n elements, same order, physics and dt rule; `steps` RK3 steps from the same state): FP64 plain
    and FP32 plain against the oracle with the modal indicator, FP32 + learned against the oracle with
    the FP64 restatement of the learned indicator (oracle/mlp.py).  The oracle is the checker here."""
    import horses2d_b200 as hg
    from horses2d_b200 import mesh as hmesh, cases
    from oracle import oracle as O, mlp as omlp
    O.lib().or_set_threads(os.cpu_count() or 1)
    N, dt = 7, kh_dt(n)
    okw = dict(nodes=O.LG, riemann=O.ROE, mach=0.3, reynolds=1.0e4, navier_stokes=1, viscous=O.IP, ip_method=0,
               sigma0_ip=10.0, bcs=hmesh.periodic_bcs_cartesian(), av_type=O.AV_LAPLACIAN, av_intensity=1.0)
    m = hmesh.cartesian(n, n, 0.0, 1.0, 0.0, 1.0)
    om = O.Oracle(m, N, av_indicator=O.IND_MODAL, **okw)
    ol = O.Oracle(m, N, av_indicator=O.IND_EXTERNAL, **okw)
    X = om.coords()
    Q0 = cases.kelvin_helmholtz(X[:, 0], X[:, 1], seed=SEED).ravel()
    t0 = time.perf_counter()
    om.set_state(Q0)
    ol.set_state(Q0)
    xi = omlp.gauss_nodes(N + 1)
    s0 = np.log10(1.0 / (N + 1) ** 4)
    for k in range(steps):
        om.time_step(O.RK3, k * dt, dt)
        omlp.step_learned(ol, params, lo, hi, xi, O.RK3, k * dt, dt, s0)
    oracle_s = time.perf_counter() - t0
    ref = {"modal": om.state()[0::4], "learned": ol.state()[0::4]}
    desc = om.export_mesh()
    out = {}
    for name, prec, sensor, against in (("fp64_plain", hg.PREC_FP64, hg.SENSOR_MODAL, "modal"),
                                        ("fp32_plain", hg.PREC_FP32, hg.SENSOR_MODAL, "modal"),
                                        ("fp32_learned", hg.PREC_FP32, hg.SENSOR_LEARNED, "learned")):
        g = hg.GpuDGSEM(desc, precision=prec, **kh_kwargs(hg))
        if sensor == hg.SENSOR_LEARNED:
            g.set_sensor(sensor, mlp=params, lo=lo, hi=hi)
        else:
            g.set_sensor(sensor)
        g.set_state(Q0)
        g.time_steps(hg.SCHEME_RK3, steps, 0.0, dt)
        r = g.state()[0::4]
        out[name] = float(np.linalg.norm(r - ref[against]) / np.linalg.norm(ref[against]))
        g.close()
    return {"sample": f"{n}x{n} elements of the kh workload (N=7, same physics, dt = {KH_DT_COEF}/n^2 = {dt:.3e}), "
                      f"{steps} RK3 steps from the same state (t = {steps * dt:.3e}); oracle runs {oracle_s:.1f} s",
            "reference": "FP64 oracle: modal indicator for the plain paths; for fp32_learned the oracle with the "
                         "learned indicator evaluated in FP64 (oracle/mlp.py) at each step's start",
            "rel_l2_density": out, "tolerance": 1e-5}


def run_kh(args, rank, world, local, dist):
    """The Kelvin-Helmholtz shear layer (configuration C5: NS, SIPG, Roe, Laplacian artificial viscosity).
    value = the plain FP64 path (modal-decay sensor); the FP32-bulk + learned-sensor path is timed beside
    it on the same workload; roofline of the dominant kernel from the timed region; density error of each
    path against the FP64 oracle on a bounded sample."""
    import torch
    import horses2d_b200 as hg
    from horses2d_b200 import sensor as S, mesh as hmesh
    n, N = args.kh_n, 7
    cfg = workload_config("kh", args, world)
    t0 = time.perf_counter()
    params, lo, hi, info = S.train_two_rounds(100, SEED, nx=512, ny=64, N=3, steps=100, epochs=30, batch=4096)
    train_s = time.perf_counter() - t0
    xi, _ = hg._lib.nodes(N, hg.NODES_LG)
    Qh = kh_state_pinned(n, N, xi, SEED)
    desc = hmesh.box_descriptor(n, n, 0.0, 1.0, 0.0, 1.0, N, hg.NODES_LG)
    stream = torch.cuda.Stream()

    def context(prec, learned):
        g = hg.GpuDGSEM(desc, precision=prec, **kh_kwargs(hg))
        g.set_stream(stream.cuda_stream)
        g.set_state(Qh.numpy())
        if learned:
            g.set_sensor(hg.SENSOR_LEARNED, mlp=params, lo=lo, hi=hi)
        else:
            g.set_sensor(hg.SENSOR_MODAL)
        return dict(g=g, Qh=Qh, N=N, ninst=1, cfl=None, tune=g.autotune(trials=5))

    c64 = [context(hg.PREC_FP64, False)]
    c32 = [context(hg.PREC_FP32, True)]
    del desc
    g64, g32 = c64[0]["g"], c32[0]["g"]
    ndof = g64.ndof
    assert ndof == cfg["ndof"]
    dt = cfg["dt"]
    flush = L2Flush(False)       # Q alone is 2.1 GB: inputs larger than L2
    clocks = ClockSampler(local)
    clocks.start()
    ms64, launches = device_timed(c64, args.steps, args.warmup, dt, stream, world, dist, flush, min_load_s=2.0)
    clk = clocks.stop()
    ms32, _ = device_timed(c32, args.steps, args.warmup, dt, stream, world, dist, flush)
    split_steps = max(3, min(args.steps, 5))
    split64 = kernel_split(c64, split_steps, dt, stream, flush)
    split32 = kernel_split(c32, split_steps, dt, stream, flush)
    # sensor statistics of the learned path on the stepped state
    _, out32 = g32.sensor_eval()
    # end to end through the public API with host buffers (plain FP64 path): state from pinned host,
    # K x (hg_time_step + hg_residuals), the final state into pinned host
    Qpin = torch.empty(ndof, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    g64.set_state(Qh.numpy())
    res = np.zeros(4)
    for k in range(args.steps):
        g64.time_step(hg.SCHEME_RK3, k * dt, dt)
        res = np.maximum(res, g64.residuals())
    Qe = g64.state(out=Qpin.numpy())
    e2e_ms = (time.perf_counter() - t1) * 1e3
    if not (np.all(np.isfinite(Qe)) and np.all(np.isfinite(res))):
        raise SystemExit("non-finite state after the timed steps")
    del Qe
    ms64, ms32, e2e_ms = max_over_ranks([ms64, ms32, e2e_ms], world, dist)
    value = ndof * 3 * args.steps * world / (ms64 * 1e-3)
    value32 = ndof * 3 * args.steps * world / (ms32 * 1e-3)
    peak, peak_kind = peaks()
    roof64 = roofline_from_split(split64, split_steps, ms64 / args.steps, ndof, False, True, False, peak, peak_kind,
                                 "ns_stage_kernel_kh_fp64")
    roof32 = roofline_from_split(split32, split_steps, ms32 / args.steps, ndof, True, True, False, peak, peak_kind,
                                 "ns_stage_kernel_kh_fp32")
    troubled = float((out32[:, 3] > S.TROUBLED).mean())
    line = {"metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms64 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "tiling": tiling_summary(c64),
            "e2e": {"value": ndof * 3 * args.steps * world / (e2e_ms * 1e-3), "unit": "DOF-stage/s",
                    "h2d_bytes_per_step": ndof * 8 / args.steps, "d2h_bytes_per_step": 32 + ndof * 8 / args.steps,
                    "note": "hg_set_state from pinned host, K x (hg_time_step + hg_residuals), hg_get_state into "
                            "pinned host; plain FP64 path"},
            "gpu_launches": launches,
            "roofline": roof64["kernel"], "step_roofline": roof64["step"], "kernel_share": roof64["share"],
            "fp32_learned": {"value": value32, "ms_per_step": ms32 / args.steps, "dtype": "f32+f64acc",
                             "speedup_vs_fp64_plain": ms64 / ms32, "tiling": tiling_summary(c32),
                             "roofline": roof32["kernel"], "step_roofline": roof32["step"],
                             "kernel_share": roof32["share"],
                             "sensor": {"training_s": train_s, "training_snapshots": 200,
                                        "troubled_fraction": troubled,
                                        "fires_on_this_workload": bool(troubled > 0.0),
                                        "ood_fraction": float(out32[:, 2].mean()),
                                        "disagreement_vs_modal": S.disagreement(out32[:, 0], out32[:, 3]),
                                        "note": ("the learned indicator runs every step (inference fused into the "
                                                 "epilogue of each step's last stage); the shear layer is smooth, "
                                                 "and it flags "
                                                 f"{troubled:.1%} of the elements (the modal indicator: "
                                                 f"{float((out32[:, 0] > S.TROUBLED).mean()):.1%})")}},
            "clocks": clk}
    if rank == 0 and not args.no_cpu_baseline:
        rate, cores, sample = CpuArm("kh").sample(12.0)
        line["cpu_baseline"] = {"value": rate, "unit": "DOF-stage/s", "cores": cores, "kind": "port", "sample": sample}
        line["accuracy"] = kh_accuracy(params, lo, hi)
    line["node_stage_per_s"] = line["value"] / 4.0   # DOF-stage/s over the 4 variables of a node
    if rank == 0:
        print(json.dumps(line), flush=True)
    for c in c32 + c64:
        c["g"].close()
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="kh", choices=CONFIGS)
    ap.add_argument("--precision", default=None, choices=["fp32", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kh-n", type=int, default=1024, help="elements per side of the kh workload")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    import horses2d_b200 as hg
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    if args.config == "shock":
        return run_shock(args, rank, world, local, dist)
    if args.config == "kh":
        return run_kh(args, rank, world, local, dist)
    precision = args.precision or ("fp32" if args.config == "ensemble" else "fp64")
    prec = hg.PREC_FP32 if precision == "fp32" else hg.PREC_FP64
    parts = build_parts(args.config)
    stream = torch.cuda.Stream()
    ctxs = make_contexts(parts, prec, stream)
    ndof = sum(c["g"].ndof for c in ctxs)
    dt = min(c["g"].estimate_time_step(c["cfl"], 1.0) for c in ctxs)
    affine = all(c["g"].info()["affine"] for c in ctxs)
    ns = any(p[4].get("navier_stokes") for p in parts)
    flush = L2Flush(ndof * 8 * 3 < 2 * L2_BYTES)
    torch.cuda.synchronize()

    # ---- device-resident timed region
    clocks = ClockSampler(local)
    clocks.start()
    ms, launches = device_timed(ctxs, args.steps, args.warmup, dt, stream, world, dist, flush, min_load_s=2.0)
    clk = clocks.stop()
    # ---- per-kernel split (library CUDA-event timing, separate loop)
    split = kernel_split(ctxs, max(3, min(args.steps, 10)), dt, stream, flush)
    # ---- end to end through the public API with host buffers
    res_host = np.zeros(4)
    Qpin = [torch.empty(c["g"].ndof, dtype=torch.float64).pin_memory() for c in ctxs]   # result buffers
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record(stream)
    for c in ctxs:
        c["g"].set_state(c["Qh"].numpy())
    for s in range(args.steps):
        for c in ctxs:
            c["g"].time_step(hg.SCHEME_RK3, s * dt, dt)
            res_host = np.maximum(res_host, c["g"].residuals())
    Qout = [c["g"].state(out=q.numpy()) for c, q in zip(ctxs, Qpin)]
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3)
    if not np.all(np.isfinite(res_host)) or not all(np.all(np.isfinite(q)) for q in Qout):
        raise SystemExit("non-finite state after the timed steps")
    ms, e2e_ms = max_over_ranks([ms, e2e_ms], world, dist)
    value = ndof * 3 * args.steps * world / (ms * 1e-3)
    e2e = ndof * 3 * args.steps * world / (e2e_ms * 1e-3)

    # ---- roofline of the dominant kernel (fused stage kernel), launch time from the timed region
    peak, peak_kind = peaks()
    br1 = any(p[4].get("navier_stokes") and p[4].get("viscous", 0) == hg.BR1 for p in parts)
    roof = roofline_from_split(split, max(3, min(args.steps, 10)), ms / args.steps, ndof, prec == hg.PREC_FP32,
                               affine, br1, peak, peak_kind,
                               f"{'ns_' if ns else ''}stage_kernel_{args.config}_{precision}", ns=ns)
    line = {"metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64acc" if prec == hg.PREC_FP32 else "f64",
            "data": "synthetic", "config": workload_config(args.config, args, world), "tiling": tiling_summary(ctxs),
            "e2e": {"value": e2e, "unit": "DOF-stage/s", "h2d_bytes_per_step": ndof * 8 / args.steps,
                    "d2h_bytes_per_step": 32 * len(ctxs) + ndof * 8 / args.steps,
                    "note": "hg_set_state from pinned host, K x (hg_time_step + hg_residuals), hg_get_state "
                            "into pinned host; consecutive steps, no L2 flush"},
            "gpu_launches": launches,
            "roofline": roof["kernel"], "step_roofline": roof["step"], "kernel_share": roof["share"],
            "clocks": clk}

    if args.config == "ensemble":
        lc = bucket_launch_cost(prec, stream, dt)
        lc["extra_share_of_step"] = (lc["five_orders_ms_per_step"] - lc["one_order_ms_per_step"]) / (ms / args.steps)
        line["bucket_launches"] = lc

    # ---- FP32-bulk companion on the same workload (FP64 runs): speed and density error after K steps
    if prec == hg.PREC_FP64 and args.config == "cylinder":
        c32 = make_contexts(parts, hg.PREC_FP32, stream)
        ms32, _ = device_timed(c32, args.steps, args.warmup, dt, stream, 1, dist, flush)
        for c in ctxs + c32:
            c["g"].set_state(c["Qh"].numpy())
        for s in range(args.steps):
            for c in ctxs + c32:
                c["g"].time_step(hg.SCHEME_RK3, s * dt, dt)
        r64 = np.concatenate([c["g"].state().reshape(-1, 4)[:, 0] for c in ctxs])
        r32 = np.concatenate([c["g"].state().reshape(-1, 4)[:, 0] for c in c32])
        line["fp32_bulk"] = {"value": ndof * 3 * args.steps / (ms32 * 1e-3), "ms_per_step": ms32 / args.steps,
                             "speedup_vs_fp64": ms / ms32,
                             "rel_l2_density_vs_fp64_after_K_steps": float(np.linalg.norm(r32 - r64)
                                                                           / np.linalg.norm(r64))}
        for c in c32:
            c["g"].close()
    if rank == 0 and not args.no_cpu_baseline:
        rate, cores, sample = CpuArm(args.config).sample(12.0)
        line["cpu_baseline"] = {"value": rate, "unit": "DOF-stage/s", "cores": cores, "kind": "port",
                                "sample": sample}
    line["node_stage_per_s"] = line["value"] / 4.0   # DOF-stage/s over the 4 variables of a node
    if rank == 0:
        print(json.dumps(line), flush=True)
    for c in ctxs:
        c["g"].close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
