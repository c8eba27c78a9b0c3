"""Benchmark of the B200 DGSEM residual + Williamson RK3 stepper (DOF-stage updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--precision fp32|fp64]
    python bench.py --impl reference ...      # CPU arm: the oracle restatement on all host cores

One "step" is one Williamson RK3 time step (3 residual evaluations + updates)
over the whole workload.  DOF-stage updates/s = NDOF * 3 * K / time, NDOF =
size(Storage%Q) = 4 x nodes (the reference's DOF count, DGSEM_class.f90:337-340).

Workloads (synthetic inputs with the configurations' shapes; seeds fixed):
  ensemble : 512 periodic isentropic-vortex instances on [-5,5]^2, n x n elements with
             n ~ U{8..48}, N ~ U{3..7}, vortex centre ~ U[-2,2]^2, beta ~ U[2,6],
             M 0.5 at 45 deg, LGL nodes, Roe, packed by polynomial order into one
             element list per order; FP32 bulk with FP64 state accumulator by default.
  vortex16 : the reference-runnable case: 16 x 16 periodic vortex, N = 4, LGL, Roe, FP64.
  box512   : one 512 x 512 periodic vortex box, N = 4, LGL, Roe, FP64 (profiling case).
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


def build_buckets(config, precision):
    """[(descriptor, Q0, N, n_instances)] per polynomial order."""
    from horses2d_b200 import mesh as hmesh, cases, NODES_LGL
    if config == "vortex16":
        inst = [dict(n=16, N=4, xc=0.0, yc=0.0, beta=5.0)]
    elif config == "box512":
        inst = [dict(n=512, N=4, xc=0.0, yc=0.0, beta=5.0)]
    elif config == "ensemble":
        inst = ensemble_spec()
    else:
        raise SystemExit(f"unknown config {config}")
    buckets = []
    for N in sorted({i["N"] for i in inst}):
        descs, qs = [], []
        eo = fo = 0
        for it in (i for i in inst if i["N"] == N):
            d = hmesh.box_descriptor(it["n"], it["n"], -5.0, 5.0, -5.0, 5.0, N, NODES_LGL, elem_offset=eo, edge_offset=fo)
            x = d["x"].reshape(-1, 2)
            qs.append(cases.isentropic_vortex(x[:, 0], x[:, 1], mach=0.5, beta=it["beta"], xc=it["xc"], yc=it["yc"]))
            eo += len(d["N"])
            fo += len(d["edge_marker"])
            descs.append(d)
        buckets.append((hmesh.concat_descriptors(descs), np.concatenate(qs).ravel(), N,
                        sum(1 for i in inst if i["N"] == N)))
    return buckets


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


# ----------------------------------------------------------------------------- reference arm (CPU)
def cpu_rate(config, budget_s=12.0, threads=None):
    """Oracle restatement timed on the host cores on a bounded sample of the workload.

    Instances of the workload are stepped concurrently (one oracle per thread; the
    ctypes calls release the GIL).  Returns (DOF-stage/s, cores, sample text)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    from horses2d_b200 import mesh as hmesh, cases
    threads = threads or os.cpu_count() or 1
    inst = ensemble_spec() if config == "ensemble" else [dict(n=16, N=4, xc=0.0, yc=0.0, beta=5.0)]
    if config == "box512":
        inst = [dict(n=64, N=4, xc=0.0, yc=0.0, beta=5.0)]
    sample = inst[:threads] if config == "ensemble" else inst * threads
    orcs = []
    for it in sample:
        o = O.Oracle(hmesh.cartesian(it["n"], it["n"], -5.0, 5.0, -5.0, 5.0), it["N"], nodes=O.LGL, riemann=O.ROE,
                     mach=0.5, bcs=hmesh.periodic_bcs_cartesian())
        X = o.coords()
        o.set_state(cases.isentropic_vortex(X[:, 0], X[:, 1], beta=it["beta"], xc=it["xc"], yc=it["yc"]).ravel())
        orcs.append((o, o.estimate_dt(0.4, 1.0)))

    def run(arg):
        o, dt = arg
        t0 = time.perf_counter()
        steps = 0
        while time.perf_counter() - t0 < budget_s:
            o.time_step(O.RK3, steps * dt, dt)
            steps += 1
        return o.ndof * 3 * steps, time.perf_counter() - t0

    with ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(run, orcs))
    rate = sum(r[0] / r[1] for r in res)
    txt = (f"{len(sample)} instance(s) ({', '.join(str(it['n']) + 'x' + str(it['n']) + ' N=' + str(it['N']) for it in sample[:4])}"
           f"{', ...' if len(sample) > 4 else ''}), RK3 steps for ~{budget_s:.0f} s each, one oracle per host thread")
    return rate, threads, txt


def run_reference(args, rank, world):
    if rank != 0:
        return
    per_step_rates = []
    cores = 0
    sample = ""
    for s in range(args.warmup + args.steps):
        rate, cores, sample = cpu_rate(args.config, budget_s=3.0)
        if s >= args.warmup:
            per_step_rates.append(rate)
    value = float(np.mean(per_step_rates))
    line = {"impl": "reference", "metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.config},
            "cpu_baseline": {"value": value, "unit": "DOF-stage/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Fortran needs gfortran + NetCDF-Fortran (absent); its C++ FP64 restatement is timed"}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="ensemble", choices=["ensemble", "vortex16", "box512"])
    ap.add_argument("--precision", default=None, choices=["fp32", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    precision = args.precision or ("fp32" if args.config == "ensemble" else "fp64")
    prec = hg.PREC_FP32 if precision == "fp32" else hg.PREC_FP64
    buckets = build_buckets(args.config, prec)
    stream = torch.cuda.Stream()
    ctxs = []
    for desc, Q0, N, ninst in buckets:
        g = hg.GpuDGSEM(desc, mach=0.5, node_type=hg.NODES_LGL, riemann=hg.ROE, bcs=[dict(type=hg.BC_PERIODIC)] * 4,
                        precision=prec)
        g.set_stream(stream.cuda_stream)
        Qh = torch.from_numpy(Q0).pin_memory()
        ctxs.append((g, Qh, N, ninst))
    ndof = sum(g.ndof for g, _, _, _ in ctxs)
    for g, Qh, _, _ in ctxs:
        g.set_state(Qh.numpy())
    dt = min(g.estimate_time_step(0.4, 1.0) for g, _, _, _ in ctxs)
    torch.cuda.synchronize()

    def step(s):
        for g, _, _, _ in ctxs:
            g.time_step(hg.SCHEME_RK3, s * dt, dt)

    for s in range(args.warmup):
        step(s)
    torch.cuda.synchronize()
    # ---- device-resident timed region
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = sum(g.launch_count() for g, _, _, _ in ctxs)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for s in range(args.steps):
        step(args.warmup + s)
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    launches = sum(g.launch_count() for g, _, _, _ in ctxs) - launches0
    clk = clocks.stop()
    # ---- end to end through the public API with host buffers
    res_host = np.zeros(4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for g, Qh, _, _ in ctxs:
        g.set_state(Qh.numpy())
    for s in range(args.steps):
        step(s)
        for g, _, _, _ in ctxs:
            res_host = np.maximum(res_host, g.residuals())
    Qout = [np.empty(g.ndof) for g, _, _, _ in ctxs]
    for (g, _, _, _), q in zip(ctxs, Qout):
        q[:] = g.state()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3)
    if not np.all(np.isfinite(res_host)) or not all(np.all(np.isfinite(q)) for q in Qout):
        raise SystemExit("non-finite state after the timed steps")
    t_max = torch.tensor([ms, e2e_ms], device="cuda")
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms, e2e_ms = float(t_max[0]), float(t_max[1])
    value = ndof * 3 * args.steps * world / (ms * 1e-3)
    e2e = ndof * 3 * args.steps * world / (e2e_ms * 1e-3)
    # roofline of the dominant kernel (the fused stage kernel is every launch of the timed region)
    sq, sg = 8, (4 if prec == hg.PREC_FP32 else 8)
    bytes_step = ndof * (3 * (sq + sq + sg) + 2 * sg)           # Q r/w + G w every stage, G r in stages 2-3
    n_stage_launches = 3 * args.steps * len(ctxs)
    avg_launch_s = ms * 1e-3 / n_stage_launches
    bytes_per_launch = bytes_step * args.steps / n_stage_launches
    achieved = bytes_per_launch / avg_launch_s / 1e9
    peak, peak_kind = peaks()
    traffic = None
    tpath = os.path.join(ROOT, "profiles", f"stage_kernel_{args.config}_{precision}.traffic.json")
    if os.path.exists(tpath):
        try:
            t = json.load(open(tpath))
            traffic = t["bytes_per_dof_stage"] * ndof / len(ctxs)
        except Exception:
            traffic = None
    line = {"metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64acc" if prec == hg.PREC_FP32 else "f64",
            "data": "synthetic",
            "config": {"workload": args.config, "ndof": ndof, "precision": precision,
                       "orders": [c[2] for c in ctxs], "instances": sum(c[3] for c in ctxs),
                       "scheme": "Williamson RK3", "l2": "inputs larger than L2" if ndof * 8 > L2_BYTES
                       else "working set fits L2 (no flush)", "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e, "unit": "DOF-stage/s", "h2d_bytes_per_step": ndof * 8 / args.steps,
                    "d2h_bytes_per_step": 32 * len(ctxs) + ndof * 8 / args.steps,
                    "note": "hg_set_state from pinned host, K x (hg_time_step + hg_residuals), hg_get_state"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "algorithmic_bytes_per_dof_stage": bytes_step / ndof / 3},
            "clocks": clk}
    if rank == 0 and not args.no_cpu_baseline:
        rate, cores, sample = cpu_rate(args.config)
        line["cpu_baseline"] = {"value": rate, "unit": "DOF-stage/s", "cores": cores, "kind": "port",
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    for g, _, _, _ in ctxs:
        g.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
