#!/usr/bin/env python
"""Benchmark: DGSEM time steps of the 3D Navier-Stokes Taylor-Green vortex.

Workload (default): periodic 32^3 hexahedral mesh on [0, 2pi]^3, N = 3 on
Gauss-Lobatto nodes (128^3 nodes, 5 conserved fields), Mach 0.1, Re 1600,
Pr 0.71, gamma 1.4, Chandrashekar flux differencing with the reference's
surface flux, BR1 lifting, Carpenter-Kennedy LSRK4(5), FP64, seeded-free
synthetic initial condition (the standard TGV).  One "step" is one full RK
time step (5 RHS evaluations with fused stage updates).

metric: DOF-updates/s = nodes * fields * steps / device time (whole job over
all ranks).  Every rank runs an independent replica (no collectives on the
data path); the timed region is bracketed by a barrier and synchronisation
and the maximum over ranks is used.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the CPU implementation of the same path on the host
cores (all threads) on a bounded sample of the workload; under torchrun only
rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 2 ** 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=32, help="elements per direction")
    p.add_argument("--order", type=int, default=3)
    p.add_argument("--quirks", choices=["reference", "fixed"], default="fixed")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-fp64-peak", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    return p.parse_args()


def workload_name(n, order):
    return f"tgv3d_navier_stokes_{n}^3_N{order}_lsrk45_fp64"


def physics():
    return dict(parabolic=True, blending=False, mu=1.0 / 1600.0, Pr=0.71, gamma=1.4)


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- algorithmic cost
def algorithmic_bytes(mesh, kernel):
    """Compulsory DRAM bytes of one launch: every input read once, every output
    written once (FP64).  S = one state vector."""
    S = mesh.num_fields * mesh.ndof * 8
    dim, E = mesh.dim, mesh.num_elements
    tables = E * (dim * dim + 1) * 8 + E * 2 * dim * 16 + mesh.num_faces * dim * 8
    if kernel == "lift":      # read u, write dim gradient vectors
        return S + dim * S + tables
    # rhs with LSRK epilogue: read u, gradients, du; write du, u_out
    return S + dim * S + S + S + S + tables


def flops_per_launch(mesh, kernel):
    """FP64 operations of one launch from the operation counts of the
    point-wise routines (add/mul/div/sqrt/log = 1, FMA = 2)."""
    Np, dim, E = mesh.order + 1, mesh.dim, mesh.num_elements
    nd = Np ** dim
    nf = dim + 2
    pairs = dim * Np ** (dim - 1) * Np * (Np - 1) // 2
    faces = 2 * dim * Np ** (dim - 1)
    if kernel == "lift":
        ent = 40            # entropy variables incl. log and pow as 1 each
        per = (nd + faces) * ent + nd * dim * Np * nf * 2 + nd * dim * dim * nf * 2 + nd * dim * 35
        return E * per
    vol_pair = 123 + 2 * nf * 2      # Chandrashekar volume flux + two D-weighted accumulations
    face_item = 150 + 2 * 60 + dim * nf * 2 + nf * 2
    visc_node = 60 + dim * dim * nf * 2 + dim * Np * nf * 2
    per = pairs * vol_pair + faces * face_item + nd * visc_node + nd * nf * 6
    return E * per


# ---------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{index}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        s, m = float(parts[1]), float(parts[2])
                    except ValueError:
                        continue
                    mx = m
                    sm.append(s)
                    for nm, v in zip(names, parts[5:9]):
                        if v.lower() == "active":
                            reasons.add(nm)
        except OSError:
            return None
        if not sm:
            return None
        load = [s for s in sm if s > 0.5 * (mx or 1)] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU side
def _cpu_worker(job):
    """One CPU replica: LSRK4(5) steps of the TGV sample mesh.  kind 'reference'
    runs the reference's own integrator sources (oracle/_ref), kind 'port' the
    oracle restatement.  Returns (DOF updates, seconds)."""
    kind, n_cpu, order, steps, seconds, threads = job
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import pyoracle
    from prandtl_b200 import cases
    from prandtl_b200.mesh import periodic_box
    mesh = periodic_box(3, n_cpu, order, 0.0, 2 * np.pi)
    u = cases.taylor_green(mesh)
    kw = dict(parabolic=1, blending=0, mu=1.0 / 1600.0, Pr=0.71, gamma=1.4)
    cls = pyoracle.RefOperator if kind == "reference" else pyoracle.Oracle
    op = cls(mesh, nthreads=threads, **kw)
    lam = pyoracle.Oracle(mesh, nthreads=1, **kw).rhs(u)["lambda_max"]
    dt = 0.1 * mesh.hmin / (lam * (order + 1) ** 2)
    u = op.step(u, dt, scheme=1, nsteps=1)   # warm-up
    done, t0 = 0, time.perf_counter()
    while True:
        u = op.step(u, dt, scheme=1, nsteps=1)
        done += 1
        el = time.perf_counter() - t0
        if (steps is not None and done >= steps) or (steps is None and el >= seconds):
            break
    return mesh.ndof * mesh.num_fields * done, el, done


def cpu_rate(order, steps=None, seconds=12.0):
    """DOF-updates/s of the CPU path on the host cores.

    With the reference's own sources built (oracle/_ref) this is the
    reference: one process per core, each advancing its own 4^3-element TGV
    sample (the reference scales over cores by MPI domain decomposition,
    run.sh `mpiexec -n`).  Otherwise the oracle port runs 8^3 elements with one
    OpenMP thread per core."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import multiprocessing as mp
    import pyoracle
    cores = os.cpu_count() or 1
    if pyoracle.ref_available():
        n_cpu, kind = 4, "reference"
        jobs = [(kind, n_cpu, order, steps, seconds, 1)] * cores
        with mp.get_context("spawn").Pool(cores) as pool:
            res = pool.map(_cpu_worker, jobs)
        upd = sum(r[0] for r in res)
        el = max(r[1] for r in res)
        nstep = res[0][2]
        sample = (f"reference DGSEM sources (oracle/_ref, -O2) x {cores} processes, each TGV "
                  f"{n_cpu}^3 elements N={order}, {nstep} LSRK4(5) steps")
    else:
        n_cpu, kind = 8, "port"
        with mp.get_context("spawn").Pool(1) as pool:
            upd, el, nstep = pool.map(_cpu_worker, [(kind, n_cpu, order, steps, seconds, cores)])[0]
        sample = (f"oracle C++ restatement -O2, {cores} OpenMP threads, TGV {n_cpu}^3 elements "
                  f"N={order}, {nstep} LSRK4(5) steps")
    return upd / el, dict(kind=kind, cores=cores, steps=nstep, seconds=el, sample=sample)


def run_reference(args, rank):
    if rank != 0:
        return
    # W warm-up steps, then K timed steps of the sample workload
    cpu_rate(args.order, steps=max(1, args.warmup))
    rate, info = cpu_rate(args.order, steps=max(1, args.steps))
    line = {
        "metric": "DOF-updates/s/GPU", "value": rate, "unit": "DOF-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * info["seconds"] / max(1, info["steps"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (standard TGV initial condition)",
        "config": {"workload": workload_name(args.n, args.order), "order": args.order,
                   "scheme": "LSRK45", "quirks": "reference (the reference's own code)"},
        "cpu_baseline": {"value": rate, "unit": "DOF-updates/s", "cores": info["cores"],
                         "kind": info["kind"], "sample": info["sample"]},
        "e2e": {"value": rate, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU side
def fp64_peak_tflops(torch):
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2 * 8192 ** 3 / best / 1e12


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import numpy as np
    import torch
    from prandtl_b200 import cases
    from prandtl_b200.mesh import periodic_box
    from prandtl_b200.operator import DGSEMOperator

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    mesh = periodic_box(3, args.n, args.order, 0.0, 2 * np.pi)
    u0 = cases.taylor_green(mesh)
    op = DGSEMOperator(mesh, quirks=args.quirks, **physics())
    stream = torch.cuda.current_stream()
    op.set_stream(stream.cuda_stream)
    u = torch.from_numpy(u0).cuda()
    dudt = torch.empty_like(u)
    op.Mult(u, dudt)
    lam = op.GetMaxCharSpeed()
    dt = op.cfl_dt(0.1, lam)    # CFL 0.1 as the reference TGV case (Simulation.cpp:906)

    for _ in range(args.warmup):
        op.Step(u, dt, scheme="LSRK45")
    torch.cuda.synchronize()

    op.profile(True)
    op.profile_reset()
    launches0 = op.kernel_launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            op.Step(u, dt, scheme="LSRK45")
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
    elapsed = ev0.elapsed_time(ev1) / 1e3
    launches = op.kernel_launches - launches0
    prof = op.profile_read()
    op.profile(False)
    if dist is not None:
        t = torch.tensor([elapsed], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    finite = bool(torch.isfinite(u).all().item())

    dof = mesh.ndof * mesh.num_fields
    value = dof * args.steps * world / elapsed

    # ---- end to end through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        host = torch.from_numpy(u0.copy()).pin_memory()
        for _ in range(2):
            op.Step(host, dt, scheme="LSRK45")
        torch.cuda.synchronize()
        ke = max(3, min(args.steps, 50))
        barrier()
        t0 = time.perf_counter()
        for _ in range(ke):
            op.Step(host, dt, scheme="LSRK45")   # H2D u, 5 fused stages, D2H u, wait
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([el], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        e2e = {"value": dof * ke * world / el, "unit": "DOF-updates/s",
               "h2d_bytes_per_step": dof * 8, "d2h_bytes_per_step": dof * 8, "steps": ke}

    # ---- roofline of the dominant kernel (device time measured with events above)
    hbm_peak, peak_kind = load_peaks()
    dom = max(prof, key=lambda k: prof[k][0])
    ms, n = prof[dom]
    t_launch = ms / 1e3 / max(1, n)
    ab = algorithmic_bytes(mesh, dom)
    fl = flops_per_launch(mesh, dom)
    fp64_peak = fp64_peak_tflops(torch) if (rank == 0 and not args.no_fp64_peak) else None
    gbs = ab / t_launch / 1e9
    tfl = fl / t_launch / 1e12
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            with open(tpath) as f:
                traffic = json.load(f).get(f"{dom}_bytes_per_launch")
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
                "frac": gbs / hbm_peak, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": traffic, "algorithmic_bytes_per_launch": ab,
                "avg_launch_ms": t_launch * 1e3,
                "fp64": {"achieved_tflops": tfl, "peak_tflops": fp64_peak,
                         "frac": (tfl / fp64_peak) if fp64_peak else None,
                         "peak_source": "measured live: cuBLAS DGEMM 8192^3 (torch.matmul float64)",
                         "flops_per_launch": fl},
                "kernels": {k: {"total_ms": v[0], "launches": v[1]} for k, v in prof.items()}}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            rate, info = cpu_rate(args.order, seconds=args.cpu_seconds)
            cpu = {"value": rate, "unit": "DOF-updates/s", "cores": info["cores"],
                   "kind": info["kind"], "sample": info["sample"]}
        except Exception as exc:   # the oracle build is missing on this host
            cpu = {"value": None, "unit": "DOF-updates/s", "cores": os.cpu_count(),
                   "kind": "port", "sample": f"unavailable: {exc}"}

    if rank == 0:
        S = dof * 8
        line = {
            "metric": "DOF-updates/s/GPU", "value": value, "unit": "DOF-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (standard TGV initial condition, no dataset)",
            "config": {"workload": workload_name(args.n, args.order), "mesh": f"{args.n}^3 periodic hex",
                       "order": args.order, "dof": dof, "scheme": "LSRK45", "cfl": 0.1,
                       "quirks": args.quirks, "parallelism": f"replicas x{world}",
                       "l2": f"no flush: working set {(7 * S) / 2**20:.0f} MiB per stage > 126 MiB L2"},
            "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
            "finite": finite,
        }
        clk_sum = clk.summary()
        line["clocks"] = clk_sum
        print(json.dumps(line), flush=True)
    op.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
