#!/usr/bin/env python
"""Benchmark: the batched FP32-bulk DGSEM form against the plain FP64 path.

Headline workload ("tgv_ensemble_512"): 512 independent 3D Navier-Stokes
Taylor-Green vortices drawn with numpy PCG64(20261203).  Each member has n^3
periodic hexes on [0,2pi]^3 with n ~ U{4..16}, N ~ U{2,3,4,5},
Mach ~ U[0.05,0.3] and Re ~ logU[100,3200] (Pr 0.71, gamma 1.4); the total is
about 0.43 G DOF.  Each member takes Carpenter-Kennedy LSRK4(5) steps with
its own fixed dt (CFL 0.1 on the initial max |V|+c).  The inputs are
synthetic: the standard TGV initial condition, no dataset.  One "step"
advances every member by one RK step.  Per stage and per order class there is
one persistent lifting launch and one persistent RHS + stage-update launch,
replayed from a CUDA graph.

Keys of the JSON line:
  value       DOF-updates/s of the FP32-bulk batch: sum(nodes*fields) * K
              over the device time of K steps (CUDA events on the batch's
              stream).
  fp64_plain  the same metric for members advanced one at a time through the
              one-operator FP64 path (DGSEMOperator.Step) on every 8th member.
  error       FP32-batched vs FP64-plain states of those members after W+K
              steps: relative L2 and Linf of density, momentum (as a vector)
              and energy.
  tgv32       the 32^3 N=3 TGV (one solve) through the plain FP64 path, with
              its RHS kernel's FP64 roofline.
  serving     Poisson request stream through prandtl_serve_*: p50/p99
              time-to-solution and throughput.
  e2e         the headline metric through the C ABI with pinned host buffers:
              admission (H2D), tuning, W+K steps and reading every result
              (D2H), by wall clock (the clock sampler's own start and stop,
              0.4 s of sleeps, are left out of that window).
  roofline    the dominant launch (the N=5 class RHS): FP32 CUDA-core FLOP/s
              against the FP32 SGEMM rate measured live in this run, with the
              launch's HBM bytes alongside.

Every rank runs an independent replica: no collectives on the data path, a
barrier and device synchronisation around the timed region, and the maximum
time over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own DGSEM sources (oracle/_ref) on all
host cores, on a bounded sample of the same ensemble; under torchrun only
rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "tgv_ensemble_512"
CFL = 0.1


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--ensemble", type=int, default=512, help="members of the ensemble")
    p.add_argument("--plain-every", type=int, default=8, help="FP64-plain subsample stride")
    p.add_argument("--serve-requests", type=int, default=500)
    p.add_argument("--serve-only", action="store_true",
                   help="run only the serving stream and print its record (long streams, e.g. 10000 requests)")
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--no-tgv32", action="store_true")
    p.add_argument("--no-configs", action="store_true", help="skip the 2D vortex and Kelvin-Helmholtz keys")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-peaks", action="store_true", help="skip the live SGEMM/DGEMM peak runs")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--profile-case", choices=["batch", "tgv32"], default=None,
                   help="run only this part and print nothing (for ncu captures)")
    return p.parse_args()


def load_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- algorithmic cost
def flops_per_element(dim, order, ns=True):
    """Floating-point operations of one RHS launch per element, from the
    operation counts of the point-wise routines (add/mul/div/sqrt/log = 1,
    FMA = 2): two-point volume fluxes of every unique node pair with their two
    D-weighted accumulations, surface fluxes of the element's face nodes, the
    Dhat-divergence of the contravariant viscous fluxes and their signed face
    average (NS; the viscous fluxes themselves are the lifting's work), and
    the RK epilogue."""
    Np = order + 1
    nd, nf = Np ** dim, dim + 2
    pairs = dim * Np ** (dim - 1) * Np * (Np - 1) // 2
    faces = 2 * dim * Np ** (dim - 1)
    vol_pair = 123 + 2 * nf * 2
    face_item = 150 + dim * nf * 2 + nf * 2 + ((nf - 1) * 3 if ns else 0)
    visc_node = dim * Np * (nf - 1) * 2 if ns else 0
    return pairs * vol_pair + faces * face_item + nd * visc_node + nd * nf * 6


def rhs_bytes_per_element(dim, order, visc_bytes, ns=True):
    """Compulsory DRAM bytes of one RHS + LSRK launch per element: u read, the
    contravariant viscous fluxes read (NS: dim*(nf-1) values per node of
    visc_bytes each), du read and written, the next state written, and the
    geometry rows."""
    nd, nf = (order + 1) ** dim, dim + 2
    per_node = nf * (8 + 8 + 8 + 8) + (dim * (nf - 1) * visc_bytes if ns else 0)
    return nd * per_node + (dim * dim + 1) * 8 + 2 * dim * 16


def measured_traffic():
    """DRAM bytes per launch from the committed ncu summaries (profiles/)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples every 100 ms while the block runs; the
    CSV goes to PRANDTL_BENCH_CLOCKS_DIR if set, else a temporary folder."""

    def __init__(self, index, tag):
        import tempfile
        self.index = index
        self.proc = None
        self.overhead_s = 0.0   # time spent starting and stopping the sampler
        folder = os.environ.get("PRANDTL_BENCH_CLOCKS_DIR") or tempfile.mkdtemp(prefix="prandtl_clocks_")
        self.path = os.path.join(folder, f"clocks_{tag}_rank{index}.csv")

    def __enter__(self):
        t0 = time.perf_counter()
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        self.overhead_s += time.perf_counter() - t0
        return self

    def __exit__(self, *a):
        t0 = time.perf_counter()
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()
        self.overhead_s += time.perf_counter() - t0

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
    """One CPU process advances one ensemble member on its own mesh (the same
    n^3 elements, N, Mach and Re as in the GPU batch) with LSRK4(5) stages for
    a fixed wall-clock window, stage by stage.  kind 'reference' runs the
    reference's own DGSEM sources (oracle/_ref), kind 'port' the oracle
    restatement.  Returns (DOF updates, seconds, stages, elements, order)."""
    kind, index, seconds, threads = job
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import pyoracle
    from prandtl_b200.ensemble import fixed_dt, tgv_ensemble
    m = tgv_ensemble(index + 1)[index]
    mesh = m.mesh()
    u = m.initial_state(mesh)
    kw = dict(parabolic=1, blending=0, mu=1.0 / m.re, Pr=0.71, gamma=1.4, quirks=1)
    cls = pyoracle.RefOperator if kind == "reference" else pyoracle.Oracle
    op = cls(mesh, nthreads=threads, **kw)
    dt = fixed_dt(mesh, u, CFL)
    A, B = pyoracle._LSRK_A, pyoracle._LSRK_B
    du = np.zeros_like(u)
    op.rhs(u)   # warm-up
    stages, t0 = 0, time.perf_counter()
    while True:
        k = stages % 5
        du = A[k] * du + dt * op.rhs(u)["dudt"]
        u = u + B[k] * du
        stages += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return mesh.ndof * mesh.num_fields * stages / 5.0, el, stages, mesh.num_elements, m.order


def cpu_rate(seconds=12.0, single_core=True):
    """DOF-updates/s of the CPU path on all host cores: with the reference's own
    sources built (oracle/_ref) this is the reference, one process per core
    (the reference scales by MPI domain decomposition, run.sh `mpiexec -n`),
    process i advancing ensemble member i on its own mesh; otherwise the
    oracle restatement runs the same sample.  Every process runs for the same
    wall-clock window, so no core idles, and the rate is the sum of the
    processes' own rates.  With single_core, member 0 is also timed alone on
    one core."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import multiprocessing as mp
    import pyoracle
    cores = os.cpu_count() or 1
    kind = "reference" if pyoracle.ref_available() else "port"
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_cpu_worker, [(kind, i, seconds, 1) for i in range(cores)])
    rate = sum(r[0] / r[1] for r in res)
    one = None
    if single_core:
        # the sampled member of median size, alone on one core
        order = sorted(range(len(res)), key=lambda i: res[i][0] / max(1, res[i][2]))
        mid = order[len(order) // 2]
        with ctx.Pool(1) as pool:
            r1 = pool.map(_cpu_worker, [(kind, mid, seconds, 1)])[0]
        one = {"value": r1[0] / r1[1], "unit": "DOF-updates/s", "cores": 1,
               "sample": f"ensemble member {mid} ({r1[3]} elements, N={r1[4]}, the sample's median size) "
                         f"alone on one core, {r1[2]} LSRK stages in {r1[1]:.1f} s"}
    src = "reference DGSEM sources (oracle/_ref, -O2)" if kind == "reference" else "oracle C++ restatement -O2"
    elems = sorted({(r[3], r[4]) for r in res})
    sample = (f"{src} x {cores} processes, each for {seconds:.0f} s of wall clock: process i advances "
              f"ensemble member i on its own mesh (the batch's sizes: {len(res)} members, "
              f"{min(e for e, _ in elems)}..{max(e for e, _ in elems)} elements, N "
              f"{sorted({o for _, o in elems})}) with LSRK4(5) stages; rate = sum of the processes' rates; "
              f"{min(r[2] for r in res)}..{max(r[2] for r in res)} stages each")
    return rate, dict(kind=kind, cores=cores, seconds=max(r[1] for r in res),
                      stages=sum(r[2] for r in res), sample=sample, single_core=one)


def run_reference(args, rank):
    if rank != 0:
        return
    budget = max(10.0, min(120.0, 0.6 * (args.steps + args.warmup)))
    rate, info = cpu_rate(seconds=budget, single_core=False)
    line = {
        "metric": "DOF-updates/s/GPU", "value": rate, "unit": "DOF-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * info["seconds"] * 5.0 * info["cores"] / max(1, info["stages"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (standard TGV initial condition)",
        "config": {"workload": WORKLOAD, "scheme": "LSRK45", "cfl": CFL,
                   "sample": "each host core advances one ensemble member on its own mesh for the same window"},
        "cpu_baseline": {"value": rate, "unit": "DOF-updates/s", "cores": info["cores"],
                         "kind": info["kind"], "sample": info["sample"]},
        "e2e": {"value": rate, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU side
def max_over_ranks(dist, x, device):
    """The largest of every rank's x (each rank times its own replica; the job
    takes as long as its slowest rank).  dist is torch.distributed or None."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gemm_tflops(torch, dtype, n=8192):
    """Best-of-5 cuBLAS GEMM rate (TF32 off for float32: CUDA-core FP32)."""
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(n, n, dtype=dtype, device="cuda")
    b = torch.randn(n, n, dtype=dtype, device="cuda")
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
    torch.backends.cuda.matmul.allow_tf32 = old
    del a, b
    return 2 * n ** 3 / best / 1e12


def rel_errors(a, b, nf):
    """Relative L2 and Linf of density, momentum (vector) and energy."""
    import numpy as np
    a, b = a.reshape(nf, -1), b.reshape(nf, -1)
    out = {}
    for name, g in (("rho", [0]), ("momentum", list(range(1, nf - 1))), ("energy", [nf - 1])):
        d = a[g] - b[g]
        out[name] = (float(np.linalg.norm(d) / np.linalg.norm(b[g])), float(np.abs(d).max() / np.abs(b[g]).max()))
    return out


def build_items(members):
    from prandtl_b200.ensemble import fixed_dt
    items = []
    for m in members:
        mesh = m.mesh()
        u0 = m.initial_state(mesh)
        items.append((m, mesh, u0, fixed_dt(mesh, u0, CFL)))
    return items


def run_batch(torch, items, K, W, barrier, local):
    """FP32-bulk batch over all members.  The wall-clock window (e2e) spans
    admission from pinned host memory, W+K steps and reading every state back;
    the autotuner runs inside the first warm-up steps (one launch shape per
    step, timed by CUDA events around every launch), so it does real steps.
    The device window (value) spans the last K steps."""
    from prandtl_b200.batch import Batch
    pinned = [torch.from_numpy(u0).pin_memory() for _, _, u0, _ in items]
    outs = [torch.empty(p.shape, dtype=torch.float64).pin_memory() for p in pinned]
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    b = Batch("fp32", "LSRK45")
    ids = b.add_many([(mesh, pinned[k], dict(dt=dt, nsteps=W + K, **m.physics()))
                      for k, (m, mesh, _, dt) in enumerate(items)])
    b.sync()
    t_admit = time.perf_counter() - t0
    if W >= 3:   # the 3 launch shapes are timed inside the warm-up steps
        b.tune_in_steps()
    else:
        b.tune(reps=2)
    t_tw = time.perf_counter()
    b.advance(W)
    b.sync()
    t_warm = time.perf_counter() - t_tw
    stream = torch.cuda.ExternalStream(b.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = b.kernel_launches
    with ClockSampler(local, "batch") as clk:
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        b.advance(K)
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        barrier()
    device_s = ev0.elapsed_time(ev1) / 1e3
    launches = b.kernel_launches - launches0
    t_r = time.perf_counter()
    b.read_many(ids, outs)
    t_read = time.perf_counter() - t_r
    # the e2e window without the clock sampler's own start and stop (instrumentation)
    wall = time.perf_counter() - t0 - clk.overhead_s
    classes = {}
    for order in sorted({m.order for m, _, _, _ in items}):
        v, ms, lift = b.class_info(3, order, True)
        classes[order] = {"variant": v, "rhs_ms_per_variant": ms, "lift_ms": lift}
    info = {"device_s": device_s, "wall_s": wall, "launches": launches, "device_bytes": b.device_bytes,
            "window_s": {"admit": t_admit, "warmup_with_tuning": t_warm, "read": t_read, "total": wall},
            "classes": classes, "clocks": clk.summary()}
    b.close()
    return [o.numpy() for o in outs], info


def run_plain(torch, items, K, W, batch_states=None):
    """Members one at a time through the one-operator FP64 path: W untimed and
    K timed steps each (CUDA events on the current stream).  Outside the timed
    region, the FP64 device budgets (mass, energy, entropy) of the initial
    state, the final FP64 state and the member's final FP32-batched state."""
    from prandtl_b200.operator import DGSEMOperator
    stream = torch.cuda.current_stream()
    total_s, dofs, states, launches, budgets = 0.0, 0, [], 0, []
    for k, (m, mesh, u0, dt) in enumerate(items):
        op = DGSEMOperator(mesh, **m.physics())
        op.set_stream(stream.cuda_stream)
        u = torch.from_numpy(u0).cuda()
        op.Step(u, dt, scheme="LSRK45", nsteps=W)
        l0 = op.kernel_launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        op.Step(u, dt, scheme="LSRK45", nsteps=K)
        e1.record(stream)
        e1.synchronize()
        total_s += e0.elapsed_time(e1) / 1e3
        launches += op.kernel_launches - l0
        dofs += u0.size
        states.append(u.cpu().numpy())
        b0 = op.budgets(torch.from_numpy(u0).cuda())
        bp = op.budgets(u)
        bb = op.budgets(torch.from_numpy(batch_states[k]).cuda()) if batch_states is not None else None
        budgets.append((b0, bp, bb))
        op.close()
    return states, {"device_s": total_s, "dof": dofs, "launches": launches, "budgets": budgets}


def budget_summary(budgets, steps):
    """Largest relative drifts of mass and energy over the run, per path, and
    the FP32-batched vs FP64-plain entropy difference (relative to the initial
    entropy)."""
    def drift(b0, b1, f):
        return abs(b1["conserved"][f] - b0["conserved"][f]) / abs(b0["conserved"][f])
    out = {"members": len(budgets), "steps": steps,
           "reduction": "FP64 on the device, node weights w_i w_j w_k |J|, fixed-order two-pass sum"}
    for name, j in (("fp64_plain", 1), ("fp32_batched", 2)):
        if any(b[j] is None for b in budgets):
            continue
        out[name] = {"mass_rel_drift_max": max(drift(b[0], b[j], 0) for b in budgets),
                     "energy_rel_drift_max": max(drift(b[0], b[j], 4) for b in budgets),
                     "entropy_rel_change_max": max(abs(b[j]["entropy"] - b[0]["entropy"]) / abs(b[0]["entropy"])
                                                   for b in budgets)}
    if all(b[2] is not None for b in budgets):
        out["entropy_fp32_vs_fp64_rel_max"] = max(abs(b[2]["entropy"] - b[1]["entropy"]) / abs(b[0]["entropy"])
                                                  for b in budgets)
    return out


def run_tgv32(torch, steps, fp32_steps=200, extras=True):
    """BASELINE config 2, the 32^3 N=3 TGV (one solve), through the plain FP64
    path: per-kernel CUDA-event times of `steps` LSRK steps; the drop-in call
    pattern (DGSEMOperator::Mult on host vectors, one call per RK stage:
    pageable H2D, lift + RHS, D2H) by wall clock; and the FP32-bulk form against
    FP64 after `fp32_steps` steps at CFL 0.5 (L2 / Linf of rho, momentum, energy)."""
    import numpy as np
    from prandtl_b200 import cases
    from prandtl_b200.ensemble import fixed_dt
    from prandtl_b200.mesh import periodic_box
    from prandtl_b200.operator import DGSEMOperator
    mesh = periodic_box(3, 32, 3, 0.0, 2 * np.pi)
    u0 = cases.taylor_green(mesh)
    phys = dict(parabolic=True, mu=1.0 / 1600.0, Pr=0.71, quirks="fixed")
    op = DGSEMOperator(mesh, **phys)
    stream = torch.cuda.current_stream()
    op.set_stream(stream.cuda_stream)
    u = torch.from_numpy(u0).cuda()
    d = torch.empty_like(u)
    op.Mult(u, d)
    dt = op.cfl_dt(CFL, op.GetMaxCharSpeed())
    for _ in range(3):
        op.Step(u, dt, scheme="LSRK45")
    torch.cuda.synchronize()
    op.profile(True)
    op.profile_reset()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    op.Step(u, dt, scheme="LSRK45", nsteps=steps)
    e1.record(stream)
    torch.cuda.synchronize()
    el = e0.elapsed_time(e1) / 1e3
    prof = op.profile_read()
    op.profile(False)
    if not extras:
        op.close()
        return None
    # drop-in pattern: Mult with host (pageable) vectors, as mfem::ODESolver calls it
    uh = u.cpu().numpy()
    dh = np.empty_like(uh)
    op.Mult(uh, dh)
    reps = 10
    t0 = time.perf_counter()
    for _ in range(reps):
        op.Mult(uh, dh)
    mult_s = (time.perf_counter() - t0) / reps
    op.close()
    dof = mesh.ndof * mesh.num_fields
    rhs_ms = prof["rhs"][0] / prof["rhs"][1]
    lift_ms = prof["lift"][0] / prof["lift"][1]
    E = mesh.num_elements
    # FP32 bulk vs FP64 after fp32_steps steps at CFL 0.5
    dt5 = fixed_dt(mesh, u0, 0.5)
    fin, ftime = {}, {}
    for prec in ("fp64", "fp32"):
        o = DGSEMOperator(mesh, precision=prec, **phys)
        o.set_stream(stream.cuda_stream)
        x = torch.from_numpy(u0).cuda()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        o.Step(x, dt5, scheme="LSRK45", nsteps=fp32_steps)
        b.record(stream)
        o.synchronize()
        ftime[prec] = a.elapsed_time(b) / 1e3
        fin[prec] = x.cpu().numpy()
        o.close()
    return {"workload": "tgv3d_navier_stokes_32^3_N3_lsrk45_fp64", "dof": dof,
            "value": dof * steps / el, "unit": "DOF-updates/s", "ms_per_step": 1e3 * el / steps,
            "rhs_ms": rhs_ms, "lift_ms": lift_ms,
            "rhs_flops": E * flops_per_element(3, 3), "rhs_algorithmic_bytes": E * rhs_bytes_per_element(3, 3, 8),
            "dropin_mult_host": {
                "ms_per_call": 1e3 * mult_s, "kernels_ms": rhs_ms + lift_ms,
                "dof_rhs_per_s": dof / mult_s, "bytes_per_call": 2 * dof * 8,
                "pattern": "DGSEMOperator.Mult(u, dudt) on pageable numpy vectors: H2D of u, lift + RHS "
                           "kernels, D2H of dudt, wait; one call per RK stage as mfem::ODESolver::Step makes"},
            "fp32_vs_fp64": {"steps": fp32_steps, "cfl": 0.5, "scheme": "LSRK45",
                             **rel_errors(fin["fp32"], fin["fp64"], mesh.num_fields),
                             "fp64_dof_updates_per_s": dof * fp32_steps / ftime["fp64"],
                             "fp32_dof_updates_per_s": dof * fp32_steps / ftime["fp32"],
                             "format": "per field: [relative L2, relative Linf]"}}


def run_ivortex32(torch, steps=100):
    """2D Euler isentropic vortex 32^2 N=3 (plain method,
    FP64), SSP-RK3 at CFL 0.5 (dt from the initial lambda_max), `steps` steps."""
    from prandtl_b200 import cases
    from prandtl_b200.ensemble import fixed_dt
    from prandtl_b200.operator import DGSEMOperator
    mesh, u0, _ = cases.make_case("ivortex", 32, 3)
    op = DGSEMOperator(mesh, quirks="reference")
    stream = torch.cuda.current_stream()
    op.set_stream(stream.cuda_stream)
    u = torch.from_numpy(u0).cuda()
    dt = fixed_dt(mesh, u0, 0.5)
    op.Step(u, dt, scheme="RK3SSP", nsteps=3)
    op.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    op.Step(u, dt, scheme="RK3SSP", nsteps=steps)
    b.record(stream)
    op.synchronize()
    el = a.elapsed_time(b) / 1e3
    dof = mesh.ndof * mesh.num_fields
    op.close()
    return {"workload": "ivortex2d_euler_32^2_N3_ssprk3_fp64", "steps": steps, "dof": dof,
            "value": dof * steps / el, "unit": "DOF-updates/s", "ms_per_step": 1e3 * el / steps,
            "note": "65,536 DOF: far too small to fill a B200 (launch- and latency-bound)"}


def run_kh256(torch, t_final=3.0, precisions=("fp64", "fp32")):
    """2D Euler Kelvin-Helmholtz 256^2 N=3 with the modal
    indicator and subcell FV blending (alpha_max 0.5), SSP-RK3 with
    dt = 0.4 hmin / (lambda_max (N+1)^2) after every step (on the device), to
    t = 3, one batch solve per precision.  Every stage checks every node
    (non-finite, rho <= 0, p <= 0); mass and energy budgets on the device;
    the blending field at t = 3 from one RHS of the final state."""
    import numpy as np
    from prandtl_b200 import cases
    from prandtl_b200.batch import Batch
    from prandtl_b200.ensemble import fixed_dt
    from prandtl_b200.operator import DGSEMOperator
    mesh, u0, _ = cases.make_case("kh", 256, 3)
    phys = dict(blending=True, alpha_max=0.5, quirks="reference")
    out = {"workload": "kh2d_euler_256^2_N3_blended_ssprk3_cfl0.4_to_t3", "dof": mesh.ndof * mesh.num_fields}
    for prec in precisions:
        b = Batch(prec, "RK3SSP", arena_bytes=2 << 30)
        sid = b.add(mesh, u0, dt=fixed_dt(mesh, u0, 0.4), nsteps=1 << 30, cfl=0.4, t_final=t_final, **phys)
        b0 = b.budgets(sid)
        stream = torch.cuda.ExternalStream(b.stream)
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        status = "ok"
        a.record(stream)
        try:
            while sid not in b.finished():
                b.advance(2000)
                b.query(sid)
        except Exception as exc:   # a failed state check (PRANDTL_ENONFINITE) ends the run
            status = str(exc)
        e.record(stream)
        b.sync()
        dev_s = a.elapsed_time(e) / 1e3
        q = b.query(sid) if status == "ok" else {}
        t = b.time(sid)
        b1 = b.budgets(sid)
        u = b.read(sid) if status == "ok" else None
        b.close()
        rec = {"status": status, "t": t, "steps": q.get("steps_done"), "device_s": dev_s,
               "dof_updates_per_s": out["dof"] * q.get("steps_done", 0) / dev_s if q else None,
               "state_check": "every node of every stage: finite, rho > 0, p > 0" + (" - passed" if status == "ok"
                                                                                         else " - FAILED"),
               "mass_rel_drift": abs(b1["conserved"][0] - b0["conserved"][0]) / abs(b0["conserved"][0]),
               "energy_rel_drift": abs(b1["conserved"][3] - b0["conserved"][3]) / abs(b0["conserved"][3])}
        if u is not None:
            v = u.reshape(4, -1)
            p = 0.4 * (v[3] - 0.5 * (v[1] ** 2 + v[2] ** 2) / v[0])
            rec["min_rho"], rec["min_p"] = float(v[0].min()), float(p.min())
            op = DGSEMOperator(mesh, **phys)
            d = np.empty_like(u)
            op.Mult(u, d)
            al = op.alpha()
            op.close()
            rec["alpha_at_t"] = {"elements_blended": int((al > 0).sum()), "fraction": float((al > 0).mean()),
                                 "max": float(al.max()), "mean": float(al.mean())}
        out[prec] = rec
    return out


def run_ramp(torch, t_final=3.0, dt=1e-4):
    """The reference's axisymmetric 15-degree ramp case (TestCases/Euler/2D/Ramp:
    Mach-2 free stream, order 1, subcell FV blending, SSP-RK3 with the fixed dt
    1e-4 of its config, to t = 3) on a 98 x 49 structured ramp mesh whose cells
    over the cone are trapezoids: the FP64 kernels with per-node geometry.
    Every stage checks every node for non-finite values; the density and
    pressure range and the blending field are taken from the state at t = 3
    (at N = 1 the modal indicator has no resolved modes to compare, so every
    element takes alpha_max, as in the reference)."""
    import numpy as np
    from prandtl_b200 import cases
    from prandtl_b200.operator import DGSEMOperator
    mesh = cases.ramp_mesh(1)
    u0 = cases.ramp_ic(mesh)
    op = DGSEMOperator(mesh, quirks="reference", blending=True, bcs=cases.RAMP_BCS, axisymmetric=True)
    stream = torch.cuda.current_stream()
    op.set_stream(stream.cuda_stream)
    u = torch.from_numpy(u0).cuda()
    steps = int(round(t_final / dt))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    status, done = "ok", 0
    a.record(stream)
    try:
        while done < steps:
            k = min(2000, steps - done)
            op.Step(u, dt, scheme="RK3SSP", nsteps=k)   # raises on a failed state check
            done += k
    except Exception as exc:
        status = str(exc)
    b.record(stream)
    op.synchronize()
    el = a.elapsed_time(b) / 1e3
    dof = mesh.ndof * mesh.num_fields
    rec = {"workload": "ramp15_axisymmetric_euler_98x49_N1_blended_ssprk3_dt1e-4_to_t3",
           "mesh": "98 x 49 quadrilaterals, multilinear over the cone (per-node geometry)",
           "dof": dof, "status": status, "steps": done, "t": done * dt, "device_s": el,
           "dof_updates_per_s": dof * done / el, "ms_per_step": 1e3 * el / max(done, 1),
           "state_check": "every node of every stage: finite" + (" - passed" if status == "ok" else " - FAILED")}
    if status == "ok":
        rU = u.cpu().numpy()
        U = op.recover_state(rU).reshape(4, -1)
        p = 0.4 * (U[3] - 0.5 * (U[1] ** 2 + U[2] ** 2) / U[0])
        rec["min_rho"], rec["min_p"] = float(U[0].min()), float(p.min())
        rec["max_rho"], rec["max_p"] = float(U[0].max()), float(p.max())   # the shock off the cone
        d = np.empty_like(rU)
        op.Mult(rU, d)
        al = op.alpha()
        rec["alpha_at_t"] = {"elements_blended": int((al > 0).sum()), "fraction": float((al > 0).mean()),
                             "max": float(al.max())}
    op.close()
    return rec


def run_serving(torch, n_req, check_every=15):
    """Calibrate the server's capacity with a closed burst, then replay a
    Poisson stream at 80 % of it.  Requests are FP32-bulk solves.  A submitter
    thread builds each request's initial state when it arrives (meshes are
    cached per size) and a consumer thread collects results as they complete,
    so host memory stays bounded for long streams; every check_every-th result
    is checked against the FP64 plain path afterwards."""
    import numpy as np
    from prandtl_b200.batch import Server
    from prandtl_b200.ensemble import fixed_dt, serving_stream

    def prep(m):
        mesh = m.mesh()
        u0 = m.initial_state(mesh)
        return mesh, u0, fixed_dt(mesh, u0, 0.3 if m.kind == "ivortex" else CFL)

    burst = serving_stream(48, seed=7, rate=1.0)
    s = Server("fp32", steps_per_tick=4)
    t0 = time.perf_counter()
    tickets = []
    for m in burst:
        mesh, u0, dt = prep(m)
        tickets.append(s.submit(mesh, u0, dt=dt, nsteps=m.nsteps, **m.physics()))
    for t in tickets:
        s.wait(t, 600.0)
    cap_s = time.perf_counter() - t0
    s.close()
    capacity = len(burst) / cap_s
    rate = 0.8 * capacity
    reqs = serving_stream(n_req, seed=20261204, rate=rate)
    s = Server("fp32", steps_per_tick=4)
    tickets = [None] * len(reqs)
    submitted = threading.Semaphore(0)
    lat = [None] * len(reqs)
    kept = {}
    errors = []

    def submitter():
        start = time.perf_counter()
        for k, m in enumerate(reqs):
            mesh, u0, dt = prep(m)
            delay = m.arrival - (time.perf_counter() - start)
            if delay > 0:
                time.sleep(delay)
            tickets[k] = s.submit(mesh, u0, dt=dt, nsteps=m.nsteps, **m.physics())
            submitted.release()

    def consumer():
        for k in range(len(reqs)):
            submitted.acquire()
            try:
                u, sec = s.wait(tickets[k], 1800.0)
            except Exception as exc:   # a failed request is reported, not fatal
                errors.append((k, str(exc)))
                continue
            lat[k] = sec
            if k % check_every == 0:
                kept[k] = u

    th_s, th_c = threading.Thread(target=submitter), threading.Thread(target=consumer)
    t_start = time.perf_counter()
    th_s.start()
    th_c.start()
    th_s.join()
    th_c.join()
    t_end = time.perf_counter()
    st = s.stats()
    s.close()
    from prandtl_b200.operator import DGSEMOperator
    worst, checked = 0.0, 0
    for k, u in sorted(kept.items()):
        m = reqs[k]
        mesh, u0, dt = prep(m)
        op = DGSEMOperator(mesh, **m.physics())
        ref = u0.copy()
        op.Step(ref, dt, scheme="LSRK45", nsteps=m.nsteps)
        op.close()
        e = rel_errors(u, ref, mesh.num_fields)
        worst = max(worst, max(v[0] for v in e.values()))
        checked += 1
    ok = np.array([x for x in lat if x is not None]) * 1e3
    # per-request work, to relate latency to size
    work = np.array([(m.n ** (3 if m.kind == "tgv" else 2)) * (m.order + 1) ** (3 if m.kind == "tgv" else 2)
                     * (5 if m.kind == "tgv" else 4) * m.nsteps for m in reqs], dtype=np.float64)
    # slowdown: time to solution over the request's own share of the device at the
    # stream's busy throughput (its DOF-updates / busy rate); 1 = served as if alone
    busy_rate = st["dof_updates"] / max(st["busy_s"], 1e-9)
    slow = np.array([lat[k] / (work[k] / busy_rate) for k in range(len(reqs)) if lat[k] is not None])
    return {"requests": len(reqs), "completed": int(len(ok)), "failed": len(errors), "precision": "fp32-bulk",
            "arrivals": f"Poisson at {rate:.2f}/s = 0.8 x capacity {capacity:.2f}/s (closed burst of 48)",
            "p50_ms": float(np.percentile(ok, 50)), "p99_ms": float(np.percentile(ok, 99)),
            "mean_ms": float(ok.mean()), "max_ms": float(ok.max()),
            "stream_s": t_end - t_start,
            "throughput_dof_updates_per_s": st["dof_updates"] / (t_end - t_start),
            "busy_dof_updates_per_s": st["dof_updates"] / max(st["busy_s"], 1e-9),
            "batch_steps": st["steps"], "checked_vs_fp64_plain": checked,
            "max_rel_l2_vs_fp64_plain": worst,
            "work_dof_updates_p50_p99": [float(np.percentile(work, 50)), float(np.percentile(work, 99))],
            "slowdown_p50_p99": [float(np.percentile(slow, 50)), float(np.percentile(slow, 99))],
            "admission": "arrival order; later requests that fit may pass a waiting one, at most 64 times each",
            "mix": "50% 2D Euler isentropic vortex (16^2..128^2, N 3|4), 50% 3D NS TGV (8^3..24^3, N 2|3), "
                   "50..500 steps"}


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
    from prandtl_b200.ensemble import tgv_ensemble

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    K, W = args.steps, args.warmup
    if args.serve_only:
        rec = run_serving(torch, args.serve_requests, check_every=max(15, args.serve_requests // 50))
        print(json.dumps({"serving": rec}), flush=True)
        return
    if args.profile_case == "tgv32":
        run_tgv32(torch, K, extras=False)
        return
    members = tgv_ensemble(args.ensemble)
    items = build_items(members)
    dof = sum(u0.size for _, _, u0, _ in items)

    states, binfo = run_batch(torch, items, K, W, barrier, local)
    if args.profile_case == "batch":
        return
    device_s = max_over_ranks(dist, binfo["device_s"], "cuda")
    wall_s = max_over_ranks(dist, binfo["wall_s"], "cuda")
    value = dof * K * world / device_s

    line = None
    if rank == 0:
        # FP64 plain path on every k-th member, and the FP32-batched error against it
        sample = list(range(0, len(items), max(1, args.plain_every)))
        pstates, pinfo = run_plain(torch, [items[k] for k in sample], K, W, [states[k] for k in sample])
        plain_rate = pinfo["dof"] * K / pinfo["device_s"]
        errs = [rel_errors(states[k], p, 5) for k, p in zip(sample, pstates)]
        err = {f: {"rel_l2_max": max(e[f][0] for e in errs), "rel_l2_median": statistics.median(e[f][0] for e in errs),
                   "rel_linf_max": max(e[f][1] for e in errs)} for f in ("rho", "momentum", "energy")}
        # roofline of the dominant launch: the class with the largest tuned RHS time
        fp32_peak = gemm_tflops(torch, torch.float32) if not args.no_peaks else None
        fp64_peak = gemm_tflops(torch, torch.float64) if not args.no_peaks else None
        dom_order = max(binfo["classes"], key=lambda o: binfo["classes"][o]["rhs_ms_per_variant"][binfo["classes"][o]["variant"]])
        dc = binfo["classes"][dom_order]
        t_launch = dc["rhs_ms_per_variant"][dc["variant"]] / 1e3
        E_dom = sum(mesh.num_elements for m, mesh, _, _ in items if m.order == dom_order)
        fl = E_dom * flops_per_element(3, dom_order)
        # mean over the 5 LSRK stages: the first (A_1 = 0) does not read du
        by = E_dom * (rhs_bytes_per_element(3, dom_order, 4) - (dom_order + 1) ** 3 * 5 * 8 / 5)
        hbm_peak, hbm_src = load_hbm_peak()
        tfl = fl / t_launch / 1e12
        tr = measured_traffic().get(f"rhs_batch_N{dom_order}_fp32")
        traffic = tr["bytes_per_element"] * E_dom if tr else None
        roofline = {
            "bound": "compute (FP32 CUDA cores; the kernel is neither HBM- nor tensor-bound)",
            "kernel": f"rhs_batch_kernel<3, N={dom_order}, NS, float> (all N={dom_order} members, one stage)",
            "achieved": tfl, "peak": fp32_peak, "unit": "TFLOP/s",
            "frac": (tfl / fp32_peak) if fp32_peak else None,
            "peak_source": "measured live in this run: cuBLAS SGEMM 8192^3, TF32 off (torch.matmul float32)",
            "traffic": traffic,
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of this kernel on the N=5 members "
                               "of a 24-member ensemble, scaled by elements (ncu summary rhs_batch_kernel_N5_fp32_ncu under profiles/); "
                               "that launch was an LSRK first stage, which does not read du") if tr else None,
            "flops_per_launch": fl, "avg_launch_ms": t_launch * 1e3,
            "launch_timing": ("CUDA events on the batch stream around this class's RHS launches in the autotuner's "
                              "step for the chosen shape (inside the warm-up; mean over the step's 5 LSRK stages)"),
            "hbm": {"algorithmic_bytes_per_launch": by, "achieved_gbs": by / t_launch / 1e9,
                    "peak_gbs": hbm_peak, "frac": by / t_launch / 1e9 / hbm_peak, "peak_source": hbm_src},
            "classes": {str(o): c for o, c in binfo["classes"].items()},
        }
        # the same class's lifting launch: HBM-bound by design (u read, FP32 viscous rows written)
        t_lift = dc["lift_ms"] / 1e3
        nd_dom = (dom_order + 1) ** 3
        lby = E_dom * nd_dom * (5 * 8 + 3 * 4 * 4)
        ltr = measured_traffic().get(f"lift_batch_N{dom_order}_fp32")
        roofline["lift"] = {
            "kernel": f"lift_batch_kernel<3, N={dom_order}, float> (all N={dom_order} members, one stage)",
            "bound": "hbm", "algorithmic_bytes_per_launch": lby, "avg_launch_ms": t_lift * 1e3,
            "achieved_gbs": lby / t_lift / 1e9, "peak_gbs": hbm_peak, "frac": lby / t_lift / 1e9 / hbm_peak,
            "peak_source": hbm_src,
            "traffic": ltr["bytes_per_element"] * E_dom if ltr else None,
            "traffic_source": ("ncu dram bytes of this kernel on the N=5 members of a 24-member ensemble, scaled by "
                               "elements (ncu summary lift_batch_kernel_N5_fp32_ncu under profiles/)") if ltr else None}
        ivortex32 = run_ivortex32(torch) if not args.no_configs else None
        kh256 = run_kh256(torch) if not args.no_configs else None
        ramp = run_ramp(torch) if not args.no_configs else None
        tgv32 = None
        if not args.no_tgv32:
            tgv32 = run_tgv32(torch, 50)
            tf = tgv32["rhs_flops"] / (tgv32["rhs_ms"] / 1e3) / 1e12
            tgv32["rhs_fp64_tflops"] = tf
            tgv32["fp64_peak_tflops"] = fp64_peak
            tgv32["rhs_fp64_frac"] = (tf / fp64_peak) if fp64_peak else None
            tgv32["fp64_peak_source"] = "measured live: cuBLAS DGEMM 8192^3"
            t32 = measured_traffic().get("rhs_tgv32_fp64")
            tgv32["rhs_traffic_bytes"] = t32["bytes_per_launch"] if t32 else None
        serving = None
        if not args.no_serve:
            serving = run_serving(torch, args.serve_requests)
        cpu = None
        if not args.no_cpu_baseline:
            try:
                rate, info = cpu_rate(seconds=args.cpu_seconds)
                cpu = {"value": rate, "unit": "DOF-updates/s", "cores": info["cores"],
                       "kind": info["kind"], "sample": info["sample"], "single_core": info["single_core"]}
            except Exception as exc:
                cpu = {"value": None, "unit": "DOF-updates/s", "cores": os.cpu_count(), "kind": "port",
                       "sample": f"unavailable: {exc}"}
        u_bytes = dof * 8
        line = {
            "metric": "DOF-updates/s/GPU", "value": value, "unit": "DOF-updates/s",
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": 1e3 * device_s / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32-bulk/f64-state",
            "data": "synthetic (standard TGV initial conditions, seeded ensemble; no dataset)",
            "config": {"workload": WORKLOAD, "members": len(items), "dof": dof, "seed": 20261203,
                       "orders": "N ~ U{2,3,4,5}", "mesh": "n^3 periodic hexes, n ~ U{4..16}",
                       "mach": "U[0.05,0.3]", "re": "logU[100,3200]", "scheme": "LSRK45", "cfl": CFL,
                       "form": "batched FP32 bulk, FP64 RK state; persistent per-order launches in a CUDA graph",
                       "parallelism": f"replicas x{world}",
                       "l2": f"no flush: working set {binfo['device_bytes'] / 2**30:.1f} GiB >> 126 MiB L2"},
            "fp64_plain": {"value": plain_rate, "unit": "DOF-updates/s", "members": len(sample),
                           "sample": f"every {args.plain_every}th member, each alone through DGSEMOperator.Step",
                           "ratio_fp32_batched_over_fp64_plain": (value / world) / plain_rate},
            "error": {"fp32_batched_vs_fp64_plain_after_steps": W + K, "members": len(sample), **err},
            "budgets": budget_summary(pinfo["budgets"], W + K),
            "e2e": {"value": dof * (W + K) * world / wall_s, "unit": "DOF-updates/s",
                    "h2d_bytes_per_step": u_bytes / (W + K), "d2h_bytes_per_step": u_bytes / (W + K),
                    "window": "admission from pinned host memory + W+K steps (the autotuner inside the first warm-up steps) + every state read back; "
                              "the states cross once per solve, bytes shown per step",
                    "window_s": binfo["window_s"]},
            "gpu_launches": binfo["launches"],
            "roofline": roofline,
            "cpu_baseline": cpu,
            "tgv32": tgv32,
            "ivortex32": ivortex32,
            "kh256": kh256,
            "ramp": ramp,
            "serving": serving,
            "clocks": binfo["clocks"],
        }
    barrier()
    if line is not None:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
