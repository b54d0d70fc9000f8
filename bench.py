"""Benchmark: batched 3D eikonal travel-time tables on one B200.

Workload (the batched-tables configuration): 64 surface sources (seeded
uniform x, y; z = 0, which takes the reference's on-node nudge) solved on 4
grids of uneven size, all h = 50 m, nx x ny x nz = 96x96x64, 128x128x80,
160x160x96, 200x120x100, cell velocity v(z) = 3000 + 0.5 z (cell centre).
Every (grid, source) pair is one work item: 256 solves per step, one kernel
launch replayed from a CUDA graph.  A step = the whole batch: field
initialisation, the 8 initialisation sweeps and nsweep = 2 Gauss-Seidel
passes of 8 sweeps (the reference's default, no convergence test in 3D).

metric: node updates per second, counted as the reference evaluates them:
per source and grid, the masked initialisation sweeps plus nsweep x 8 x
(nz-1)(nx-1)(ny-1).  Inputs are synthetic and seeded.

--impl reference runs the CPU restatement of the reference's OpenMP
level-set solver (oracle/, FP64, 32-node chunks, a barrier per level) on
the host cores with the same metric, on a bounded sample of the workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GRIDS = [(96, 96, 64), (128, 128, 80), (160, 160, 96), (200, 120, 100)]  # nx, ny, nz
H = 50.0
NSRC = 64
NSWEEP = 2
EPS = 5.0
METRIC = "3D eikonal node-updates/s (64-src batch)"


def workload():
    rng = np.random.default_rng(4)
    srcxy = rng.uniform(0.0, 1.0, size=(NSRC, 2))
    grids = []
    for nx, ny, nz in GRIDS:
        zc = (np.arange(nz - 1) + 0.5) * H
        vel = np.broadcast_to(3000.0 + 0.5 * zc, (ny - 1, nx - 1, nz - 1)).copy()
        xs = srcxy[:, 0] * (nx - 1) * H
        ys = srcxy[:, 1] * (ny - 1) * H
        zs = np.zeros(NSRC)
        grids.append(dict(nx=nx, ny=ny, nz=nz, vel=vel, xs=xs, ys=ys, zs=zs))
    return grids


def snap1(n, h, v):
    """source.F90:150-168 for one coordinate -> 1-based cell index."""
    a = v / h + 1.0
    if abs(a - 1.0) < 2.220446049250313e-16:
        a += 1e-4
    if a >= n:
        a -= 1e-4
    return int(a)


def node_updates(g):
    """Node updates the reference evaluates for one grid's sources
    (solver3D.F90:493-565 boxes, init boxes clamped to the grid)."""
    nz, nx, ny = g["nz"], g["nx"], g["ny"]
    per_pass = 8 * (nz - 1) * (nx - 1) * (ny - 1)
    total = 0
    for k in range(NSRC):
        si = (snap1(nz, H, g["zs"][k]), snap1(nx, H, g["xs"][k]), snap1(ny, H, g["ys"][k]))
        init = 0
        for s in range(8):
            signs = (1 if s < 4 else -1, 1 if s % 2 == 0 else -1, 1 if (s // 2) % 2 == 0 else -1)
            cnt = 1
            for sgn, n, i in zip(signs, (nz, nx, ny), si):
                if sgn > 0:
                    lo, hi = max(2, i), n
                else:
                    lo, hi = 1, min(i + 1, n - 1)
                cnt *= max(0, hi - lo + 1)
            init += cnt
        total += init + NSWEEP * per_pass
    return total


def algorithmic_bytes(grids):
    """Algorithmic DRAM bytes of one solve, per kernel.  A sweep over one
    grid reads and writes every source's FP32 field once (8 B per node and
    source) and reads the grid's FP32 slowness once (4 B per cell, shared by
    the grid's sources).  The Gauss-Seidel kernel runs nsweep passes of 8
    sweeps over whole grids; the initialisation kernel's 8 sweeps touch only
    the source-limited boxes, counted node by node."""
    pass_b = 0
    init_b = 0
    for g in grids:
        ngrd = g["nz"] * g["nx"] * g["ny"]
        ncell = (g["nz"] - 1) * (g["nx"] - 1) * (g["ny"] - 1)
        pass_b += NSWEEP * 8 * (8 * NSRC * ngrd + 4 * ncell)
        init_b += 8 * (node_updates(g) - NSRC * NSWEEP * 8 * ncell) + 8 * 4 * ncell
    return init_b, pass_b


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons}


CPU_SAMPLE_SRC = 24     # sources of the 160x160x96 grid per CPU step (a few seconds of FP64 work)


def cpu_steps(args):
    """Warm-up solves and timed steps of the CPU baseline: the same in the
    reference arm and in the line's cpu_baseline, so the two agree."""
    return max(1, min(args.warmup, 3)), min(max(1, args.steps), 3)


def config_dict(grids, world):
    return {"workload": "batched tables: 64 surface sources x %d grids (%s), h=50 m, v(z)=3000+0.5z" % (
                len(grids), ", ".join("%dx%dx%d" % (g["nx"], g["ny"], g["nz"]) for g in grids)),
            "nsweep": NSWEEP, "eps": EPS, "work_items": NSRC * len(grids),
            "node_updates_per_step": sum(node_updates(g) for g in grids),
            "l2": "fields 1.73 GB > L2 (inputs larger than L2)",
            "parallelism": "replicas (one batch per GPU)" if world > 1 else "1 GPU"}


def cpu_reference(grids, steps, warmup, nthreads, sample_src=CPU_SAMPLE_SRC, check=None):
    """CPU restatement of the reference (oracle/), timed on a bounded sample:
    `sample_src` sources on the 160x160x96 grid per step.  check(k, tt), if
    given, receives each source's FP64 field outside the timed solves."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    g = next(g for g in grids if (g["nx"], g["ny"], g["nz"]) == (160, 160, 96))
    n = (g["nz"], g["nx"], g["ny"])
    slow = (1.0 / g["vel"]).ravel()
    upd = 0
    si_sa = []
    for k in range(sample_src):
        si, sa = O.source_snap(True, n, (0, 0, 0), (H, H, H), (g["zs"][k], g["xs"][k], g["ys"][k]))
        si_sa.append((si, sa))
        ni, npass = O.count_updates3d(n, si)
        upd += ni + NSWEEP * npass
    for w in range(warmup):
        O.solve3d(n, (H, H, H), slow, *si_sa[w % len(si_sa)], EPS, NSWEEP, level_set=True, nthreads=nthreads)
    dt = 0.0
    for _ in range(steps):
        for k, (si, sa) in enumerate(si_sa):
            t0 = time.perf_counter()
            tt, _ = O.solve3d(n, (H, H, H), slow, si, sa, EPS, NSWEEP, level_set=True, nthreads=nthreads)
            dt += time.perf_counter() - t0
            if check is not None:
                check(k, tt)
    return upd * steps / dt, dt, ("%d source(s) on the %dx%dx%d grid per step, %d step(s) after %d "
                                   "warm-up solve(s); node-updates/s of that sample" % (
                                       sample_src, g["nx"], g["ny"], g["nz"], steps, warmup))


def init_updates3d(n, si):
    """Node updates of the 8 masked initialisation sweeps for a source in
    cell si (solver3D.F90:493-565 boxes, flipped axes clamped to n-1)."""
    total = 0
    for s in range(8):
        signs = (1 if s < 4 else -1, 1 if s % 2 == 0 else -1, 1 if (s // 2) % 2 == 0 else -1)
        cnt = 1
        for sgn, nn, i in zip(signs, n, si):
            lo, hi = (max(2, i), nn) if sgn > 0 else (1, min(i + 1, nn - 1))
            cnt *= max(0, hi - lo + 1)
        total += cnt
    return total


def field_errors(got, ref):
    """Max / RMS absolute and relative travel-time error against the FP64
    field (relative to the reference time, nodes within 1 ms of the source
    excluded from the relative figures)."""
    got = np.asarray(got, np.float64)
    d = np.abs(got - ref)
    m = ref > 1e-3
    rel = d[m] / ref[m]
    return {"max_abs_s": float(d.max()), "rms_abs_s": float(np.sqrt(np.mean(d * d))),
            "max_rel": float(rel.max()), "rms_rel": float(np.sqrt(np.mean(rel * rel)))}


def bench_single_2d(fk, reps=20):
    """2D plain single source: nz x nx = 201 x 201, h = 10 m, FP64, cell
    velocity v(z) = 3000 + 0.5 z at the cell centre, source at a seeded
    uniform off-grid point (seed 1), eps = 5.  The reference's 2D
    convergence test never fires (solver2D.F90:935-945), so 'converged'
    means: the smallest nsweep whose field no longer changes with one more
    pass.  Error against the analytic linear-gradient time
    (analytic.F90:853-890, velocity measured from z = 0)."""
    nz = nx = 201
    h = 10.0
    zc = (np.arange(nz - 1) + 0.5) * h
    vel = np.ascontiguousarray(np.broadcast_to(3000.0 + 0.5 * zc, (nx - 1, nz - 1))).ravel()
    rng = np.random.default_rng(1)
    zs, xs = rng.uniform(0.05, 0.95) * (nz - 1) * h, rng.uniform(0.05, 0.95) * (nx - 1) * h
    s = fk.fteik2d()

    def solve(nsweep):
        s.initialize(nx, nz, h, h, nsweep=nsweep, eps=EPS)
        s.setCellVelocityNatural(vel)
        s.setSources(xs, zs)
        s.solveSourceLSM(1)
        return s.getTravelTimeField()

    prev, nsweep = solve(1), 1
    while nsweep < 10:
        cur = solve(nsweep + 1)
        if np.array_equal(cur, prev):
            break
        prev, nsweep = cur, nsweep + 1
    tt = solve(nsweep)
    t0 = time.perf_counter()
    for _ in range(reps):
        s.solveSourceLSM(1)
        tt = s.getTravelTimeField()
    dt = (time.perf_counter() - t0) / reps
    # all-sources solve (solver2D.F90:740-773): 256 seeded sources, one launch
    nmany = 256
    zsm, xsm = rng.uniform(0, (nz - 1) * h, nmany), rng.uniform(0, (nx - 1) * h, nmany)
    s.setSources(xsm, zsm)
    s.setReceivers(np.linspace(0, (nx - 1) * h, 16), np.zeros(16))
    s.solveLSM()
    t0 = time.perf_counter()
    for _ in range(3):
        s.solveLSM()
        s.getTravelTimes()
    dtm = (time.perf_counter() - t0) / 3
    upd_many = 0
    for zz, xx in zip(zsm, xsm):
        a, b = snap1(nz, h, zz), snap1(nx, h, xx)
        upd_many += (len(range(max(2, a), nz + 1)) * len(range(max(2, b), nx + 1))
                     + len(range(max(2, a), nz + 1)) * len(range(1, min(b + 1, nx - 1) + 1))
                     + len(range(1, min(a + 1, nz - 1) + 1)) * len(range(max(2, b), nx + 1))
                     + len(range(1, min(a + 1, nz - 1) + 1)) * len(range(1, min(b + 1, nx - 1) + 1))
                     + nsweep * 4 * (nz - 1) * (nx - 1))
    s.free()
    z = np.arange(nz) * h
    x = np.arange(nx) * h
    Z, X = np.meshgrid(z, x)                       # (nx, nz): z fastest when raveled
    g = 0.5
    r2 = (Z - zs) ** 2 + (X - xs) ** 2
    ana = np.arccosh(1.0 + 0.5 * g * g * r2 / ((3000.0 + g * Z) * (3000.0 + g * zs))) / g
    zsi, xsi = snap1(nz, h, zs), snap1(nx, h, xs)
    init = sum(len(range(*zr)) * len(range(*xr)) for zr, xr in (
        ((max(2, zsi), nz + 1), (max(2, xsi), nx + 1)), ((max(2, zsi), nz + 1), (1, min(xsi + 1, nx - 1) + 1)),
        ((1, min(zsi + 1, nz - 1) + 1), (max(2, xsi), nx + 1)),
        ((1, min(zsi + 1, nz - 1) + 1), (1, min(xsi + 1, nx - 1) + 1))))
    upd = init + nsweep * 4 * (nz - 1) * (nx - 1)
    return {"workload": "2D single source, 201 x 201 nodes, h = 10 m, v(z) = 3000 + 0.5 z, FP64",
            "source_zx_m": [zs, xs], "nsweep_converged": nsweep,
            "gpu_ms_per_solve_e2e": dt * 1e3, "node_updates_per_solve": upd,
            "node_updates_per_s_e2e": upd / dt,
            "error_vs_analytic": field_errors(tt, ana.ravel()),
            "all_sources": {"sources": nmany, "receivers": 16, "ms_e2e": dtm * 1e3,
                            "node_updates_per_s_e2e": upd_many / dtm,
                            "method": "solveLSM: one launch, one CTA per source, batched receiver gather"},
            "_field": tt, "_src": (zs, xs), "_vel": vel, "_n": (nz, nx), "_h": h, "_upd_many": upd_many}


def bench_single_3d(fk, torch, steps):
    """3D plain single source: 128^3 nodes, h = 25 m, four layers (3000 /
    4000 / 5000 / 6000 m/s, seeded interfaces, >= 5 cells each) times
    (1 + 0.05 GRF with a 10-cell correlation length, seed 2), source at a
    seeded interior off-grid point (seed 3), FP32 on the GPU, iterated to
    convergence (passes until no FP32 node changes, cap 30)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from models import interior_source, layered_grf_cells
    n, h = (128, 128, 128), 25.0
    vel = layered_grf_cells(*n, seed=2)
    src = interior_source(n, (h, h, h), 3)
    b = fk.Batch3D([(n[0], n[1], n[2], h, h, h)], eps=EPS, convTol=0.0, maxPass=30, precision=4)
    b.setVelocityModel(1, vel)
    b.setSources(1, [src[0]], [src[1]], [src[2]])
    b.solve()
    stream = torch.cuda.ExternalStream(fk.lib().fteik_b200_stream())
    for _ in range(3):
        b.solveAsync()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        b.solveAsync()
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    init_ms, pass_ms = b.kernelTimes()
    out = np.empty(n[0] * n[1] * n[2], np.float32)

    def e2e_once():
        """model and source up, solve, field down (the drop-in call sequence)"""
        b.setVelocityModel(1, vel)
        b.setSources(1, [src[0]], [src[1]], [src[2]])
        b.solve()
        b.fields32(1, out)

    e2e_once()                               # untimed: the download's staging buffer, first copies
    t0 = time.perf_counter()
    for _ in range(max(1, steps)):
        e2e_once()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / max(1, steps)
    res, npass = b.solveInfo(1, 1)
    b.finalize()
    si = (snap1(n[0], h, src[0]), snap1(n[1], h, src[1]), snap1(n[2], h, src[2]))
    upd = init_updates3d(n, si) + npass * 8 * (n[0] - 1) * (n[1] - 1) * (n[2] - 1)
    return {"workload": "3D single source, 128^3 nodes, h = 25 m, layered + 5 % GRF, FP32, "
                        "converged", "source_zxy_m": list(src), "passes_to_converge": npass,
            "gpu_ms": ms, "init_kernel_ms": init_ms, "pass_kernel_ms": pass_ms,
            "gpu_ms_e2e": e2e_ms, "node_updates": upd, "node_updates_per_s": upd / (ms * 1e-3),
            "_field": out, "_vel": vel, "_src": src, "_n": n, "_h": h}


def single_cpu_baselines(c1, c2, nthreads):
    """The oracle (FP64 restatement of the reference's solvers) on the two
    single-source workloads, timed on the host cores: its fields are also
    the FP64 references for the GPU fields' error."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    nz, nx = c1["_n"]
    h = c1["_h"]
    si, sa = O.source_snap(False, (nz, nx, 1), (0, 0, 0), (h, h, 1.0), (c1["_src"][0], c1["_src"][1], 0.0))
    t0 = time.perf_counter()
    tt2, _ = O.solve2d((nz, nx), (h, h), 1.0 / c1["_vel"], si[:2], sa[:2], EPS, c1["nsweep_converged"])
    dt2 = time.perf_counter() - t0
    c1["cpu_baseline"] = {"value": c1["node_updates_per_solve"] / dt2, "unit": "node-updates/s",
                          "ms_per_solve": dt2 * 1e3, "cores": 1, "kind": "port",
                          "sample": "the whole 2D solve"}
    c1["max_abs_diff_vs_fp64_oracle_s"] = float(np.max(np.abs(c1["_field"] - tt2)))
    c1["all_sources"]["cpu_baseline"] = {
        "value": c1["node_updates_per_solve"] / dt2, "unit": "node-updates/s", "cores": 1, "kind": "port",
        "sample": "one source's solve, the per-source rate applies to all 256"}
    n, h = c2["_n"], c2["_h"]
    si, sa = O.source_snap(True, n, (0, 0, 0), (h, h, h), c2["_src"])
    t0 = time.perf_counter()
    tt3, np64 = O.solve3d(n, (h, h, h), (1.0 / c2["_vel"]).ravel(), si, sa, EPS, 1, conv_tol=0.0,
                          max_pass=30, level_set=True, nthreads=nthreads)
    dt3 = time.perf_counter() - t0
    upd64 = init_updates3d(n, si) + np64 * 8 * (n[0] - 1) * (n[1] - 1) * (n[2] - 1)
    c2["cpu_baseline"] = {"value": upd64 / dt3, "unit": "node-updates/s", "ms_per_solve": dt3 * 1e3,
                          "passes_to_converge": np64, "cores": nthreads, "kind": "port",
                          "sample": "the whole FP64 solve to convergence (max |dt| = 0)"}
    c2["error_vs_fp64_oracle"] = field_errors(c2["_field"], tt3)


def layered_grf_batch_error(fk, grids, nsrc=8):
    """The batch's FP32 fields on the other reading of the batch's velocity
    recipe -- four layers (3000 / 4000 / 5000 / 6000 m/s, seeded interfaces)
    times (1 + 0.05 GRF, 10-cell correlation length, seed 2) -- on the
    160x160x96 grid, for the first `nsrc` of the batch's surface sources,
    against the FP64 oracle's fields of the same solves."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    from models import layered_grf_cells
    g = next(g for g in grids if (g["nx"], g["ny"], g["nz"]) == (160, 160, 96))
    n = (g["nz"], g["nx"], g["ny"])
    vel = layered_grf_cells(*n, seed=2)
    b = fk.Batch3D([(n[0], n[1], n[2], H, H, H)], nsweep=NSWEEP, eps=EPS, precision=4)
    b.setVelocityModel(1, vel)
    b.setSources(1, g["zs"][:nsrc], g["xs"][:nsrc], g["ys"][:nsrc])
    b.solve()
    f32 = b.fields32(1).reshape(nsrc, -1)
    b.finalize()
    slow = (1.0 / vel).ravel()
    errs = []
    for k in range(nsrc):
        si, sa = O.source_snap(True, n, (0, 0, 0), (H, H, H), (g["zs"][k], g["xs"][k], g["ys"][k]))
        tt, _ = O.solve3d(n, (H, H, H), slow, si, sa, EPS, NSWEEP, level_set=True, nthreads=os.cpu_count() or 1)
        errs.append(field_errors(f32[k], tt))
    out = {key: (max if key.startswith("max") else lambda v: float(np.sqrt(np.mean(np.square(v)))))(
        [e[key] for e in errs]) for key in errs[0]}
    out["sample"] = ("%d surface sources of the batch on the 160x160x96 grid, velocity 4 layers x "
                     "(1 + 0.05 GRF), FP32 batch fields against FP64 oracle solves (relative figures "
                     "over nodes more than 1 ms from the source)" % nsrc)
    return out


def max_over_ranks(x, dist):
    """The slowest rank's value of a per-rank time (every rank gets it); x
    itself without a process group.  NCCL reduces on the GPU, gloo on the
    host."""
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, rank, world):
    grids = workload()
    nth = os.cpu_count() or 1
    if rank != 0:
        return
    warmup, steps = cpu_steps(args)        # each timed step: 24 FP64 solves, a few seconds
    value, dt, sample = cpu_reference(grids, steps=steps, warmup=warmup, nthreads=nth)
    cfg = config_dict(grids, 1)
    cfg["cpu_sample"] = sample
    line = {"metric": METRIC, "value": value, "unit": "node-updates/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": steps, "warmup": warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": "node-updates/s", "cores": nth, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "node-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


LOC_GRID = 3        # 1-based: the 160x160x96 grid, 64 station tables
LOC_NEV = 10000
LOC_EXACT_SAMPLE = 512
LOC_L1_SAMPLE = 128
SUR_WIDTH, SUR_DEPTH = 256, 5          # surrogate: 6 -> 5 x 256 SiLU -> tau
# 65,536 rows x 375 steps (lr 4e-3, 24.6e6 sample evaluations) keeps the
# pruning agreement at 100 % (as 16,384 x 750 and 4,096 x 3,000 at lr
# 2e-3 do) with products large enough for the tensor cores' throughput
SUR_SAMPLES, SUR_STEPS, SUR_BATCH, SUR_LR = 2_000_000, 375, 65536, 4e-3
SUR_BLOCK = (4, 4, 4)                  # fine nodes per coarse block (z, x, y)
SUR_WARMUP_STEPS = 22                  # more than 21: the warm-up takes the captured-step path


def locate_workload(b, g, nev, igrid=LOC_GRID):
    """Grid-search workload on one grid's 64 tables: hypocentres uniform in
    the volume (seed 5), origin times U[0, 60] s; exact times = trilinear
    interpolation of the tables at the hypocentre (receiver.F90:246-285 on
    the GPU); picks = exact + N(0, 0.02 s), 5 % of picks replaced by
    exact + U[-1, 1] s (seed 6); all weights 1."""
    rng = np.random.default_rng(5)
    z = rng.uniform(0, (g["nz"] - 1) * H, nev)
    x = rng.uniform(0, (g["nx"] - 1) * H, nev)
    y = rng.uniform(0, (g["ny"] - 1) * H, nev)
    t0 = rng.uniform(0, 60, nev)
    b.setReceivers(igrid, z, x, y)
    exact = b.travelTimes(igrid).T + t0[:, None]
    rng2 = np.random.default_rng(6)
    picks = exact + rng2.normal(0, 0.02, exact.shape)
    out = rng2.random(exact.shape) < 0.05
    picks[out] = exact[out] + rng2.uniform(-1, 1, int(out.sum()))
    return picks


def _mlp_products(fk):
    from ctypes import byref, c_int
    v = c_int()
    fk.lib().fteik_b200_mlp_getTensorProducts(byref(v))
    return v.value


def bench_locate(fk, b, grids, stream, steps, nev=LOC_NEV, igrid=LOC_GRID, sur_steps=SUR_STEPS,
                 sur_batch=SUR_BATCH, sur_lr=SUR_LR):
    import torch
    g = grids[LOC_GRID - 1]
    ngrd = g["nz"] * g["nx"] * g["ny"]
    picks = locate_workload(b, g, nev, igrid)
    loc = fk.Locator(nev, NSRC, ngrd)
    b.exportToLocator(igrid, 1)
    o2t = np.arange(1, NSRC + 1)
    w = np.ones(NSRC)
    for e in range(nev):
        loc.setObservation(e + 1, o2t, picks[e], w)
    ev = np.arange(1, nev + 1, dtype=np.int32)

    def timed(evs, k):
        loc.locateEvents(evs)          # warm-up: table packing, uploads
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            res = loc.locateEvents(evs)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / k, res

    loc.setMethod(1)
    tc_ms, (tc_idx, _, _) = timed(ev, max(1, steps))
    nprod = loc.setRankingProducts(3)        # the three-product ranking once, for its hypocentres
    _, (tc3_idx, _, _) = timed(ev, 1)
    loc.setRankingProducts(nprod)
    agree_tc3 = float(np.mean(tc_idx == tc3_idx))

    # learned pruning: surrogate trained on these tables, block centres
    # ranked on the tensor cores, 8 blocks x 64 = 512 fine cells re-scored
    # exactly
    loc.setGeometry(g["nz"], g["nx"], g["ny"], H, H, H, g["zs"], g["xs"], g["ys"])
    net = fk.MLP(SUR_WIDTH, SUR_DEPTH, seed=7)
    mlp_products = _mlp_products(fk)
    # untimed warm-up training call (the network's buffers, the kernels'
    # first loads, the captured-step path), then the initial weights back
    # (which also clears the Adam state): the timed run starts from the
    # same state a fresh network would
    w0 = net.weights()
    loc.trainSurrogate(nsamples=SUR_SAMPLES, steps=SUR_WARMUP_STEPS, batch=sur_batch, lr=sur_lr, vref=3000.0,
                       seed=7)
    net.setWeights(w0)
    torch.cuda.synchronize()
    t_tr = time.perf_counter()
    sur_loss = loc.trainSurrogate(nsamples=SUR_SAMPLES, steps=sur_steps, batch=sur_batch, lr=sur_lr,
                                  vref=3000.0, seed=7)
    t_tr = time.perf_counter() - t_tr
    t_bd0 = time.perf_counter()
    loc.buildSurrogate(SUR_BLOCK)          # first build: allocations and first kernel loads included
    t_bd0 = time.perf_counter() - t_bd0
    t_bd = time.perf_counter()
    loc.buildSurrogate(SUR_BLOCK)          # rebuilt in place (the network's output tables)
    t_bd = time.perf_counter() - t_bd
    loc.setPruning(4, 8)
    loc.setMethod(2)
    pr_ms, (pr_idx, _, _) = timed(ev, max(1, steps))
    nfb, ncoarse, nblk = loc.pruneInfo()
    loc.stageTimes(True)
    loc.locateEvents(ev)
    stage = loc.stageTimes()
    loc.stageTimes(False)
    flops_row = 2 * (6 * SUR_WIDTH + (SUR_DEPTH - 1) * SUR_WIDTH * SUR_WIDTH + SUR_WIDTH)
    loc.setMethod(0)
    sample = ev[:LOC_EXACT_SAMPLE]
    ex_ms, (ex_idx, _, _) = timed(sample, 1)
    loc.setNorm(1)
    l1_sample = ev[:LOC_L1_SAMPLE]
    l1_ms, _ = timed(l1_sample, 1)
    loc.setNorm(2)
    agree = float(np.mean(tc_idx[:LOC_EXACT_SAMPLE] == ex_idx))
    loc.finalize()
    flops = 2.0 * NSRC * ngrd * nev
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_s, src = 1590.0, 1400.0, "fallback"
    if os.path.exists(peaks_path):
        pk = json.load(open(peaks_path))
        peak, peak_s, src = pk["bf16_tflops"], pk["bf16_tflops_sustained"], "measured"
    ach = flops / (tc_ms * 1e-3) / 1e12
    return {"workload": "grid search: %d events x %d stations on the %dx%dx%d tables, L2 with "
                        "origin-time removal" % (nev, NSRC, g["nx"], g["ny"], g["nz"]),
            "metric": "events located/s",
            "tensor_core": {"events_per_s": nev / (tc_ms * 1e-3), "ms": tc_ms,
                            "method": "BF16 tcgen05 ranking (%d products: tables hi+lo, events %s), FP64 "
                                      "re-score of 8 candidates" % (nprod, "hi+lo" if nprod == 3 else "hi"),
                            "hypocentre_agreement_vs_three_products": agree_tc3,
                            "roofline": {"bound": "tensor", "achieved": ach, "peak": peak,
                                         "unit": "TFLOP/s", "frac": ach / peak,
                                         "frac_of_sustained": ach / peak_s, "peak_source": src,
                                         "algorithmic_flops": flops,
                                         "note": "2*stations*gridpoints per event, one contracted "
                                                 "term; the %d hi/lo products are not counted" % nprod}},
            "surrogate_pruned": {
                "events_per_s": nev / (pr_ms * 1e-3), "ms": pr_ms,
                "speedup_vs_tensor_core": tc_ms / pr_ms,
                "hypocentre_agreement_vs_tensor_core": float(np.mean(pr_idx == tc_idx)),
                "fallback_events": nfb, "coarse_nodes": ncoarse,
                "fine_blocks_examined_per_event": nblk / max(1, nev - nfb),
                "stage_ms": {"coarse_ranking": stage[0], "pruned_rescore": stage[1],
                             "results_to_host": stage[2]},
                "network": "6 -> %d x %d SiLU -> tau; hidden-layer GEMMs on the tensor cores (tcgen05, %s), "
                           "first / last layer, SiLU, Adam on the CUDA cores in FP32" % (
                               SUR_DEPTH, SUR_WIDTH, {0: "off: FP32 CUDA cores", 1: "BF16 operands, FP32 accumulators",
                                                      3: "split-BF16 operands, FP32 accumulators"}[mlp_products]),
                "training": {"samples": SUR_SAMPLES, "steps": sur_steps, "batch": sur_batch, "lr": sur_lr,
                             "untimed_warmup_steps": SUR_WARMUP_STEPS, "seconds": t_tr, "final_mse_tau": sur_loss,
                             "tflops": 3.0 * flops_row * sur_steps * sur_batch / t_tr / 1e12},
                "coarse_build": {"block_zxy": list(SUR_BLOCK), "seconds": t_bd, "seconds_first_build": t_bd0,
                                 "rows": ncoarse * NSRC, "method": "fused forward pass" if mlp_products == 1
                                 else "layer by layer",
                                 "tflops": flops_row * ncoarse * NSRC / t_bd / 1e12}},
            "l1_exhaustive": {"events_per_s": len(l1_sample) / (l1_ms * 1e-3), "ms": l1_ms,
                              "sample_events": len(l1_sample),
                              "method": "median origin time, 64-key bitonic sort per grid point, FP32 ranking, "
                                        "FP64 optimum"},
            "exact_fp32": {"events_per_s": len(sample) / (ex_ms * 1e-3), "ms": ex_ms,
                           "sample_events": len(sample)},
            "hypocentre_agreement_tc_vs_exact": agree}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-locate", action="store_true")
    ap.add_argument("--no-single", action="store_true",
                    help="skip the single-source 2D (201x201) and 3D (128^3, converged) sections")
    ap.add_argument("--locate-only", action="store_true",
                    help="solve only the 160x160x96 grid once and run the grid-search section")
    ap.add_argument("--locate-events", type=int, default=LOC_NEV)
    ap.add_argument("--surrogate-steps", type=int, default=SUR_STEPS)
    ap.add_argument("--surrogate-batch", type=int, default=SUR_BATCH)
    ap.add_argument("--surrogate-lr", type=float, default=SUR_LR)
    ap.add_argument("--slab-config", default=None,
                    help="staged,pairs,progress,blocks_per_sm for the 3D sweep kernels "
                         "(fteik_b200_setSlabConfig; default: chosen by the library's tuner)")
    ap.add_argument("--grids", default="1,2,3,4",
                    help="subset of the 4 batched grids (1-based, comma separated) for profiling")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    import fteik_b200 as fk
    if not os.path.exists(fk.LIB_PATH):
        fk.build()

    if args.slab_config:
        fk.set_slab_config(*[int(v) for v in args.slab_config.split(",")])
    grids = workload()
    if args.locate_only:
        g = grids[LOC_GRID - 1]
        b = fk.Batch3D([(g["nz"], g["nx"], g["ny"], H, H, H)], nsweep=NSWEEP, eps=EPS, precision=4)
        b.setVelocityModel(1, g["vel"])
        b.setSources(1, g["zs"], g["xs"], g["ys"])
        b.solve()
        stream = torch.cuda.ExternalStream(fk.lib().fteik_b200_stream())
        res = bench_locate(fk, b, grids, stream, args.steps, nev=args.locate_events, igrid=1,
                           sur_steps=args.surrogate_steps,
                           sur_batch=args.surrogate_batch, sur_lr=args.surrogate_lr)
        print(json.dumps({"locate": res}), flush=True)
        b.finalize()
        return
    sel = [int(v) for v in args.grids.split(",")]
    if sel != [1, 2, 3, 4]:
        args.no_locate = True   # the grid-search section needs the 160x160x96 grid at index 3
    grids = [grids[i - 1] for i in sel]
    upd_total = sum(node_updates(g) for g in grids)
    init_bytes, pass_bytes = algorithmic_bytes(grids)

    b = fk.Batch3D([(g["nz"], g["nx"], g["ny"], H, H, H) for g in grids], nsweep=NSWEEP, eps=EPS,
                   precision=4)
    for i, g in enumerate(grids, start=1):
        b.setVelocityModel(i, g["vel"])
        b.setSources(i, g["zs"], g["xs"], g["ys"])
    t_tune = time.perf_counter()
    b.solve()  # chooses the launch configuration (timed candidates), captures the graph
    t_tune = time.perf_counter() - t_tune
    slab_cfg = b.slabConfig()
    slab_cfg["first_solve_s"] = t_tune
    stream = torch.cuda.ExternalStream(fk.lib().fteik_b200_stream())

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-resident timing: K graph replays on the library stream ----
    for _ in range(args.warmup):
        b.solveAsync()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            rc = b.solveAsync()
            assert rc == 0, rc
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    # per-kernel device time, from the events inside the solve graph
    ki, kp = [], []
    for _ in range(args.steps):
        a, c = b.kernelTimes()
        ki.append(a)
        kp.append(c)
    init_ms, pass_ms = float(np.mean(ki)), float(np.mean(kp))
    ms = max_over_ranks(ms, dist)
    value = upd_total * world / (ms * 1e-3)

    # ---- end to end through the C ABI with host buffers ----
    e2e = None
    if not args.no_e2e:
        outs = []
        for g in grids:
            n = NSRC * g["nz"] * g["nx"] * g["ny"]
            outs.append(torch.empty(n, dtype=torch.float32, pin_memory=True).numpy())
        vels = [torch.from_numpy(np.ascontiguousarray(g["vel"].ravel())).pin_memory().numpy() for g in grids]
        h2d = sum(v.nbytes for v in vels) + sum(3 * 8 * NSRC for _ in grids)
        d2h = sum(o.nbytes for o in outs)

        def e2e_step():
            """Models and sources up, solve, tables down: the download is
            queued on the library's copy stream and overlaps the next step's
            uploads and solve; every step's copies are inside the timed
            region (the last one waited for before the clock stops)."""
            for i, g in enumerate(grids, start=1):
                b.setVelocityModel(i, vels[i - 1])
                b.setSources(i, g["zs"], g["xs"], g["ys"])
            b.solve()
            for i in range(1, len(grids) + 1):
                b.fields32Async(i, outs[i - 1])

        e2e_step()
        b.waitDownloads()
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        ke = max(1, args.steps)
        for _ in range(ke):
            e2e_step()
        b.waitDownloads()
        torch.cuda.synchronize()
        barrier()
        te = (time.perf_counter() - t0) / ke
        te = max_over_ranks(te, dist)
        e2e = {"value": upd_total * world / te, "unit": "node-updates/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": te * 1e3}

    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6651.0, "fallback"
    if os.path.exists(peaks_path):
        peak = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    achieved = pass_bytes / (pass_ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "slab_pass_traffic.json")
    if os.path.exists(tp) and sel == [1, 2, 3, 4]:   # captured on the 4-grid batch
        traffic = json.load(open(tp)).get("dram_bytes_per_launch")
    roofline = {"bound": "hbm", "kernel": "fk3rw::slab_kernel<float, passes, 2 sources per thread>",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_src, "traffic": traffic,
                "algorithmic_bytes_per_launch": pass_bytes, "launch_ms": pass_ms,
                "init_kernel": {"launch_ms": init_ms, "algorithmic_bytes_per_launch": init_bytes,
                                "achieved": init_bytes / (init_ms * 1e-3) / 1e9}}

    locate = None
    if not args.no_locate:
        locate = bench_locate(fk, b, grids, stream, args.steps, nev=args.locate_events,
                              sur_steps=args.surrogate_steps,
                           sur_batch=args.surrogate_batch, sur_lr=args.surrogate_lr)

    cpu = None
    batch_err = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and 3 in sel:
        # the baseline's FP64 fields (160x160x96 grid) check the batch's FP32 fields of the same sources
        f32 = b.fields32(sel.index(3) + 1).reshape(NSRC, -1)
        acc = {"max_abs": 0.0, "sq_abs": 0.0, "n": 0, "max_rel": 0.0, "sq_rel": 0.0, "nrel": 0}

        seen = set()

        def check(k, tt):
            if k in seen:          # every timed step solves the same sample
                return
            seen.add(k)
            d = np.abs(f32[k].astype(np.float64) - tt)
            m = tt > 1e-3
            rel = d[m] / tt[m]
            acc["max_abs"] = max(acc["max_abs"], float(d.max()))
            acc["sq_abs"] += float(np.dot(d, d))
            acc["n"] += d.size
            acc["max_rel"] = max(acc["max_rel"], float(rel.max()))
            acc["sq_rel"] += float(np.dot(rel, rel))
            acc["nrel"] += rel.size

        cw, cs = cpu_steps(args)
        v, dt, sample = cpu_reference(grids, steps=cs, warmup=cw, nthreads=os.cpu_count() or 1, check=check)
        cpu = {"value": v, "unit": "node-updates/s", "cores": os.cpu_count(), "kind": "port",
               "sample": sample}
        batch_err = {"max_abs_s": acc["max_abs"], "rms_abs_s": (acc["sq_abs"] / acc["n"]) ** 0.5,
                     "max_rel": acc["max_rel"], "rms_rel": (acc["sq_rel"] / acc["nrel"]) ** 0.5,
                     "sample": "the FP32 batch fields of the baseline's %s, against its FP64 fields "
                               "(relative figures over nodes more than 1 ms from the source)" % sample}

    b.finalize()            # the library holds one batch; the sections below make their own
    grf_err = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and 3 in sel:
        grf_err = layered_grf_batch_error(fk, grids)
    single = None
    if rank == 0 and world == 1 and not args.no_single:
        c1 = bench_single_2d(fk)
        c2 = bench_single_3d(fk, torch, args.steps)
        if not args.no_cpu_baseline:
            single_cpu_baselines(c1, c2, os.cpu_count() or 1)
        single = {"plain_2d": {k: v for k, v in c1.items() if not k.startswith("_")},
                  "plain_3d_128": {k: v for k, v in c2.items() if not k.startswith("_")}}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "node-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": dict(config_dict(grids, world), slab_config=slab_cfg),
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "error_vs_fp64_oracle": batch_err,
                "error_vs_fp64_oracle_layered_grf": grf_err,
                "gpu_launches": 5 * args.steps, "clocks": clk.summary(), "locate": locate,
                "single_source": single}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
