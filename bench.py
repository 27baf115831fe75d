#!/usr/bin/env python
"""Throughput of the 3D-MT forward + adjoint solve on B200 GPUs.

Workload (default "combined"): the 200x200x100 model (12 air + 88 earth
layers, seeded Gaussian random field of log10 resistivity), 16 frequencies
log-spaced 1e-4..1e2 Hz, 2 polarisations, forward solves (plane-wave boundary
data) and adjoint (transposed) solves (synthetic receiver sources on a 20x20
array) -- 64 right-hand sides.  One step solves 8 of them in one batched call
of the C ABI: frequencies f and f+8 (f = step mod 8) x 2 polarisations x
{forward, adjoint}, each to a relative residual of 1e-7 of the FP64 system;
8 steps cover all 64.  The metric is solves/s over all ranks.  The solver:
curl-curl + grad-div, diagonal preconditioner, FP32 BiCGStab cycles of 300
iterations (restarted only at cycle starts) under FP64 residual refinement.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload combined|precision|batch|small]
                  [--no-cpu] [--no-fp64] [--no-e2e]

value: device time (CUDA events on the solver stream) of the K timed steps,
inputs resident in HBM.  e2e: the same solves through mt3d_fwdsolve_batch
with pinned host buffers (host->device copies of the inputs and the
device->host copy of the fields inside the timed region), over min(K, 2)
steps (the first ones, whose own device-time rate it reports beside it, as
device_value_same_steps: the steps differ in frequency and so in cost).  fp64: the same right-hand sides as the first timed step, solved one
at a time by the plain FP64 path.  With N > 1 (torchrun) every rank solves its
own copy of the workload (replicas; the right-hand sides are independent),
timed between barriers, max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "modem-gpu_b200"))
sys.path.insert(0, ROOT)

from mt3d import bc as mbc  # noqa: E402
from mt3d import models  # noqa: E402

METRIC = "fwd+adjoint solves/s, mixed-precision batched vs plain FP64 GPU at 1e-7 residual"
TOL = 1e-7
# refinement cycle: FP32 BiCGStab iterations between FP64 residual updates;
# cycles of 40-120 stall the low-frequency forward solves of the 200x200x100
# model, 300 converges all 64 right-hand sides
CYCLE = 300
# BiCGStab restarts only at cycle starts (each cycle begins from the true
# residual); cuBiCG's 120-iteration restarts cost 14 % more iterations here
RESTART = 0
MAX_CYCLES = 30
# the FP32 iteration runs in preconditioned variables with the diagonal
# preconditioner fused into the stencil kernels (mt3d_set_fused)
FUSED = True
# polynomial preconditioner c D^-1 (2I - c A D^-1) of the fused FP32 cycles
# (mt3d_set_poly): c = 0.9 halves the iterations of this workload for two
# stencil passes per preconditioned product; c = 1 sends right-hand sides
# to the FP64 fall-back
POLY = 0.9 if FUSED else 0.0
# FP64 tolerance of the tight reference solve of the parity comparison
TIGHT_TOL = 1e-10


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------------
# workloads
# --------------------------------------------------------------------------
def receiver_sources(model: models.Model, nrec: int, seed: int) -> np.ndarray:
    """Synthetic adjoint sources: complex weights on the surface x- and
    y-edges next to an nrec x nrec array of receivers on the core cells (the
    sparse structure of LmultT sources, f90/3D_MT/DataSens.f90:130-225),
    V_E-weighted; one vector per polarisation."""
    g = model.grid
    rng = np.random.default_rng(seed)
    nx, ny, nz, na = g.nx, g.ny, g.nz, g.nzAir
    nX = nx * (ny + 1) * (nz + 1)
    ix = np.linspace(nx * 0.3, nx * 0.7, nrec).astype(int)
    iy = np.linspace(ny * 0.3, ny * 0.7, nrec).astype(int)
    k = na  # surface node plane (0-based)
    out = np.zeros((2, g.n_edges), np.complex128)
    dX = np.concatenate([[g.dx[0]], g.dx[:-1] + g.dx[1:], [g.dx[-1]]]) / 2
    dY = np.concatenate([[g.dy[0]], g.dy[:-1] + g.dy[1:], [g.dy[-1]]]) / 2
    dZ = np.concatenate([[g.dz[0]], g.dz[:-1] + g.dz[1:], [g.dz[-1]]]) / 2
    for p in range(2):
        for i in ix:
            for j in iy:
                w = rng.standard_normal(2) + 1j * rng.standard_normal(2)
                ex = i + nx * (j + (ny + 1) * k)
                ey = nX + i + (nx + 1) * (j + ny * k)
                out[p, ex] += w[0] * g.dx[i] * dY[j] * dZ[k]
                out[p, ey] += w[1] * g.dy[j] * dX[i] * dZ[k]
    return out


def workload(name: str):
    """[(model, omegas[nf*2], bc[nf*2], src[nf*2])] (rows: frequency major,
    polarisation minor) and a description."""
    if name == "combined":
        m, f = models.config_combined()
        probs = [(m, f)]
        desc = "200x200x100 (12 air + 88 earth) random field, 16 freq 1e-4..1e2 Hz, 2 pol, fwd+adj"
    elif name == "precision":
        m, f = models.config_precision()
        probs = [(m, f)]
        desc = "100x100x60 (10 air + 50 earth) random field, 1 Hz, 2 pol, fwd+adj"
    elif name == "batch":
        probs = models.config_batch()
        desc = "40x40x40 + 64x64x48 + 96x96x56 random fields, 8 freq 1e-3..1e2 Hz, 2 pol, fwd+adj"
    elif name == "small":
        m, f = models.config_small_forward()
        probs = [(m, f)]
        desc = "24x24x24 halfspace + 1 ohm-m block, 0.1 Hz, 2 pol, fwd+adj"
    else:
        raise SystemExit(f"unknown workload {name}")
    out = []
    for k, (m, f) in enumerate(probs):
        om = 2 * np.pi * np.asarray(f, np.float64)
        bcs, srcs, oms = [], [], []
        rs = receiver_sources(m, 20 if name == "combined" else 8, seed=100 + k)
        for w in om:
            for mode in (1, 2):
                bcs.append(mbc.boundary_1d(m, w, mode))
                srcs.append(rs[mode - 1])
                oms.append(w)
        out.append((m, np.asarray(oms), np.stack(bcs), np.stack(srcs)))
    return out, desc


def step_rows(name: str, nf: int, step: int) -> list:
    """Frequency indices solved by a step (all 2 x {fwd, adj} of each)."""
    if name == "combined":
        h = nf // 2
        return [step % h, step % h + h]
    return list(range(nf))


def step_batch(oms, bcs, srcs, fidx):
    """Right-hand sides of the frequencies fidx: forward rows (boundary data,
    no source) then adjoint rows (source, no boundary data)."""
    rows = [2 * f + p for f in fidx for p in (0, 1)]
    n = len(rows)
    om = np.concatenate([oms[rows]] * 2)
    bc = np.concatenate([bcs[rows], np.zeros_like(bcs[rows])])
    src = np.concatenate([np.zeros_like(srcs[rows]), srcs[rows]])
    tr = np.concatenate([np.zeros(n, np.int32), np.ones(n, np.int32)])
    return om, bc, src, tr


# --------------------------------------------------------------------------
# clocks sampled during the timed region
# --------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev: int):
        self.dev = dev
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() in ("active", "1"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        load = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------
# CPU baseline: the oracle (a C restatement of ModEM's CPU solver: QMR with
# the D-ILU preconditioner and divergence correction every 40 iterations)
# --------------------------------------------------------------------------
CPU_SAMPLE_ITERS = 10
# QMR + D-ILU iterations (divergence correction every 40) per solve to 1e-7,
# measured with the oracle on the workloads' own right-hand sides
# (oracle/cpu_iterations.py writes the 200x200x100 counts); the 100x100x60
# counts are the oracle's two forward polarisations at 1 Hz (3450 and 3059)
CPU_ITERS_PRECISION = 3250


def cpu_iterations(name: str):
    """(mean QMR + D-ILU iterations per solve, where the count comes from)."""
    if name == "combined":
        p = os.path.join(ROOT, "oracle", "cpu_iterations_200x200x100.json")
        if os.path.exists(p):
            d = json.load(open(p))
            per = ", ".join(f"{r['kind']} {r['freq_hz']:.3g} Hz: {r['iterations']}" for r in d["solves"])
            return float(d["mean_iterations"]), f"oracle runs to 1e-7 on this workload's right-hand sides ({per})"
        return float(CPU_ITERS_PRECISION), "the 100x100x60 workload's forward solves (this grid's counts unmeasured)"
    return float(CPU_ITERS_PRECISION), "the 100x100x60 workload's forward solves at 1 Hz (3450, 3059)"


def _models(name: str):
    """[(model, frequencies)] of a workload, without its right-hand sides."""
    if name == "combined":
        return [models.config_combined()]
    if name == "precision":
        return [models.config_precision()]
    if name == "batch":
        return models.config_batch()
    return [models.config_small_forward()]


_CPU_ORACLE = {}


def _cpu_init(name):
    """Pool initializer: the oracle's operator and D-ILU factors for the
    workload's first frequency, set up once per process (not timed)."""
    from oracle.oracle import Oracle, QMR, PC_DILU
    m, f = _models(name)[0]
    omega = 2 * np.pi * float(f[0])
    o = Oracle(m.grid)
    o.update_cond(m.m_earth, m.air_cond)
    o.update_freq(omega)
    o.set_control(solver=QMR, precond=PC_DILU, IterPerDivCor=CPU_SAMPLE_ITERS, MaxDivCor=1)
    _CPU_ORACLE.update(o=o, m=m, omega=omega)


def _cpu_worker(mode):
    """One bounded sample: CPU_SAMPLE_ITERS QMR + D-ILU iterations and one
    divergence correction of the forward solve of polarisation `mode`."""
    o, m, omega = _CPU_ORACLE["o"], _CPU_ORACLE["m"], _CPU_ORACLE["omega"]
    bc = mbc.boundary_1d(m, omega, mode)
    t0 = time.perf_counter()
    o.fwdsolve(bc=bc)
    d = o.diagnostics()
    return (time.perf_counter() - t0), max(1, d["nIterTotal"])


def cpu_baseline(name: str, procs: int, steps: int = 1, warmup: int = 0):
    """CPU solves/s of the reference solver on this workload, projected: the
    time per iteration is measured on the workload grid from bounded samples
    (each step: CPU_SAMPLE_ITERS Krylov iterations + one divergence correction
    in each of `procs` processes, one process per core as ModEM's MPI farm
    runs one (frequency, polarisation) per rank) and scaled by the iterations
    a solve needs.  Returns the baseline and the measured wall time of each
    timed sample step."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    iters, src = cpu_iterations(name)
    walls, res = [], []
    with ctx.Pool(procs, initializer=_cpu_init, initargs=(name,)) as pool:
        for k in range(warmup + steps):
            t0 = time.perf_counter()
            r = pool.map(_cpu_worker, [1 + i % 2 for i in range(procs)], chunksize=1)
            if k >= warmup:
                walls.append(time.perf_counter() - t0)
                res += r
    t_it = float(np.mean([t / n for t, n in res]))
    per_proc = 1.0 / (t_it * iters)
    return {"value": procs * per_proc, "unit": "solves/s", "cores": procs, "kind": "port-projected",
            "sample": f"{steps} step(s) of {procs} processes x {CPU_SAMPLE_ITERS} QMR+D-ILU iterations (+1 div. "
                      f"correction) of the first frequency's forward solves on the workload grid "
                      f"({np.mean(walls):.1f} s wall per step); {t_it:.3f} s/iteration x {iters:.0f} iterations "
                      f"per solve, the mean of {src}",
            "seconds_per_iteration": t_it, "iterations_per_solve": iters}, walls


# --------------------------------------------------------------------------
# replicas: every rank solves its own copy; the job's rate is the solves of all
# ranks over the slowest rank's time
# --------------------------------------------------------------------------
def make_max_over_ranks(dist, device):
    """x -> max of x over the ranks of the default process group (identity
    without one)."""
    def f(x):
        if dist is None:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return f


def replica_rate(solves_per_rank: float, seconds: float, world: int, max_over_ranks) -> float:
    """Whole-job throughput of `world` replicas: world * solves / max time."""
    return world * solves_per_rank / max_over_ranks(seconds)


# --------------------------------------------------------------------------
def stencil_bytes(kprec: int, nE: int, nN: int, fused: bool = False) -> float:
    """Algorithmic bytes per edge and right-hand side of one staged stencil
    launch.  Unfused (v = A ph with rt . v, or t = A sh with t . s, t . t):
    read the input vector, the auxiliary vector and sigma, the signed node
    weight (nN / nE per edge), write the output.  Fused FP32 iteration:
    vh = D^-1 A u with the shadow's (rt, v) reads the same, th = D^-1 A sh
    with its dots needs no auxiliary vector (s is the staged input); the
    two launches alternate, so a launch averages 2.5 vectors.  With the
    polynomial preconditioner the first launch of each product (w = D^-1 A
    u) reads and writes two vectors and the second (with the dots) three:
    2.5 again."""
    sc = 8 if kprec else 16
    sr = 4 if kprec else 8
    return (2.5 if (fused and kprec) else 3) * sc + sr + sr * nN / nE


# DRAM bytes (read + write) per edge and right-hand side of one stencil
# launch, measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum) on
# the 200x200x100 workload with 8 right-hand sides: the unfused kct_vt, and
# the fused kh_vt averaged over the four stages of the polynomial iteration
TRAFFIC_PER_EDGE_RHS = 28.7
TRAFFIC_PER_EDGE_RHS_FUSED = 23.8


def surface_sites(model: models.Model, nrec: int) -> np.ndarray:
    """nrec x nrec sites at the surface centres of the core cells that carry
    the adjoint sources (x, y, z from the grid origin)."""
    g = model.grid
    xe = np.concatenate([[0.0], np.cumsum(g.dx)])
    ye = np.concatenate([[0.0], np.cumsum(g.dy)])
    ix = np.linspace(g.nx * 0.3, g.nx * 0.7, nrec).astype(int)
    iy = np.linspace(g.ny * 0.3, g.ny * 0.7, nrec).astype(int)
    return np.array([[0.5 * (xe[i] + xe[i + 1]), 0.5 * (ye[j] + ye[j + 1]), 0.0] for j in iy for i in ix])


def z_error(Z, Zref) -> float:
    """Largest impedance error over sites, relative per site to the largest
    |Z_ij| of the reference tensor there."""
    Z, Zref = np.asarray(Z).reshape(-1, 4), np.asarray(Zref).reshape(-1, 4)
    return float(np.max(np.max(np.abs(Z - Zref), axis=1) / np.max(np.abs(Zref), axis=1)))


def bench_config(workload_name: str, desc: str, per_step: list, world: int) -> dict:
    """The workload description both arms report."""
    return {"workload": f"{workload_name}: {desc}", "solves_per_step": per_step[0], "tol": TOL,
            "precision": "mixed: FP32 BiCGStab cycles, FP64 residual refinement",
            "formulation": "curl-curl + grad-div (SP2)",
            "l2": "fields larger than L2 (no flush)" if workload_name == "combined" else
                  "no flush: the solve re-reads its own vectors every iteration",
            "parallelism": f"replicas x{world}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=os.environ.get("MT3D_BENCH_WORKLOAD", "combined"))
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    probs, desc = workload(args.workload)
    per_step = [sum(4 * len(step_rows(args.workload, len(p[1]) // 2, s)) for p in probs) for s in range(args.steps)]
    config = bench_config(args.workload, desc, per_step, world)

    if args.impl == "reference":
        if rank != 0:
            return
        procs = min(os.cpu_count() or 1, 8)
        # each step is a bounded sample of the workload (a fixed number of
        # Krylov iterations per process); ms_per_step is its measured wall time
        cb, walls = cpu_baseline(args.workload, procs, steps=args.steps, warmup=min(args.warmup, 1))
        line = {"metric": METRIC, "value": cb["value"], "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": float(np.mean(walls)) * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c128",
                "data": "synthetic (seeded random-field models of the stated shapes)",
                "config": config, "impl": "reference", "cpu_baseline": cb,
                "note": "value projected: the CPU time per Krylov iteration measured in the timed sample steps "
                        "times the iterations a solve needs; ms_per_step is the measured wall time of one "
                        "sample step (not of a whole step of the workload)",
                "e2e": {"value": cb["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=900))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    from mt3d import capi

    def mixed_control(s):
        s.set_control(tolEMfwd=TOL, tolEMadj=TOL, IterPerDivCor=CYCLE, MaxDivCor=MAX_CYCLES, precision=capi.PREC_MIXED)

    # per model: solver handle and the device-resident inputs of every step
    solvers = []
    nsteps_distinct = min(args.steps, 8) if args.workload == "combined" else 1
    for m, oms, bcs, srcs in probs:
        s = capi.Solver(m.grid, device=local)
        s.set_formulation(capi.FORM_CCGD)
        s.set_restart(RESTART)
        s.set_fused(FUSED)
        s.set_poly(POLY)
        s.update_cond(m.m_earth, m.air_cond)
        mixed_control(s)
        s.set_stream(stream.cuda_stream)
        batches = []
        for st in range(nsteps_distinct):
            om, bc, src, tr = step_batch(oms, bcs, srcs, step_rows(args.workload, len(oms) // 2, st))
            batches.append((om, torch.from_numpy(bc).to(dev), torch.from_numpy(src).to(dev), tr))
        nmax = max(len(b[0]) for b in batches)
        d_e = torch.zeros((nmax, s.nE), dtype=torch.complex128, device=dev)
        solvers.append((s, batches, d_e, m))

    multi = len(solvers) > 1
    zchunks = None
    if multi:
        # models of uneven size in one call per step (mt3d_fwdsolve_multi);
        # the per-grid stencil chunking tuned once and cached
        from mt3d import tune
        b0 = [batches[0] for _, batches, _, _ in solvers]
        zchunks = tune.tune([s for s, *_ in solvers], [b[0] for b in b0],
                            [d_e[:len(b[0])].data_ptr() for (_, _, d_e, _), b in zip(solvers, b0)],
                            [b[1].data_ptr() for b in b0], [b[2].data_ptr() for b in b0], [b[3] for b in b0],
                            lambda: torch.cuda.synchronize(dev),
                            cache_path=os.environ.get("MT3D_TUNE_CACHE",
                                                      os.path.join(tempfile.gettempdir(), "mt3d_tune.json")),
                            reset=lambda: [d_e.zero_() for _, _, d_e, _ in solvers])

    def step(k):
        if multi:
            bs = [batches[k % len(batches)] for _, batches, _, _ in solvers]
            es = [d_e[:len(b[0])] for (_, _, d_e, _), b in zip(solvers, bs)]
            for e in es:
                e.zero_()
            capi.fwdsolve_multi([s for s, *_ in solvers], [b[0] for b in bs], [e.data_ptr() for e in es],
                                trans=[b[3] for b in bs], bc=[b[1].data_ptr() for b in bs],
                                src=[b[2].data_ptr() for b in bs], zchunks=zchunks, device=True)
            return
        for s, batches, d_e, _ in solvers:
            om, d_bc, d_src, tr = batches[k % len(batches)]
            e = d_e[:len(om)]
            e.zero_()
            s.fwdsolve_batch_device(om, e.data_ptr(), bc_ptr=d_bc.data_ptr(), src_ptr=d_src.data_ptr(), trans=tr)

    def step_stats(k):
        out = []
        for s, batches, *_ in solvers:
            n = len(batches[k % len(batches)][0])
            it, rr = s.batch_diagnostics(n)
            out.append((it.copy(), rr.copy()))
        return out

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    max_over_ranks = make_max_over_ranks(dist, dev)

    for k in range(args.warmup):
        step(k)
    # timed region: the K steps alone (no kernel profiling; the per-step
    # diagnostics are read between the steps' events)
    clocks = Clocks(local)
    stats = []
    L = capi.load()
    barrier()
    launches0 = int(L.mt3d_launch_counter())
    clocks.start()
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for k in range(args.steps):
        ev0[k].record(stream)
        step(k)
        ev1[k].record(stream)
        stats.append(step_stats(k))
    barrier()
    launches = int(L.mt3d_launch_counter()) - launches0
    ck = clocks.stop()
    step_ms = [ev0[k].elapsed_time(ev1[k]) for k in range(args.steps)]
    ms_dev = max_over_ranks(sum(step_ms))
    n_solves = sum(per_step)
    value = replica_rate(n_solves, sum(step_ms) / 1e3, world, max_over_ranks)

    # profiling pass (after the timed region): the first step again with
    # CUDA events around every stencil launch.  Roofline of the FP32 stencil
    # kernel (both launches of every iteration): algorithmic bytes of the
    # right-hand-side sweeps the kernel made, over its summed event time; the
    # FP64 launches of the refinement fallback are reported beside it.  The
    # mixed fields of this step are kept for the parity comparison.
    for s, *_ in solvers:
        s.profile(True)
    step(0)
    barrier()
    kn = {0: 0, 1: 0}
    kms = {0: 0.0, 1: 0.0}
    alg = {0: 0.0, 1: 0.0}
    units = {0: 0.0, 1: 0.0}
    for s, *_ in solvers:
        for prec in (0, 1):
            n, ms, sw = s.kernel_time(prec)
            kn[prec] += n
            kms[prec] += ms
            units[prec] += float(s.nE) * sw
            alg[prec] += float(s.nE) * sw * stencil_bytes(prec, s.nE, s.nN, FUSED)
        s.profile(False)
    e_mixed = [d_e[:len(b[0][0])].clone() for _, b, d_e, _ in solvers]
    converged = all(np.all(rr <= TOL) for st in stats for _, rr in st)
    max_relres = max(float(np.max(rr)) for st in stats for _, rr in st)
    its = np.concatenate([it for st in stats for it, _ in st])
    peak, peak_kind = peaks()
    kp = 1 if kms[1] > 0 else 0
    # with the polynomial preconditioner each timed event pair brackets the
    # two stencil launches of one preconditioned product
    st_launches = kn[kp] * (2 if (kp and POLY > 0) else 1)
    achieved = (alg[kp] / (kms[kp] / 1e3) / 1e9) if kms[kp] > 0 else None
    traffic = None
    if kp and st_launches:
        per_unit = (TRAFFIC_PER_EDGE_RHS_FUSED if POLY > 0 else None) if FUSED else TRAFFIC_PER_EDGE_RHS
        traffic = per_unit * units[kp] / st_launches if per_unit else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "kernel": ((f"kh_vt (TMA-staged stencil + grad-div + D^-1 at the output edge + fused dots; "
                             f"polynomial preconditioner c = {POLY}: two launches per product)" if FUSED
                            else "kct_vt (TMA-staged stencil + grad-div + fused dots)") + ", FP32" if kp else
                           "kcs_vt (cp.async-staged stencil + grad-div + fused dots), FP64") + " complex",
                "peak_kind": peak_kind, "timed_launches": st_launches,
                "timing": "CUDA events around every stencil launch on the solver stream, in a separate pass "
                          "over the first step after the timed region",
                "bytes_per_edge_rhs": alg[kp] / units[kp] if units[kp] else None,
                "algorithmic_bytes_per_launch": alg[kp] / st_launches if st_launches else None,
                "fp64_fallback": {"launches": kn[0], "ms": kms[0],
                                  "achieved_gbs": (alg[0] / (kms[0] / 1e3) / 1e9) if kms[0] > 0 else None,
                                  "share_of_stencil_time": kms[0] / (kms[0] + kms[1]) if kms[0] + kms[1] > 0 else 0.0}}

    # end to end through the C ABI with pinned host buffers, copies inside the timed region
    e2e = None
    if not args.no_e2e and multi:
        ke = min(args.steps, 2)
        h2d = d2h = 0
        pinned = []
        for k in range(ke):
            per = []
            for s, batches, d_e, _ in solvers:
                om, d_bc, d_src, tr = batches[k % len(batches)]
                hb = torch.empty(tuple(d_bc.shape), dtype=torch.complex128).pin_memory()
                hs_ = torch.empty_like(hb).pin_memory()
                he = torch.empty_like(hb).pin_memory()
                hb.copy_(d_bc.cpu())
                hs_.copy_(d_src.cpu())
                per.append((om, hb.numpy(), hs_.numpy(), he.numpy(), tr, he))
            pinned.append(per)
        barrier()
        t0 = time.perf_counter()
        for per in pinned:
            for p in per:
                p[5].zero_()  # zero first guesses in the pinned in/out buffers
            capi.fwdsolve_multi([s for s, *_ in solvers], [p[0] for p in per], [p[3] for p in per],
                                trans=[p[4] for p in per], bc=[p[1] for p in per], src=[p[2] for p in per],
                                zchunks=zchunks)
            h2d += sum(p[1].nbytes + p[2].nbytes + p[3].nbytes for p in per)
            d2h += sum(p[3].nbytes for p in per)
        barrier()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        e2e = {"value": world * sum(per_step[:ke]) / e2e_s, "unit": "solves/s", "steps": ke,
               "h2d_bytes_per_step": h2d // ke, "d2h_bytes_per_step": d2h // ke, "entry": "mt3d_fwdsolve_multi",
               "device_value_same_steps": replica_rate(sum(per_step[:ke]), sum(step_ms[:ke]) / 1e3, world,
                                                       max_over_ranks)}
        del pinned
    elif not args.no_e2e:
        ke = min(args.steps, 2)
        pinned = []
        for s, batches, d_e, _ in solvers:
            per = []
            for k in range(ke):
                om, d_bc, d_src, tr = batches[k % len(batches)]
                hbc = torch.empty(tuple(d_bc.shape), dtype=torch.complex128).pin_memory()
                hsrc = torch.empty_like(hbc).pin_memory()
                he = torch.empty_like(hbc).pin_memory()
                hbc.copy_(d_bc.cpu())
                hsrc.copy_(d_src.cpu())
                per.append((om, hbc.numpy(), hsrc.numpy(), he, tr))
            pinned.append(per)
        h2d = d2h = 0
        barrier()
        t0 = time.perf_counter()
        for k in range(ke):
            for (s, batches, d_e, _), per in zip(solvers, pinned):
                om, hbc, hsrc, he, tr = per[k]
                # zero first guess in the pinned in/out buffer (host threads),
                # copied to the device and the solution back by the library
                he.zero_()
                s.fwdsolve_batch(om, bc=hbc, src=hsrc, trans=tr, out=he.numpy())
                h2d += hbc.nbytes + hsrc.nbytes + he.numel() * he.element_size()
                d2h += he.numel() * he.element_size()
        barrier()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        e2e = {"value": world * sum(per_step[:ke]) / e2e_s, "unit": "solves/s", "steps": ke,
               "h2d_bytes_per_step": h2d // ke, "d2h_bytes_per_step": d2h // ke,
               "entry": "mt3d_fwdsolve_batch (pinned host buffers)",
               "device_value_same_steps": replica_rate(sum(per_step[:ke]), sum(step_ms[:ke]) / 1e3, world,
                                                       max_over_ranks)}
        del pinned

    # plain FP64 path on the right-hand sides of the first step, one at a
    # time; its fields are compared with the mixed ones of the same step
    fp64 = None
    parity = None
    if not args.no_fp64:
        e_fp64 = []
        barrier()
        t0 = time.perf_counter()
        nfp = 0
        for s, batches, d_e, _ in solvers:
            om, d_bc, d_src, tr = batches[0]
            s.set_control(tolEMfwd=TOL, tolEMadj=TOL, IterPerDivCor=CYCLE, MaxDivCor=MAX_CYCLES,
                          precision=capi.PREC_FP64)
            ef = torch.zeros((len(om), s.nE), dtype=torch.complex128, device=dev)
            for r in range(len(om)):
                s.fwdsolve_batch_device(om[r:r + 1], ef[r].data_ptr(), bc_ptr=d_bc[r:r + 1].data_ptr(),
                                        src_ptr=d_src[r:r + 1].data_ptr(), trans=tr[r:r + 1])
                nfp += 1
            mixed_control(s)
            e_fp64.append(ef)
        barrier()
        fp64_s = max_over_ranks(time.perf_counter() - t0)
        fp64 = {"value": world * nfp / fp64_s, "unit": "solves/s", "solves": nfp,
                "kernel": "kcs_vt (cp.async-staged FP64 stencil on the reference's edge order)",
                "mixed_same_rhs": world * per_step[0] / max_over_ranks(step_ms[0] / 1e3),
                "speedup": (per_step[0] / (step_ms[0] / 1e3)) / (nfp / fp64_s)}
        if not args.no_parity:
            parity = field_parity(capi, solvers, e_mixed, e_fp64, dev, mixed_control)

    if rank == 0:
        cb = None
        if world == 1 and not args.no_cpu:
            cb, _ = cpu_baseline(args.workload, min(os.cpu_count() or 1, 8))
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_dev / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c64 (Krylov) / c128 (refinement)",
                "data": "synthetic (seeded random-field models of the stated shapes)", "config": config,
                "converged": bool(converged), "max_relres": max_relres,
                "iterations_per_solve": {"mean": float(its.mean()), "min": int(its.min()), "max": int(its.max())},
                "fp64": fp64, "parity": parity, "e2e": e2e, "roofline": roofline, "cpu_baseline": cb, "clocks": ck,
                "gpu_launches": launches}
        if multi:
            line["config"]["multi_grid"] = {"entry": "mt3d_fwdsolve_multi_device, one call per step",
                                            "zchunks": zchunks}
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def field_parity(capi, solvers, e_mixed, e_fp64, dev, mixed_control):
    """Mixed-precision against FP64 fields of the first step's right-hand
    sides, and the impedances (Full_Impedance at the receiver array) of its
    forward solves: the relative 2-norm difference of every field, and the
    site-relative impedance difference.  One frequency's forward pair is
    also solved in FP64 to TIGHT_TOL, three orders below the benchmark's
    tolerance, and both 1e-7 solutions' impedances are compared with it."""
    import torch
    out = {"tight_tol": TIGHT_TOL}
    e_err, z_err, z_tight = [], [], {"mixed": 0.0, "fp64": 0.0}
    for (s, batches, d_e, m), em, ef in zip(solvers, e_mixed, e_fp64):
        om, d_bc, d_src, tr = batches[0]
        n = len(om)
        for r in range(n):
            e_err.append(float(torch.linalg.norm(em[r] - ef[r]) / torch.linalg.norm(ef[r])))
        sites = surface_sites(m, 20)
        fwd = [r for r in range(n) if tr[r] == 0]
        pairs = [(fwd[q], fwd[q + 1]) for q in range(0, len(fwd) - 1, 2)]
        for a, b in pairs:
            zm = s.impedance(om[a], sites, em[a].data_ptr(), em[b].data_ptr())
            zf = s.impedance(om[a], sites, ef[a].data_ptr(), ef[b].data_ptr())
            z_err.append(z_error(zm, zf))
        # tight FP64 reference for the first forward pair
        a, b = pairs[0]
        s.set_control(tolEMfwd=TIGHT_TOL, tolEMadj=TIGHT_TOL, IterPerDivCor=CYCLE, MaxDivCor=4 * MAX_CYCLES,
                      precision=capi.PREC_FP64)
        et = torch.zeros((2, s.nE), dtype=torch.complex128, device=dev)
        bc2 = d_bc[[a, b]].contiguous()
        st, rc = s.fwdsolve_batch_device(om[[a, b]], et.data_ptr(), bc_ptr=bc2.data_ptr(), src_ptr=None,
                                         trans=tr[[a, b]])
        torch.cuda.synchronize(dev)
        del bc2
        it, rr = s.batch_diagnostics(2)
        mixed_control(s)
        zt = s.impedance(om[a], sites, et[0].data_ptr(), et[1].data_ptr())
        z_tight["mixed"] = max(z_tight["mixed"],
                               z_error(s.impedance(om[a], sites, em[a].data_ptr(), em[b].data_ptr()), zt))
        z_tight["fp64"] = max(z_tight["fp64"],
                              z_error(s.impedance(om[a], sites, ef[a].data_ptr(), ef[b].data_ptr()), zt))
        out["tight_relres"] = float(np.max(rr))
        out["tight_freq_hz"] = float(om[a] / (2 * np.pi))
    out.update({"E_mixed_vs_fp64_max": max(e_err), "Z_mixed_vs_fp64_max": max(z_err),
                "Z_vs_tight": z_tight, "sites": "20x20 surface receivers on the core cells",
                "E_norm": "relative 2-norm over the full edge vector, every right-hand side of the step",
                "Z_norm": "max over sites of max_ij |dZ_ij| / max_ij |Z_ij|"})
    return out


if __name__ == "__main__":
    main()
