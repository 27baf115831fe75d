#!/usr/bin/env python
"""Throughput of the 3D-MT forward + adjoint solve on B200 GPUs.

One step = every right-hand side of the workload solved to a relative residual
of 1e-7 of the FP64 system: the forward solves (all frequencies x 2
polarisations, plane-wave boundary data) and the adjoint (transposed) solves
(all frequencies x 2 polarisations, synthetic receiver sources), each batch in
one call of the C ABI.  The metric is solves/s over all ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload combined|precision|batch|small]

With N > 1 (torchrun) every rank solves its own copy of the workload (replicas;
the right-hand sides are independent), timed between barriers, max over ranks.
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
    """[(model, omegas, bc[nf*2], src[nf*2])] and a description."""
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


def _cpu_worker(args):
    name, k, w, seconds = args
    from oracle.oracle import Oracle, QMR, PC_DILU
    probs, _ = workload(name)
    m, oms, bcs, _ = probs[k]
    o = Oracle(m.grid)
    o.update_cond(m.m_earth, m.air_cond)
    o.update_freq(oms[w])
    o.set_control(solver=QMR, precond=PC_DILU, IterPerDivCor=CPU_SAMPLE_ITERS, MaxDivCor=1)
    t0 = time.perf_counter()
    o.fwdsolve(bc=bcs[w])
    d = o.diagnostics()
    return (time.perf_counter() - t0), max(1, d["nIterTotal"])


def cpu_baseline(name: str, iters_per_solve: float, procs: int):
    """Per-iteration cost of the CPU solver on the workload grid from a bounded
    sample (CPU_SAMPLE_ITERS Krylov iterations + one divergence correction per
    process, one process per core as ModEM's MPI farm runs one (frequency,
    polarisation) per rank), scaled by the iterations a solve needs."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        t0 = time.perf_counter()
        res = pool.map(_cpu_worker, [(name, 0, i % 2, 0) for i in range(procs)])
        wall = time.perf_counter() - t0
    t_it = float(np.mean([t / n for t, n in res]))
    per_proc = 1.0 / (t_it * iters_per_solve)
    return {"value": procs * per_proc, "unit": "solves/s", "cores": procs, "kind": "port",
            "sample": f"{procs} processes x {CPU_SAMPLE_ITERS} QMR+D-ILU iterations (+1 div. correction) of the "
                      f"first forward right-hand side on the workload grid ({wall:.1f} s wall); "
                      f"{t_it:.3f} s/iteration scaled by {iters_per_solve:.0f} iterations per solve"}


# --------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=os.environ.get("MT3D_BENCH_WORKLOAD", "precision"))
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        probs, desc = workload(args.workload)
        procs = min(os.cpu_count() or 1, 8)
        iters = float(os.environ.get("MT3D_CPU_ITERS_PER_SOLVE", "600"))
        cb = cpu_baseline(args.workload, iters, procs)
        step_s = 1.0 / cb["value"] * sum(2 * len(p[1]) for p in probs)
        line = {"metric": METRIC, "value": cb["value"], "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "c128", "data": "synthetic",
                "config": {"workload": f"{args.workload}: {desc}"}, "impl": "reference", "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from mt3d import capi

    probs, desc = workload(args.workload)
    solvers = []
    for m, oms, bcs, srcs in probs:
        s = capi.Solver(m.grid, device=local)
        s.set_formulation(capi.FORM_CCGD)
        s.update_cond(m.m_earth, m.air_cond)
        s.set_control(tolEMfwd=TOL, tolEMadj=TOL, IterPerDivCor=120, MaxDivCor=100, precision=capi.PREC_MIXED)
        s.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        nr = len(oms)
        # rows 0..nr-1: forward (boundary data, no source); nr..2nr-1: adjoint (source, no boundary data)
        zb = np.zeros_like(bcs)
        d_bc = torch.from_numpy(np.concatenate([bcs, zb])).to(dev)
        d_src = torch.from_numpy(np.concatenate([zb, srcs])).to(dev)
        d_e = torch.zeros((2 * nr, s.nE), dtype=torch.complex128, device=dev)
        tr = np.concatenate([np.zeros(nr, np.int32), np.ones(nr, np.int32)])
        solvers.append((s, np.concatenate([oms, oms]), d_bc, d_src, d_e, tr))
    n_solves = sum(2 * len(p[1]) for p in probs)

    def step(stats=None):
        # forward and adjoint right-hand sides of a model in one batched call
        for s, oms2, d_bc, d_src, d_e, tr in solvers:
            d_e.zero_()
            st, rc = s.fwdsolve_batch_device(oms2, d_e.data_ptr(), bc_ptr=d_bc.data_ptr(), src_ptr=d_src.data_ptr(),
                                             trans=tr)
            if stats is not None:
                it, rr = s.batch_diagnostics(len(oms2))
                stats.append((s.nE, it.copy(), rr.copy(), st.copy()))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        step()
    clocks = Clocks(local)
    for s, *_ in solvers:
        s.profile(True)
    stats = []
    L = capi.load()
    barrier()
    launches0 = int(L.mt3d_launch_counter())
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        step(stats)
    ev1.record()
    barrier()
    launches = int(L.mt3d_launch_counter()) - launches0
    ck = clocks.stop()
    ms_dev = max_over_ranks(ev0.elapsed_time(ev1))
    value = world * n_solves * args.steps / (ms_dev / 1e3)
    # roofline of the stencil kernels (v = A ph and t = A sh, fused dot products)
    kn, kms, kprec = 0, 0.0, 1
    for s, *_ in solvers:
        n, ms, pr = s.kernel_time()
        kn += n
        kms += ms
        kprec = pr
        s.profile(False)
    sc = 8 if kprec else 16  # bytes of one complex entry
    sr = 4 if kprec else 8
    # per edge and right-hand side: read the preconditioned vector, rt (or s),
    # sigma and the grad-div node potentials (one node per edge on average:
    # nN / nE ~ 1/3 of a complex); write the result
    b_edge = 3 * sc + sr + sc / 3
    alg_bytes = sum(float(nE) * it.sum() * 2 * b_edge for nE, it, rr, st in stats)
    converged = all(np.all(st == 0) for _, _, _, st in stats)
    max_relres = max(float(np.max(rr)) for _, _, rr, _ in stats)
    peak, peak_kind = peaks()
    achieved = (alg_bytes / (kms / 1e3) / 1e9) if kms > 0 else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": None,
                "kernel": "kb_v/kb_t (stencil + fused dots), FP32 complex" if kprec else "kb_v/kb_t FP64",
                "peak_kind": peak_kind, "timed_launches": kn, "bytes_per_edge_rhs": b_edge}

    # end to end through the C ABI with host buffers (pinned), copies inside
    pinned = []
    for s, oms2, d_bc, d_src, d_e, tr in solvers:
        hbc = torch.empty(tuple(d_bc.shape), dtype=torch.complex128).pin_memory()
        hsrc = torch.empty_like(hbc).pin_memory()
        he = torch.empty_like(hbc).pin_memory()
        hbc.copy_(d_bc.cpu())
        hsrc.copy_(d_src.cpu())
        pinned.append((hbc.numpy(), hsrc.numpy(), he.numpy()))
    h2d = d2h = 0
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for (s, oms2, d_bc, d_src, d_e, tr), (hbc, hsrc, he) in zip(solvers, pinned):
            he[:] = 0
            s.fwdsolve_batch(oms2, bc=hbc, src=hsrc, e0=he, trans=tr)
            h2d += hbc.nbytes + hsrc.nbytes + he.nbytes
            d2h += he.nbytes
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": world * n_solves * args.steps / e2e_s, "unit": "solves/s",
           "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps}

    # plain FP64 path, one right-hand side at a time (the comparison point)
    fp64 = None
    if not args.no_fp64:
        barrier()
        t0 = time.perf_counter()
        nfp = 0
        for s, oms2, d_bc, d_src, d_e, tr in solvers:
            s.set_control(tolEMfwd=TOL, tolEMadj=TOL, IterPerDivCor=120, MaxDivCor=100, precision=capi.PREC_FP64)
            for r in range(len(oms2)):
                e1 = torch.zeros((1, s.nE), dtype=torch.complex128, device=dev)
                s.fwdsolve_batch_device(oms2[r:r + 1], e1.data_ptr(), bc_ptr=d_bc[r:r + 1].data_ptr(),
                                        src_ptr=d_src[r:r + 1].data_ptr(), trans=tr[r:r + 1])
                nfp += 1
            s.set_control(tolEMfwd=TOL, tolEMadj=TOL, IterPerDivCor=120, MaxDivCor=100, precision=capi.PREC_MIXED)
        barrier()
        fp64_s = max_over_ranks(time.perf_counter() - t0)
        fp64 = world * nfp / fp64_s

    if rank == 0:
        cb = None
        if world == 1 and not args.no_cpu:
            its = [int(np.mean(it)) for _, it, _, _ in stats]
            cb = cpu_baseline(args.workload, float(os.environ.get("MT3D_CPU_ITERS_PER_SOLVE", "600")),
                              min(os.cpu_count() or 1, 8))
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_dev / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c64 inner / c128 refinement", "data": "synthetic",
                "config": {"workload": f"{args.workload}: {desc}", "solves_per_step": n_solves, "tol": TOL,
                           "precision": "mixed (FP32 BiCGStab, FP64 residual refinement)", "formulation": "curl-curl + grad-div (SP2), diagonal preconditioner",
                           "l2": "fields larger than L2 (flush not needed)" if args.workload == "combined" else
                                 "inputs smaller than L2 at this size; no flush (iterative solve re-reads its own "
                                 "vectors every iteration)",
                           "parallelism": f"replicas x{world}"},
                "converged": bool(converged), "max_relres": max_relres,
                "fp64_solves_per_s": fp64, "speedup_vs_fp64": (value / fp64) if fp64 else None,
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cb, "clocks": ck, "gpu_launches": launches}
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
