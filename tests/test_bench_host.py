"""Host logic of bench.py on CPU: the replica aggregation over ranks (gloo,
world size 2) and the step schedule of the 16-frequency workload."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    mor = bench.make_max_over_ranks(dist, "cpu")
    # rank r took 2 + r seconds for its 8 solves
    rate = bench.replica_rate(8, 2.0 + rank, world, mor)
    slowest = mor(2.0 + rank)
    q.put((rank, rate, slowest))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_rate_is_total_over_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rate, slowest in res:
        assert slowest == pytest.approx(3.0)
        assert rate == pytest.approx(2 * 8 / 3.0)


def test_single_process_rate():
    mor = bench.make_max_over_ranks(None, "cpu")
    assert bench.replica_rate(8, 4.0, 1, mor) == pytest.approx(2.0)


def test_steps_cover_all_frequencies_once():
    seen = []
    for s in range(8):
        seen += bench.step_rows("combined", 16, s)
    assert sorted(seen) == list(range(16))
    assert bench.step_rows("precision", 1, 5) == [0]


def test_impedance_error_is_site_relative():
    import numpy as np
    Zref = np.array([[[0.0, 2.0], [-2.0, 0.0]], [[0.0, 10.0], [-10.0, 0.0]]], complex)
    Z = Zref.copy()
    Z[0, 0, 1] += 2e-6  # 1e-6 of the first site's largest component
    Z[1, 1, 0] += 5e-6  # 5e-7 of the second site's
    assert abs(bench.z_error(Z, Zref) - 1e-6) < 1e-12


def test_surface_sites_lie_on_core_cells():
    import numpy as np
    from mt3d import models
    m, _ = models.config_small_forward()
    s = bench.surface_sites(m, 4)
    assert s.shape == (16, 3) and np.all(s[:, 2] == 0.0)
    assert np.all((s[:, 0] > 0) & (s[:, 0] < m.grid.dx.sum()) & (s[:, 1] > 0) & (s[:, 1] < m.grid.dy.sum()))


def test_both_arms_report_the_same_config():
    cfg = bench.bench_config("combined", "desc", [8, 8], 1)
    assert cfg == bench.bench_config("combined", "desc", [8, 8], 1)
    assert cfg["workload"] == "combined: desc" and cfg["solves_per_step"] == 8


def test_cpu_iterations_source_is_named():
    it, src = bench.cpu_iterations("combined")
    assert it > 0 and src
    it2, src2 = bench.cpu_iterations("precision")
    assert it2 == bench.CPU_ITERS_PRECISION and "100x100x60" in src2


def test_reference_arm_times_bounded_sample_steps():
    """The CPU baseline (the reference arm's measurement) on the small
    workload: the oracle is set up once per process and each timed step runs
    a fixed number of Krylov iterations in every process, so each step's wall
    time is measured and the projected rate follows from the time per
    iteration."""
    cb, walls = bench.cpu_baseline("small", 2, steps=2, warmup=1)
    assert len(walls) == 2 and all(w > 0 for w in walls)
    assert cb["kind"] == "port-projected" and cb["cores"] == 2
    assert cb["value"] == pytest.approx(2.0 / (cb["seconds_per_iteration"] * cb["iterations_per_solve"]))
    # every timed step ran CPU_SAMPLE_ITERS iterations per process
    assert max(walls) >= bench.CPU_SAMPLE_ITERS * cb["seconds_per_iteration"] * 0.5
