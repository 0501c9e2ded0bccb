"""The multi-rank bench path on CPU: ranks as gloo processes (world size 2).

The single-graph optimiser runs as independent replicas, one per GPU; the
only cross-rank step is the max over ranks of the timed region, after which
the job's throughput is every rank's links over the slowest rank's time."""
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took (r + 1) * 100 ms per step and (r + 1) * 2 s end to end
        ms, e2e = bench.slowest_over_ranks([(rank + 1) * 100.0, (rank + 1) * 2.0], dist, "cpu")
        q.put((rank, ms, e2e, bench.job_throughput(world, 1_000_000, ms / 1e3)))
    finally:
        dist.destroy_process_group()


def test_slowest_rank_sets_the_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, e2e, value in got:
        assert ms == 200.0 and e2e == 4.0  # every rank sees the slowest rank's times
        assert value == pytest.approx(2 * 1_000_000 / 0.2)


def test_single_rank_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.slowest_over_ranks([3.0, 1.5], None, "cpu") == [3.0, 1.5]
    assert bench.job_throughput(1, 10, 2.0) == 5.0


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_lpt_assign_balances_and_covers():
    import numpy as np

    from relaxmap_b200.sharding import lpt_assign
    rng = np.random.default_rng(1)
    w = rng.integers(1000, 600000, 4096).astype(np.float64)
    for world in (1, 2, 4, 8):
        parts = lpt_assign(w, world)
        allg = np.sort(np.concatenate(parts))
        assert np.array_equal(allg, np.arange(len(w)))
        loads = [w[p].sum() for p in parts]
        assert max(loads) <= w.sum() / world + w.max()  # LPT bound: within one item of the mean


def _combine_rank(rank, world, port, q):
    import datetime

    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    from relaxmap_b200.sharding import combine, lpt_assign
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w = np.arange(1, 11, dtype=np.float64)
        mine = lpt_assign(w, world)[rank]
        q.put((rank, combine(10, mine, mine * 1.5, dist, "cpu").tolist()))
    finally:
        dist.destroy_process_group()


def test_batched_results_combine_over_two_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_combine_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    for _ in range(world):
        rank, v = q.get(timeout=10)
        assert v == [1.5 * g for g in range(10)]  # every graph once, from whichever rank ran it


def test_bench_edge_list_file_reads_back(tmp_path):
    """bench.py --with-io writes the workload graph as an edge list; the
    loader reads back the same links with the weights to 6 significant
    digits."""
    import numpy as np
    import bench
    from relaxmap_b200 import parse_file, synth
    g = synth.config_small(seed=3)
    g.w = np.random.default_rng(1).uniform(1, 10, g.m)
    p = tmp_path / "g.txt"
    size = bench.write_edge_list(p, g, chunk=1000)
    assert size == p.stat().st_size
    d = parse_file(p, threads=2)
    assert d["n"] == g.n
    np.testing.assert_array_equal(d["src"], g.src)
    np.testing.assert_array_equal(d["dst"], g.dst)
    np.testing.assert_allclose(d["w"], g.w, rtol=5e-6)
    g.w = None  # unweighted: two columns, every weight read as 1
    bench.write_edge_list(p, g, chunk=777)
    d = parse_file(p, threads=1)
    np.testing.assert_array_equal(d["src"], g.src)
    np.testing.assert_array_equal(d["w"], np.ones(g.m))
