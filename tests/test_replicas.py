"""The multi-rank (replica) host logic of bench.py on CPU with gloo, world
size 2: rank discovery from the torchrun environment, the max-over-ranks
reduction every timed leg goes through, the whole-job rate, the served-stream
aggregation, and the reference arm's rank-0-only rule.  Each rank also runs
a replica of a small projector step through the oracle, so the reduction is
exercised on real per-rank timings."""
import datetime
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                          WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
        sys.path.insert(0, ROOT)
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import time

        import torch.distributed as dist

        import bench
        import oracle
        from helpers import small_circular
        dist.init_process_group("gloo", rank=rank, world_size=ws,
                                timeout=datetime.timedelta(seconds=60))
        assert bench.dist_env() == (ws, rank, rank)
        # a replica step: every rank projects its own seeded phantom
        vol, scan, x = small_circular(seed=3 + rank)
        t0 = time.perf_counter()
        oracle.view_proj3D.sinoproj_linear(None, scan.frame_vectors, *scan.shape, scan.du,
                                           scan.dv, scan.u0, scan.v0, x, *vol.grid)
        ms = (time.perf_counter() - t0) * 1e3 + 50.0 * rank  # rank 1 is the slow one
        t = bench.max_over_ranks(ms, ws)
        rate = bench.replica_rate(vol.nvox * scan.ns, ws, t)
        summ = bench._replica_summary({"wall_s": 2.0 + rank, "p50_s": 0.5 + rank,
                                       "p99_s": 1.0 + rank, "max_s": 1.5 + rank,
                                       "recon_per_s": 5.0 / (2.0 + rank)}, 5, ws, None)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ms, t, rate, summ))
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, "error", repr(e), None, None))


def test_replica_reductions_with_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=240)
        res[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert res[r][1] != "error", res[r]
    ms = [res[0][1], res[1][1]]
    for r in (0, 1):
        _, _, t, rate, summ = res[r]
        assert t == pytest.approx(max(ms))  # every rank sees the slowest rank's time
        from helpers import small_circular
        vol, scan, _ = small_circular()
        assert rate == pytest.approx(2 * vol.nvox * scan.ns / (max(ms) * 1e-3) / 1e9)
        assert summ["wall_s"] == 3.0 and summ["p99_s"] == 2.0 and summ["max_s"] == 2.5
        assert summ["recon_per_s"] == pytest.approx(10 / 3.0)


def test_single_rank_helpers_are_identities(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench.dist_env() == (1, 0, 0)
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_rate(2e9, 1, 1000.0) == pytest.approx(2.0)
    s = {"wall_s": 1.0, "p50_s": 0.1, "p99_s": 0.2, "recon_per_s": 4.0}
    assert bench._replica_summary(s, 4, 1, None) is s


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun the other ranks exit without work or output."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        gpus, steps, warmup = 2, 1, 1
    assert bench.run_reference(Args()) is None
    assert capsys.readouterr().out == ""
