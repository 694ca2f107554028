"""The batched MLEM+TV iteration (ct2b200.batch.EMBatch, C ABI ct2_batch_*):
jobs of different sizes and geometries advanced together -- one projector
launch over all jobs' pixel tiles, the gather backprojector's launches over
all jobs' items per round of view blocks, each job's update -- against the
same jobs iterated alone (ct2b200.recon.EMTVState.iterate).

Every work item runs the single-job kernels' code, so a job's iterate should
be the same alone and in the batch; the bound is 1e-6 relative L2 (the
projector alone takes the TMA-staged form, whose sums equal the untiled
form's), and the test reports whether they are bit-identical.
"""
import numpy as np
import pytest

import oracle
from ct2b200 import workloads as W
from helpers import rel_l2, small_circular

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _case(vol, scan, x, device, seed):
    import torch
    from ct2b200.autograd import ConeGeometry
    y = oracle.view_proj3D.sinoproj_linear(np.ones(scan.shape, np.int32), scan.frame_vectors,
                                           *scan.view, x.astype(np.float32), *vol.grid)
    y = np.maximum(y + 0.02 * np.random.default_rng(seed).standard_normal(y.shape), 0)
    geom = ConeGeometry.from_scan(scan, vol, device)
    return torch.tensor(y.astype(np.float32), device=device), geom


def _jobs(device):
    """Three reconstructions of different sizes and geometries, the last with
    a detector large enough that its ray table takes two view blocks."""
    out = []
    for n, ns, nd, seed in ((24, 16, 32, 1), (30, 22, 40, 2)):
        vol, scan, x = small_circular(n=n, ns=ns, nd=nd, seed=seed)
        out.append((vol,) + _case(vol, scan, x, device, seed))
    vol = W.Volume.centered((20, 18, 22), (2.0, 2.0, 2.0))
    scan = W.circular_scan(30, 1024, 1024, 0.1, 0.1, 300.0, 600.0, s0=0.2)
    x = W.voxelize(vol, W.random_ellipsoids(5, 40.0, seed=4))
    out.append((vol,) + _case(vol, scan, x, device, 4))
    return out


def _states(jobs, tv=0.002):
    import torch
    from ct2b200.recon import EMTVState
    return [EMTVState(torch.full(vol.shape, 0.5, device=y.device), y, geom, tv_weight=tv)
            for vol, y, geom in jobs]


@pytest.fixture(scope="module")
def jobs(cuda):
    return _jobs(cuda)


@pytest.mark.parametrize("graphs", [False, True])
def test_batch_matches_jobs_alone(jobs, graphs):
    import torch
    from ct2b200.batch import EMBatch
    alone = _states(jobs)
    for s in alone:
        for _ in range(3):
            s.iterate()
    batched = _states(jobs)
    B = EMBatch(4, device=batched[0].x.device, graphs=graphs)
    for s in batched:
        B.add(s)
    for _ in range(3):
        B.iterate()
    torch.cuda.synchronize()
    for a, b in zip(alone, batched):
        err = rel_l2(b.x.cpu().numpy(), a.x.cpu().numpy())
        print("batched vs alone rel-L2 %.3e (bit-identical: %s)" % (err, torch.equal(a.x, b.x)))
        assert err <= TOL
    if graphs:
        assert B.replays == 3
    B.close()


def test_batch_jobs_join_and_leave(jobs):
    """A job leaves after one iteration and another joins: each job's
    iterate still matches the same number of iterations alone."""
    import torch
    from ct2b200.batch import EMBatch
    alone = _states(jobs)
    for s, n in zip(alone, (1, 3, 2)):
        for _ in range(n):
            s.iterate()
    st = _states(jobs)
    B = EMBatch(2, device=st[0].x.device)
    s0 = B.add(st[0])
    B.add(st[1])
    B.iterate()                      # job 0: 1, job 1: 1
    B.remove(s0)
    B.add(st[2])
    B.iterate()                      # job 1: 2, job 2: 1
    B.iterate()                      # job 1: 3, job 2: 2
    torch.cuda.synchronize()
    for a, b in zip(alone, st):
        assert rel_l2(b.x.cpu().numpy(), a.x.cpu().numpy()) <= TOL
    B.close()
