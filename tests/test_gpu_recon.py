"""The fused device-resident MLEM+TV iteration (ct2b200.recon.EMTVState:
projector with the ratio epilogue, matched backprojector, the FP64-normed
update and TV step in four passes) against the same iteration written as
separate tensor operations (the projection stored, the ratio, update, norms
and TV step each a pass), and against the oracle.

Tolerances: within 1e-6 relative L2 of the unfused form after 3 iterations
(they differ only in the rounding of the TV step's scale); the EM update
itself (tv_weight 0) within 1e-5 of the oracle's emstep_linear.
"""
import numpy as np
import pytest

import oracle
from helpers import rel_l2, small_circular

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(cuda):
    import torch
    from ct2b200.autograd import ConeGeometry
    vol, scan, x = small_circular(n=24, ns=16, nd=32)
    y = oracle.view_proj3D.sinoproj_linear(np.ones(scan.shape, np.int32), scan.frame_vectors,
                                           *scan.view, x, *vol.grid)
    y = np.maximum(y + 0.02 * np.random.default_rng(1).standard_normal(y.shape), 0)
    geom = ConeGeometry.from_scan(scan, vol, cuda)
    return vol, scan, geom, torch.tensor(y.astype(np.float32), device=cuda), torch


def test_fused_iteration_matches_unfused(case):
    vol, scan, geom, y, torch = case
    from ct2b200.recon import EMTVState
    x0 = torch.full(vol.shape, 0.5, device="cuda")
    a = EMTVState(x0.clone(), y, geom, tv_weight=0.002)
    b = EMTVState(x0.clone(), y, geom, tv_weight=0.002)
    for _ in range(3):
        a.iterate()
        b.iterate_unfused()
    torch.cuda.synchronize()
    assert rel_l2(a.x.cpu().numpy(), b.x.cpu().numpy()) <= 1e-6


def test_fused_graph_replay_matches_eager(case):
    vol, scan, geom, y, torch = case
    from ct2b200.recon import EMTVState
    x0 = torch.full(vol.shape, 0.5, device="cuda")
    a = EMTVState(x0.clone(), y, geom)
    b = EMTVState(x0.clone(), y, geom)
    for i in range(4):
        a.iterate()
        if i == 0:
            b.iterate()
        else:
            b.graph_iterate()
    torch.cuda.synchronize()
    assert torch.equal(a.x, b.x)


def test_fused_em_update_matches_oracle(case):
    vol, scan, geom, y, torch = case
    from ct2b200.recon import EMTVState
    x0 = np.full(vol.shape, 0.5, np.float32)
    st = EMTVState(torch.tensor(x0, device="cuda"), y, geom, tv_weight=0.0)
    st.iterate()
    ref = oracle.view_proj3D.emstep_linear(y.cpu().numpy(), np.ones(scan.shape, np.int32),
                                           scan.frame_vectors, *scan.view, x0, *vol.grid)
    assert rel_l2(st.x.cpu().numpy(), ref) <= 1e-5
