"""Several volumes through one geometry (ct2_dev_view_proj3D_sinoproj_linear_many
/ _sinobackproject_linear_many, ct2b200.autograd.forward_project_many /
back_project_many): every volume's result equals its own single-volume call
bit for bit -- the same kernels' code over all volumes' work items -- for
volumes that admit the TMA-staged projector and volumes that do not, for a
detector whose gather table takes several view blocks, and with the scatter
backprojector selected (tolerance there: its L2 reductions sum in no fixed
order); the batched data-fit gradient equals the per-volume gradients; and a
fresh host thread's first projection takes the same (TMA-staged) path.
"""
import pytest

from ct2b200 import _lib
from ct2b200 import workloads as W
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _case(shape, scan, device, count=3, seed=5):
    import torch
    from ct2b200.autograd import ConeGeometry
    vol = W.Volume.centered(shape, (1.0, 1.0, 1.0))
    geom = ConeGeometry.from_scan(scan, vol, device)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    xs = torch.rand((count,) + tuple(shape), generator=g, device=device)
    ys = torch.rand((count,) + tuple(geom.sino_shape), generator=g, device=device)
    return geom, xs, ys


CASES = {
    "tma": ((24, 28, 32), lambda: W.circular_scan(14, 40, 44, 1.2, 1.1, 120.0, 240.0, s0=0.3)),
    "untiled": ((25, 22, 19), lambda: W.circular_scan(11, 36, 30, 1.3, 1.2, 110.0, 220.0)),
    "blocks": ((20, 18, 24), lambda: W.circular_scan(30, 1024, 1024, 0.05, 0.05, 300.0, 600.0)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_many_equals_single_calls(cuda, name):
    import torch
    from ct2b200.autograd import (back_project, back_project_many, forward_project,
                                  forward_project_many)
    shape, scan = CASES[name]
    geom, xs, ys = _case(shape, scan(), cuda)
    p = forward_project_many(xs, geom)
    b = back_project_many(ys, geom)
    for i in range(xs.shape[0]):
        assert torch.equal(p[i], forward_project(xs[i], geom)), i
        assert torch.equal(b[i], back_project(ys[i], geom)), i


def test_many_with_the_scatter(cuda):
    import torch
    from ct2b200.autograd import back_project, back_project_many
    shape, scan = CASES["tma"]
    geom, xs, ys = _case(shape, scan(), cuda)
    L = _lib.lib()
    _lib.check(L.ct2_set_backprojector(1), "ct2_set_backprojector")
    try:
        b = back_project_many(ys, geom)
        single = [back_project(ys[i], geom) for i in range(ys.shape[0])]
    finally:
        L.ct2_set_backprojector(0)
    torch.cuda.synchronize()
    for i in range(ys.shape[0]):
        assert rel_l2(b[i].cpu().numpy(), single[i].cpu().numpy()) <= 1e-6


def test_batched_data_fit_gradient(cuda):
    import torch
    from ct2b200.autograd import data_fit
    shape, scan = CASES["tma"]
    geom, xs, ys = _case(shape, scan(), cuda, count=2)
    x = xs.clone().requires_grad_(True)
    data_fit(x, ys, geom).backward()
    for i in range(2):
        xi = xs[i].clone().requires_grad_(True)
        data_fit(xi, ys[i], geom).backward()
        assert torch.equal(x.grad[i], xi.grad), i


def test_projector_first_call_on_a_new_thread(cuda):
    """A host thread whose first CUDA work is the projector (autograd's
    worker thread, a serving thread) takes the TMA-staged form like any
    other thread: the result equals the main thread's bit for bit."""
    import threading
    import torch
    from ct2b200.autograd import forward_project, forward_project_many
    shape, scan = CASES["tma"]
    geom, xs, _ = _case(shape, scan(), cuda, count=2)
    want_one = forward_project(xs[0], geom)
    want_many = forward_project_many(xs, geom)
    torch.cuda.synchronize()
    got = {}

    def worker(fn, arg, key):
        got[key] = fn(arg, geom)
        torch.cuda.synchronize()

    for key, fn, arg in (("one", forward_project, xs[0]), ("many", forward_project_many, xs)):
        t = threading.Thread(target=worker, args=(fn, arg, key))
        t.start()
        t.join()
    assert torch.equal(got["one"], want_one)
    assert torch.equal(got["many"], want_many)
