"""The differentiable form: the projector's backward is the matched
backprojector, the data-fit term projects again in its backward (or, on
request, keeps the residual from the forward), the TV term's backward is the
TV-gradient kernel.  Checked by the dot-product
test, central finite differences (step 1e-3 on 64 random voxels) and the
FP64 oracle gradient."""
import numpy as np
import pytest

import oracle
from helpers import small_circular

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(cuda):
    import torch
    from ct2b200.autograd import ConeGeometry
    vol, scan, x = small_circular(n=20, ns=12, nd=28)
    geom = ConeGeometry.from_scan(scan, vol, cuda)
    rng = np.random.default_rng(0)
    y = oracle.view_proj3D.sinoproj_linear(np.ones(scan.shape, np.int32), scan.frame_vectors,
                                           *scan.view, x, *vol.grid)
    y = (y + 0.05 * rng.standard_normal(y.shape)).astype(np.float32)
    x_eval = (0.5 * x + 0.2 * rng.random(x.shape)).astype(np.float32)
    return vol, scan, geom, x_eval, y, torch


def test_projector_backward_is_adjoint(setup):
    vol, scan, geom, x, y, torch = setup
    from ct2b200.autograd import project
    xt = torch.tensor(x, device="cuda", requires_grad=True)
    yt = torch.tensor(y, device="cuda")
    p = project(xt, geom)
    (p * yt).sum().backward()
    lhs = float(torch.sum(p.detach().double() * yt.double()))
    rhs = float(torch.sum(xt.detach().double() * xt.grad.double()))
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


def _loss(x, y, geom, torch):
    from ct2b200.autograd import data_fit, total_variation
    return data_fit(x, y, geom).double() + 0.01 * total_variation(x, 0.0).double()


def test_finite_differences_on_64_voxels(setup):
    vol, scan, geom, x, y, torch = setup
    xt = torch.tensor(x, device="cuda", requires_grad=True)
    yt = torch.tensor(y, device="cuda")
    _loss(xt, yt, geom, torch).backward()
    g = xt.grad.cpu().numpy()
    rng = np.random.default_rng(1)
    idx = [tuple(rng.integers(2, s - 2) for s in x.shape) for _ in range(64)]
    h = 1e-3
    bad = 0
    for i in idx:
        xp = torch.tensor(x, device="cuda")
        xm = torch.tensor(x, device="cuda")
        xp[i] += h
        xm[i] -= h
        with torch.no_grad():
            fd = (float(_loss(xp, yt, geom, torch)) - float(_loss(xm, yt, geom, torch))) / (2 * h)
        if abs(fd - g[i]) > 1e-2 * max(abs(g[i]), 1.0):
            bad += 1
    assert bad == 0


def test_gradient_matches_fp64_oracle(setup):
    vol, scan, geom, x, y, torch = setup
    xt = torch.tensor(x, device="cuda", requires_grad=True)
    yt = torch.tensor(y, device="cuda")
    _loss(xt, yt, geom, torch).backward()
    g = xt.grad.cpu().numpy().astype(np.float64)
    ind = np.ones(scan.shape, np.int32)
    vp = oracle.view_proj3D_f64
    r = vp.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x.astype(np.float64),
                           *vol.grid) - y
    gd = 2.0 * vp.sinobackproject_linear(r, ind, scan.frame_vectors, *scan.view, *vol.grid)
    gt, _ = oracle.totalvar_f64.total_var_grad3d(0.0, x.astype(np.float64), *vol.shape, 0)
    ref = gd + 0.01 * gt
    err = np.linalg.norm(g - ref) / np.linalg.norm(ref)
    assert err <= 1e-4, err


def test_adam_on_batch_reduces_loss(setup):
    vol, scan, geom, x, y, torch = setup
    from ct2b200.autograd import data_fit, total_variation
    yb = torch.tensor(np.stack([y, y]), device="cuda")
    xb = torch.zeros((2,) + vol.shape, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([xb], lr=1e-2)
    losses = []
    for _ in range(20):
        opt.zero_grad()
        loss = data_fit(xb, yb, geom) + 0.01 * total_variation(xb, 0.0)
        loss.backward()
        opt.step()
        losses.append(loss.item())
    assert losses[-1] < 0.5 * losses[0]


def test_data_fit_kept_and_recomputed_residual_agree(setup):
    """The residual kept from the forward and the one projected again in the
    backward (on autograd's worker thread) are the same deterministic
    projection, and the gather backprojector sums in a fixed order (every
    view of this circular scan is in its family and no ray is z-driven, so
    none goes to the scatter): equal losses and equal gradients, bit for
    bit."""
    vol, scan, geom, x, y, torch = setup
    from ct2b200.autograd import data_fit
    yb = torch.tensor(np.stack([y, y * 0.5]), device="cuda")
    grads = []
    for keep in (True, False):
        xb = torch.tensor(np.stack([x, x * 0.25]), device="cuda", requires_grad=True)
        loss = data_fit(xb, yb, geom, keep_residual=keep)
        loss.backward()
        grads.append((loss.item(), xb.grad.cpu().numpy()))
    assert grads[0][0] == grads[1][0]
    # the residual the backward projects again is the forward's bit for bit
    from ct2b200.autograd import forward_project
    xd = torch.tensor(x, device="cuda")
    yd = torch.tensor(y, device="cuda")
    r1 = forward_project(xd, geom) - yd
    r2 = forward_project(xd, geom) - yd
    assert torch.equal(r1, r2)
    g0, g1 = grads[0][1], grads[1][1]
    assert np.array_equal(g0, g1)
