"""GPU parity of the projectors, matched backprojectors and MLEM steps
against the FP32 oracle (the C restatement of emil_code/view_proj3D.f,
view_proj3D_tomo.f and ray_proj3D.f), through the C ABI.

Tolerances: projections and single backprojections <= 1e-5 relative L2 (the
plain-form bar for projections); reconstructions after the stated iteration
count <= 1e-4; the adjoint identity <Ax, y> = <x, A^T y> to 1e-6 with FP64
dot products.
"""
import numpy as np
import pytest

import oracle
import ray_proj3D
import view_proj3D
import view_proj3D_tomo
from ct2b200 import workloads as W
from helpers import rel_l2, ray_list_from_scan, small_circular, small_tomo

pytestmark = pytest.mark.gpu

PROJ_TOL = 1e-5
RECON_TOL = 1e-4


@pytest.fixture(scope="module")
def c0(cuda):
    vol, scan, ells = W.config0()
    x = W.voxelize(vol, ells)
    return vol, scan, x


def _ind(scan, frac_off=0.0, seed=0):
    ind = np.ones(scan.shape, np.int32)
    if frac_off:
        rng = np.random.default_rng(seed)
        ind[rng.random(scan.shape) < frac_off] = 0
    return ind


@pytest.mark.parametrize("kind", ["linear", "nearest"])
def test_projector_c0(c0, kind):
    vol, scan, x = c0
    ind = _ind(scan)
    got = getattr(view_proj3D, "sinoproj_" + kind)(ind, scan.frame_vectors, *scan.view, x,
                                                   *vol.grid)
    ref = getattr(oracle.view_proj3D, "sinoproj_" + kind)(ind, scan.frame_vectors, *scan.view, x,
                                                          *vol.grid)
    assert got.shape == (scan.ns, scan.nu, scan.nv) and got.dtype == np.float32
    assert rel_l2(got, ref) <= PROJ_TOL


@pytest.mark.parametrize("kind", ["linear", "nearest"])
def test_backprojector_c0(c0, kind):
    vol, scan, x = c0
    ind = _ind(scan, 0.1)
    rng = np.random.default_rng(1)
    y = rng.random(scan.shape).astype(np.float32)
    got = getattr(view_proj3D, "sinobackproject_" + kind)(y, ind, scan.frame_vectors, *scan.view,
                                                          *vol.grid)
    ref = getattr(oracle.view_proj3D, "sinobackproject_" + kind)(y, ind, scan.frame_vectors,
                                                                 *scan.view, *vol.grid)
    assert got.shape == vol.shape
    assert rel_l2(got, ref) <= PROJ_TOL


@pytest.mark.parametrize("kind", ["linear", "nearest"])
def test_adjoint_identity(c0, kind):
    vol, scan, x = c0
    ind = _ind(scan)
    rng = np.random.default_rng(2)
    y = rng.standard_normal(scan.shape).astype(np.float32)
    Ax = getattr(view_proj3D, "sinoproj_" + kind)(ind, scan.frame_vectors, *scan.view, x,
                                                  *vol.grid)
    Aty = getattr(view_proj3D, "sinobackproject_" + kind)(y, ind, scan.frame_vectors, *scan.view,
                                                          *vol.grid)
    lhs = np.dot(Ax.astype(np.float64).ravel(), y.astype(np.float64).ravel())
    rhs = np.dot(x.astype(np.float64).ravel(), Aty.astype(np.float64).ravel())
    assert abs(lhs - rhs) <= 1e-6 * max(abs(lhs), abs(rhs))


def test_projector_masked_and_small_geometry(cuda):
    vol, scan, x = small_circular()
    ind = _ind(scan, 0.3, seed=4)
    got = view_proj3D.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    ref = oracle.view_proj3D.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    assert np.all(got[ind == 0] == 0)
    assert rel_l2(got, ref) <= PROJ_TOL


@pytest.mark.parametrize("kind,small", [("linear", 1e-5), ("nearest", 1e-8)])
def test_emstep_one_step(c0, kind, small):
    vol, scan, x = c0
    ind = _ind(scan, 0.05, seed=3)
    y = oracle.view_proj3D.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    x0 = np.full(vol.shape, 0.5, np.float32)
    got = getattr(view_proj3D, "emstep_" + kind)(y, ind, scan.frame_vectors, *scan.view, x0,
                                                 *vol.grid)
    ref = getattr(oracle.view_proj3D, "emstep_" + kind)(y, ind, scan.frame_vectors, *scan.view,
                                                        x0, *vol.grid)
    assert rel_l2(got, ref) <= PROJ_TOL
    assert np.array_equal(x0, np.full(vol.shape, 0.5, np.float32))  # input untouched


def test_em_ten_iterations_c0(c0):
    """Config 0's EM run: 10 iterations from a uniform 0.5 start on the
    noiseless analytic projections of the ellipsoid phantom (sum over
    ellipsoids of att * chord), clipped at 0 as EM requires."""
    vol, scan, _ = c0
    ells = W.config0()[2]
    ind = _ind(scan)
    y = np.maximum(W.analytic_projection(scan, ells).cpu().numpy(), 0)
    assert np.count_nonzero(y) > 0.3 * y.size
    g = np.full(vol.shape, 0.5, np.float32)
    r = g.copy()
    for _ in range(10):
        g = view_proj3D.emstep_linear(y, ind, scan.frame_vectors, *scan.view, g, *vol.grid)
        r = oracle.view_proj3D.emstep_linear(y, ind, scan.frame_vectors, *scan.view, r, *vol.grid)
    assert rel_l2(g, r) <= RECON_TOL


def test_device_path_matches_host_path(c0):
    import torch
    vol, scan, x = c0
    ind = _ind(scan, 0.1)
    host = view_proj3D.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    dev = view_proj3D.sinoproj_linear(torch.as_tensor(ind).cuda(),
                                      torch.as_tensor(scan.frame_vectors).cuda(), *scan.view,
                                      torch.as_tensor(x).cuda(), *vol.grid)
    assert dev.is_cuda
    assert np.array_equal(dev.cpu().numpy(), host)


def test_tomo_z_projector_and_em(cuda):
    vol, scan, x = small_tomo()
    ind = _ind(scan)
    got = view_proj3D_tomo.sinoprojz(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    ref = oracle.view_proj3D_tomo.sinoprojz(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    assert rel_l2(got, ref) <= PROJ_TOL
    x0 = np.full(vol.shape, 0.5, np.float32)
    g = view_proj3D_tomo.emstep_linearz(ref, ind, scan.frame_vectors, *scan.view, x0, *vol.grid)
    r = oracle.view_proj3D_tomo.emstep_linearz(ref, ind, scan.frame_vectors, *scan.view, x0,
                                               *vol.grid)
    assert rel_l2(g, r) <= PROJ_TOL


def test_ray_list_family(cuda):
    vol, scan, x = small_circular(n=20, ns=4, nd=24)
    rv = ray_list_from_scan(scan)
    nr = len(rv)
    ind = np.ones(nr, np.int32)
    ind[::7] = 0
    for kind in ("linear", "nearest"):
        got = getattr(ray_proj3D, "sinoproj_" + kind)(ind, rv, nr, x, *vol.grid)
        ref = getattr(oracle.ray_proj3D, "sinoproj_" + kind)(ind, rv, nr, x, *vol.grid)
        assert rel_l2(got, ref) <= PROJ_TOL, kind
    y = np.abs(np.random.default_rng(5).standard_normal(nr)).astype(np.float32)
    got = ray_proj3D.sinobackproject_nearest(y, ind, rv, nr, *vol.grid)
    ref = oracle.ray_proj3D.sinobackproject_nearest(y, ind, rv, nr, *vol.grid)
    assert rel_l2(got, ref) <= PROJ_TOL
    x0 = np.full(vol.shape, 0.5, np.float32)
    got = ray_proj3D.emstep_nearest(y, ind, rv, nr, x0, *vol.grid)
    ref = oracle.ray_proj3D.emstep_nearest(y, ind, rv, nr, x0, *vol.grid)
    assert rel_l2(got, ref) <= PROJ_TOL


def test_driving_axis_ties(cuda):
    """Rays with |dx| = |dy|, |dx| = |dz| or all three equal (isotropic
    voxels, exact in FP32): the reference breaks ties to the later axis
    (emil_code/view_proj3D.f:811,843); the kernels follow it, so ray sums,
    nearest backprojection and EM match the oracle on exactly tied rays."""
    vol = W.Volume.centered((24, 24, 24), (1.0, 1.0, 1.0))
    x = np.random.default_rng(8).random(vol.shape).astype(np.float32)
    rays = []
    for o in np.arange(-6.0, 6.5, 1.25):
        for dz in (-7.0, 0.0, 5.5):
            rays.append([-30.0, -30.0 + o, -dz / 2, 30.0, 30.0 + o, dz / 2])    # x ~ y
            rays.append([-30.0, -dz / 2, -30.0 + o, 30.0, dz / 2, 30.0 + o])    # x ~ z
            rays.append([-dz / 2, -30.0, -30.0 + o, dz / 2, 30.0, 30.0 + o])    # y ~ z
        rays.append([-30.0 + o, -30.0, -30.0, 30.0 + o, 30.0, 30.0])             # all three
        rays.append([30.0, -30.0 + o, 30.0, -30.0, 30.0 + o, -30.0])             # reversed
    rv = np.array(rays, np.float32)
    nr = len(rv)
    for kind in ("linear", "nearest"):
        got = getattr(ray_proj3D, "sinoproj_" + kind)(None, rv, nr, x, *vol.grid)
        ref = getattr(oracle.ray_proj3D, "sinoproj_" + kind)(None, rv, nr, x, *vol.grid)
        assert ref.min() > 0, kind  # every ray crosses the volume
        assert np.abs(got - ref).max() <= 1e-5 * ref.max(), kind
    y = np.random.default_rng(9).random(nr).astype(np.float32)
    got = ray_proj3D.sinobackproject_nearest(y, None, rv, nr, *vol.grid)
    ref = oracle.ray_proj3D.sinobackproject_nearest(y, None, rv, nr, *vol.grid)
    assert rel_l2(got, ref) <= PROJ_TOL
    x0 = np.full(vol.shape, 0.5, np.float32)
    got = ray_proj3D.emstep_nearest(y, None, rv, nr, x0, *vol.grid)
    ref = oracle.ray_proj3D.emstep_nearest(y, None, rv, nr, x0, *vol.grid)
    assert rel_l2(got, ref) <= PROJ_TOL


def test_shape_errors_raise_valueerror(cuda):
    vol, scan, x = small_circular()
    with pytest.raises(ValueError):
        view_proj3D.sinoproj_linear(None, scan.frame_vectors[:-1], *scan.view, x, *vol.grid)
    with pytest.raises(ValueError):
        view_proj3D.sinoproj_linear(None, scan.frame_vectors, *scan.view, x[:-1], *vol.grid)
    with pytest.raises(ValueError):
        g = list(vol.grid)
        g[0] = 0.0
        view_proj3D.sinoproj_linear(None, scan.frame_vectors, *scan.view, x, *g)


@pytest.mark.parametrize("n", [23, 24])
def test_backprojector_odd_and_even_volumes(cuda, n):
    """Volumes whose sizes are odd (n=23: nz = 21) and even (n=24: nz = 22)
    along the stride-1 axis, with a fifth of the rays masked: the
    backprojection against the oracle and the adjoint of the projector."""
    vol, scan, x = small_circular(n=n)
    ind = _ind(scan, 0.2, seed=9)
    y = np.random.default_rng(n).random(scan.shape).astype(np.float32)
    got = view_proj3D.sinobackproject_linear(y, ind, scan.frame_vectors, *scan.view, *vol.grid)
    ref = oracle.view_proj3D.sinobackproject_linear(y, ind, scan.frame_vectors, *scan.view,
                                                    *vol.grid)
    assert rel_l2(got, ref) <= PROJ_TOL
    Ax = view_proj3D.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    lhs = np.dot(Ax.astype(np.float64).ravel(), y.astype(np.float64).ravel())
    rhs = np.dot(x.astype(np.float64).ravel(), got.astype(np.float64).ravel())
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


def test_tma_staged_projector_equals_untiled_kernel(c0):
    """The TMA-staged projector (16-byte aligned volume, nz % 4 == 0) and the
    untiled kernel (the same volume one float off alignment) take the same
    samples with the same weights; only the grouping of the FP32 additions
    differs."""
    import torch
    from ct2b200.autograd import ConeGeometry, forward_project
    vol, scan, x = c0
    geom = ConeGeometry.from_scan(scan, vol, "cuda")
    aligned = torch.tensor(x, device="cuda")
    flat = torch.zeros(x.size + 4, device="cuda")
    shifted = flat[1:x.size + 1].view(vol.shape)  # 4-byte offset: no tensor map
    shifted.copy_(aligned)
    a = forward_project(aligned, geom)
    b = forward_project(shifted, geom)
    assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) <= 1e-6
    ref = oracle.view_proj3D.sinoproj_linear(np.ones(scan.shape, np.int32), scan.frame_vectors,
                                             *scan.view, x, *vol.grid)
    assert rel_l2(a.cpu().numpy(), ref) <= PROJ_TOL
    # no bounded wait on a staged chunk ran out
    import ctypes
    from ct2b200 import _lib
    n = ctypes.c_int(-1)
    _lib.check(_lib.lib().ct2_wait_timeouts(ctypes.addressof(n), 0), "ct2_wait_timeouts")
    assert n.value == 0


def test_bounded_wait_expires_with_etimeout(cuda):
    """The bounded device wait gives up and reports CT2_ETIMEOUT: a one-thread
    kernel waits, 1000 tries at most, on an mbarrier that nothing completes
    and that no copy targets.  The context stays usable and the projector's
    own timeout count is unchanged."""
    import ctypes
    from ct2b200 import _lib
    L = _lib.lib()
    n0, n1 = ctypes.c_int(-1), ctypes.c_int(-1)
    _lib.check(L.ct2_wait_timeouts(ctypes.addressof(n0), 0), "ct2_wait_timeouts")
    assert L.ct2_wait_selftest(1000) == _lib.CT2_ETIMEOUT
    assert "gave up" in _lib.last_error()
    vol, scan, x = small_circular()
    ind = _ind(scan)
    got = view_proj3D.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    ref = oracle.view_proj3D.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    assert rel_l2(got, ref) <= PROJ_TOL
    _lib.check(L.ct2_wait_timeouts(ctypes.addressof(n1), 0), "ct2_wait_timeouts")
    assert n1.value == n0.value
