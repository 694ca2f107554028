"""The atomic-free voxel-driven backprojector (ct2_gather.cu) against the
FP32 oracle (the C restatement of emil_code/view_proj3D.f:1096-1370) and
against the ray-driven scatter it replaces, through the C ABI.

Tolerances: <= 1e-5 relative L2 against the oracle (the plain-form bar);
<= 2e-6 against the scatter (both are the projector's exact transpose, they
differ by summation order and by the hat form of the z weight); the
adjoint identity to 1e-6; bit-identical results run to run.
"""
import math

import numpy as np
import pytest

import oracle
import view_proj3D
from ct2b200 import _lib
from ct2b200 import workloads as W
from helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _bp(y, ind, scan, vol, kind=0):
    L = _lib.lib()
    _lib.check(L.ct2_set_backprojector(kind), "ct2_set_backprojector")
    try:
        return view_proj3D.sinobackproject_linear(y, ind, scan.frame_vectors, *scan.view,
                                                  *vol.grid)
    finally:
        L.ct2_set_backprojector(0)


@pytest.fixture(scope="module")
def c0(cuda):
    vol, scan, ells = W.config0()
    rng = np.random.default_rng(7)
    y = rng.random(scan.shape).astype(np.float32)
    ind = (rng.random(scan.shape) > 0.1).astype(np.int32)
    return vol, scan, y, ind


def test_gather_matches_oracle_and_scatter(c0):
    vol, scan, y, ind = c0
    g = _bp(y, ind, scan, vol, 0)
    s = _bp(y, ind, scan, vol, 1)
    ref = oracle.view_proj3D.sinobackproject_linear(y, ind, scan.frame_vectors, *scan.view,
                                                    *vol.grid)
    assert rel_l2(g, ref) <= TOL
    assert rel_l2(g, s) <= 2e-6


def test_gather_is_bit_reproducible(c0):
    vol, scan, y, ind = c0
    a = _bp(y, ind, scan, vol, 0)
    b = _bp(y, ind, scan, vol, 0)
    assert np.array_equal(a, b)


def test_gather_device_path(c0):
    """One device call (a single backprojection over all views) equals the
    host call (views pipelined in blocks into one volume) to rounding."""
    import torch
    vol, scan, y, ind = c0
    host = _bp(y, ind, scan, vol, 0)
    dev = view_proj3D.sinobackproject_linear(torch.tensor(y).cuda(), torch.tensor(ind).cuda(),
                                             torch.tensor(scan.frame_vectors).cuda(), *scan.view,
                                             *vol.grid)
    assert rel_l2(dev.cpu().numpy(), host) <= 1e-6


def test_gather_adjoint_identity(c0):
    vol, scan, _, ind = c0
    x = W.voxelize(vol, W.config0()[2])
    rng = np.random.default_rng(8)
    y = rng.standard_normal(scan.shape).astype(np.float32)
    Ax = view_proj3D.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    Aty = _bp(y, ind, scan, vol, 0)
    lhs = np.dot(Ax.astype(np.float64).ravel(), y.astype(np.float64).ravel())
    rhs = np.dot(x.astype(np.float64).ravel(), Aty.astype(np.float64).ravel())
    assert abs(lhs - rhs) <= 1e-6 * max(abs(lhs), abs(rhs))


def test_gather_with_z_driven_rays(cuda):
    """A close source and a tall detector: the top and bottom rows are
    z-driven, which the gather leaves to the ray-driven scatter."""
    vol = W.Volume.centered((20, 22, 18), (2.0, 1.8, 2.2))
    scan = W.circular_scan(8, 24, 40, 4.0, 6.0, 50.0, 100.0, s0=0.4)
    rng = np.random.default_rng(9)
    y = rng.random(scan.shape).astype(np.float32)
    ind = np.ones(scan.shape, np.int32)
    g = _bp(y, ind, scan, vol, 0)
    ref = oracle.view_proj3D.sinobackproject_linear(y, ind, scan.frame_vectors, *scan.view,
                                                    *vol.grid)
    assert rel_l2(g, ref) <= TOL
    # the case does have z-driven rays
    f = scan.frame_vectors.astype(np.float64)
    v = scan.v0 + (scan.nv - 0.5) * scan.dv
    b = f[0, 6:9] + f[0, 12:15] * v
    d = np.abs(b - f[0, 0:3]) / np.array(vol.grid[:3])
    assert d[2] > max(d[0], d[1])


def test_gather_mixed_views(cuda):
    """Views whose detector is turned (v axis not along z) are scattered;
    the others are gathered; the sum matches the oracle."""
    vol = W.Volume.centered((24, 24, 20), (1.5, 1.5, 1.5))
    scan = W.circular_scan(9, 30, 28, 2.0, 2.0, 80.0, 160.0, s0=0.1)
    fv = scan.frame_vectors.astype(np.float64)
    for s in (2, 5):
        c, sn = math.cos(0.3), math.sin(0.3)
        eu, ev = fv[s, 9:12].copy(), fv[s, 12:15].copy()
        fv[s, 9:12], fv[s, 12:15] = c * eu + sn * ev, -sn * eu + c * ev
    scan.frame_vectors = fv.astype(np.float32)
    rng = np.random.default_rng(10)
    y = rng.random(scan.shape).astype(np.float32)
    ind = np.ones(scan.shape, np.int32)
    g = _bp(y, ind, scan, vol, 0)
    ref = oracle.view_proj3D.sinobackproject_linear(y, ind, scan.frame_vectors, *scan.view,
                                                    *vol.grid)
    assert rel_l2(g, ref) <= TOL


def test_gather_across_view_blocks(cuda):
    """A detector large enough that the ray table is built in several view
    blocks, each adding its views to the volume.  Every voxel sums ~5e4 FP32
    terms here, so the gather and the scatter (different summation orders)
    are both held to the FP64 oracle instead of to each other."""
    vol = W.Volume.centered((24, 20, 28), (2.0, 2.0, 2.0))
    scan = W.circular_scan(30, 1024, 1024, 0.1, 0.1, 300.0, 600.0)
    rng = np.random.default_rng(11)
    y = rng.random(scan.shape).astype(np.float32)
    ind = np.ones(scan.shape, np.int32)
    g = _bp(y, ind, scan, vol, 0)
    s = _bp(y, ind, scan, vol, 1)
    ref = oracle.view_proj3D_f64.sinobackproject_linear_omp(
        y, ind, scan.frame_vectors, *scan.view, *vol.grid, oracle.max_threads())
    assert rel_l2(g, ref) <= TOL
    assert rel_l2(s, ref) <= TOL
    assert np.array_equal(g, _bp(y, ind, scan, vol, 0))


def test_gather_em_step(c0):
    """MLEM accumulates A^T ratio and A^T 1 with the gather: one step matches
    the oracle and the scatter form."""
    vol, scan, _, ind = c0
    x = W.voxelize(vol, W.config0()[2]) + 0.1
    y = oracle.view_proj3D.sinoproj_linear(ind, scan.frame_vectors, *scan.view,
                                           x.astype(np.float32), *vol.grid)
    x0 = np.full(vol.shape, 0.5, np.float32)
    L = _lib.lib()
    got = view_proj3D.emstep_linear(y, ind, scan.frame_vectors, *scan.view, x0, *vol.grid)
    _lib.check(L.ct2_set_backprojector(1), "ct2_set_backprojector")
    try:
        sc = view_proj3D.emstep_linear(y, ind, scan.frame_vectors, *scan.view, x0, *vol.grid)
    finally:
        L.ct2_set_backprojector(0)
    ref = oracle.view_proj3D.emstep_linear(y, ind, scan.frame_vectors, *scan.view, x0, *vol.grid)
    assert rel_l2(got, ref) <= TOL
    assert rel_l2(got, sc) <= 2e-6


def test_gather_interior_tiles(cuda):
    """A volume tall and wide enough that some tiles lie two cells inside
    every face (the kernel then takes every sample without testing its
    valid interval): relative L2 against the FP64 oracle, and the largest
    single-voxel difference from the scatter, which tests every sample
    against its interval -- a sample taken outside it would add a term of
    full weight to one voxel (~1e-2 of the largest here)."""
    vol = W.Volume.centered((36, 44, 200), (1.0, 1.0, 0.5))
    scan = W.circular_scan(12, 72, 240, 1.2, 0.8, 200.0, 400.0, s0=0.2)
    rng = np.random.default_rng(12)
    y = rng.random(scan.shape).astype(np.float32)
    ind = np.ones(scan.shape, np.int32)
    g = _bp(y, ind, scan, vol, 0)
    s = _bp(y, ind, scan, vol, 1)
    ref = oracle.view_proj3D_f64.sinobackproject_linear_omp(
        y, ind, scan.frame_vectors, *scan.view, *vol.grid, oracle.max_threads())
    assert rel_l2(g, ref) <= TOL
    assert np.abs(g - s).max() <= 2e-6 * np.abs(s).max()
    assert np.array_equal(g, _bp(y, ind, scan, vol, 0))
