"""The precision form (BF16 volume / FP16 sinogram storage, FP64 per-ray
setup, FP32 Kahan ray sums, FP64 EM+TV norms) against the FP64 oracle.

Bars: with FP32 storage the kernels' arithmetic alone is measured, and must
meet the plain form's bars (projections and backprojections <= 1e-5
relative L2 vs FP64, reconstructions <= 1e-4, adjoint to 1e-6).  With
BF16/FP16 storage the error is dominated by the storage rounding (BF16
keeps 8 significant bits: about 1.5e-3 relative RMS per voxel), so each
result is reported and bounded by a small multiple of that floor.
"""
import numpy as np
import pytest

import oracle
from ct2b200 import workloads as W
from helpers import rel_l2, small_tomo

pytestmark = pytest.mark.gpu

F32_TOL = 1e-5
RECON_TOL = 1e-4


@pytest.fixture(scope="module")
def c0(cuda):
    import torch
    from ct2b200.autograd import ConeGeometry
    vol, scan, ells = W.config0()
    x = W.voxelize(vol, ells)
    return vol, scan, x, ConeGeometry.from_scan(scan, vol, "cuda"), torch


def _dot(a, b):
    return float(np.dot(np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()))


@pytest.mark.parametrize("storage,tol", [("f32", F32_TOL), ("bf16", 1e-3)])
def test_project_vs_fp64_oracle(c0, storage, tol):
    from ct2b200 import precision as P
    vol, scan, x, geom, torch = c0
    vdt, sdt = P.STORAGE[storage]
    got = P.project(torch.tensor(x, device="cuda").to(vdt), geom)
    assert got.dtype == sdt
    ind = np.ones(scan.shape, np.int32)
    ref = oracle.view_proj3D_f64.sinoproj_linear(ind, scan.frame_vectors, *scan.view,
                                                  x.astype(np.float64), *vol.grid)
    err = rel_l2(got.float().cpu().numpy(), ref)
    print("precision projector (%s storage) rel-L2 vs FP64 oracle: %.3e" % (storage, err))
    assert err <= tol


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_backproject_vs_fp64_oracle(c0, storage):
    """The data are exactly representable in the storage type, so the
    backprojection error is the arithmetic's alone in both storages."""
    from ct2b200 import precision as P
    vol, scan, x, geom, torch = c0
    _, sdt = P.STORAGE[storage]
    rng = np.random.default_rng(4)
    y = torch.tensor(rng.random(scan.shape, np.float32), device="cuda").to(sdt)
    ind = np.ones(scan.shape, np.int32)
    ind[rng.random(scan.shape) < 0.1] = 0
    ind_t = torch.tensor(ind, device="cuda")
    got = P.back_project(y, geom, ind=ind_t).cpu().numpy()
    ref = oracle.view_proj3D_f64.sinobackproject_linear(
        y.double().cpu().numpy(), ind, scan.frame_vectors, *scan.view, *vol.grid)
    err = rel_l2(got, ref)
    print("precision backprojector (%s storage) rel-L2 vs FP64 oracle: %.3e" % (storage, err))
    assert err <= F32_TOL


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_backproject_gather_matches_scatter(c0, storage):
    """The precision backprojector's atomic-free gather (the default for the
    circular cone beam) against its ray-driven scatter on the same FP16 /
    FP32 data, A^T 1 included, and bit-identical run to run."""
    from ct2b200 import _lib
    from ct2b200 import precision as P
    vol, scan, x, geom, torch = c0
    _, sdt = P.STORAGE[storage]
    rng = np.random.default_rng(6)
    y = torch.tensor(rng.random(scan.shape, np.float32), device="cuda").to(sdt)
    L = _lib.lib()
    ones_g = torch.empty(vol.shape, device="cuda")
    g = P.back_project(y, geom, ones_out=ones_g)
    g2 = P.back_project(y, geom)
    _lib.check(L.ct2_set_backprojector(1), "ct2_set_backprojector")
    try:
        ones_s = torch.empty(vol.shape, device="cuda")
        s = P.back_project(y, geom, ones_out=ones_s)
    finally:
        L.ct2_set_backprojector(0)
    assert rel_l2(g.cpu().numpy(), s.cpu().numpy()) <= 2e-6
    assert rel_l2(ones_g.cpu().numpy(), ones_s.cpu().numpy()) <= 2e-6
    assert torch.equal(g, g2)


def test_adjoint_identity(c0):
    from ct2b200 import precision as P
    vol, scan, x, geom, torch = c0
    rng = np.random.default_rng(5)
    xt = torch.tensor(rng.random(vol.shape, np.float32), device="cuda")
    yt = torch.tensor(rng.random(scan.shape, np.float32), device="cuda")
    lhs = _dot(P.project(xt, geom).cpu(), yt.cpu())
    rhs = _dot(xt.cpu(), P.back_project(yt, geom).cpu())
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


def test_bf16_path_is_the_f32_path_on_the_same_values(c0):
    """Loading BF16 / storing FP16 changes nothing but the storage rounding."""
    from ct2b200 import precision as P
    vol, scan, x, geom, torch = c0
    xb = torch.tensor(x, device="cuda").to(torch.bfloat16)
    a = P.project(xb, geom).float()
    b = P.project(xb.float(), geom)
    # FP16 rounding of b: at most half an ulp, 2^-11 relative (normal range)
    bound = torch.clamp(b.abs() * 2.0 ** -11, min=2.0 ** -25) * 1.0001
    assert bool(torch.all((a - b).abs() <= bound))


def test_z_driven_vs_fp64_oracle(cuda):
    import torch
    from ct2b200 import precision as P
    from ct2b200.autograd import ConeGeometry
    vol, scan, x = small_tomo()
    geom = ConeGeometry.from_scan(scan, vol, "cuda")
    got = P.project(torch.tensor(x, device="cuda"), geom, z_driven=True).cpu().numpy()
    ind = np.ones(scan.shape, np.int32)
    ref = oracle.view_proj3D_tomo_f64.sinoprojz(ind, scan.frame_vectors, *scan.view,
                                                 x.astype(np.float64), *vol.grid)
    assert rel_l2(got, ref) <= F32_TOL


def _fp64_emtv(y, scan, vol, iterations, w):
    vp, tv = oracle.view_proj3D_f64, oracle.totalvar_f64
    ind = np.ones(scan.shape, np.int32)
    x = np.full(vol.shape, 0.5)
    for _ in range(iterations):
        xe = vp.emstep_linear(y, ind, scan.frame_vectors, *scan.view, x, *vol.grid)
        dn = float(np.linalg.norm(xe - x))
        g, _ = tv.total_var_grad3d(0.0, xe, *vol.shape, 1)
        x = np.maximum(xe - w * dn * g, 0.0)
    return x


@pytest.fixture(scope="module")
def emtv_case(cuda):
    import torch
    from ct2b200.autograd import ConeGeometry
    from ct2b200.serving import JobSpec, simulate_measurement
    spec = JobSpec(7, "emtv", 32, 30, 48, 10, seed=21, iterations=4)
    vol, scan, geom, truth, y = simulate_measurement(spec, "cuda")
    # data exactly representable in FP16, so both storages see the same y
    y16 = y.half()
    ref = _fp64_emtv(y16.double().cpu().numpy(), scan, vol, spec.iterations, 0.002)
    return spec, vol, scan, geom, y16, ref, torch


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_emtv_vs_fp64_oracle(emtv_case, storage):
    from ct2b200 import precision as P
    spec, vol, scan, geom, y16, ref, torch = emtv_case
    job = P.EMTV(y16, geom, storage=storage)
    for _ in range(spec.iterations):
        job.iterate()
    got = job.x.float().cpu().numpy()
    err = rel_l2(got, ref)
    floor = rel_l2(torch.tensor(ref).to(torch.bfloat16).double().numpy(), ref)
    print("precision EM+TV (%s storage, %d its) rel-L2 vs FP64 oracle: %.3e "
          "(BF16 rounding of the FP64 result itself: %.3e)" % (storage, spec.iterations, err, floor))
    if storage == "f32":
        assert err <= RECON_TOL
    else:
        assert err <= 3.0 * floor


def test_emtv_graph_replay_matches_eager(emtv_case):
    from ct2b200 import precision as P
    spec, vol, scan, geom, y16, ref, torch = emtv_case
    eager = P.EMTV(y16, geom)
    graphed = P.EMTV(y16, geom)
    eager.iterate()
    graphed.iterate()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        graphed.iterate()  # captured, not run
    for _ in range(spec.iterations - 1):
        eager.iterate()
        g.replay()
    torch.cuda.synchronize()
    # the two differ only by the order of the backprojector's FP32 additions
    assert rel_l2(graphed.x.float().cpu().numpy(), eager.x.float().cpu().numpy()) <= 1e-3


# ---------------------------------------------------------------------------
# tomosynthesis: colour-ordered ART sweeps (+TV) against the FP64 oracle run
# in the same ray order
# ---------------------------------------------------------------------------

@pytest.fixture(scope="module")
def tomo_case(cuda):
    import torch
    from ct2b200.autograd import ConeGeometry
    from ct2b200 import precision as P
    vol, scan, x = small_tomo()
    geom = ConeGeometry.from_scan(scan, vol, "cuda")
    ind = np.ones(scan.shape, np.int32)
    y = oracle.view_proj3D_tomo_f64.sinoprojz(ind, scan.frame_vectors, *scan.view,
                                              x.astype(np.float64), *vol.grid)
    y16 = torch.tensor(y, device="cuda").half()  # FP16-representable data for both storages
    col = P.art_colouring(geom)
    return vol, scan, geom, ind, y16, col, torch


def test_art_sweep_vs_fp64_oracle(tomo_case):
    from helpers import coloured_art_fp64
    from ct2b200 import precision as P
    vol, scan, geom, ind, y16, col, torch = tomo_case
    x = torch.zeros(vol.shape, device="cuda")
    P.art_sweep(x, y16.float(), geom, col, reg_fac=0.7)
    ref = coloured_art_fp64(np.zeros(vol.shape), y16.double().cpu().numpy(), ind, scan, vol, col,
                            0.7)
    err = rel_l2(x.cpu().numpy(), ref)
    print("colour-ordered ART sweep (f32 storage) rel-L2 vs FP64 oracle: %.3e" % err)
    assert err <= RECON_TOL
    # the z-major layout runs the same arithmetic on the transposed array
    xz = torch.zeros(tuple(reversed(vol.shape)), device="cuda")
    P.art_sweep(xz, y16.float(), geom, col, reg_fac=0.7, zmajor=True)
    assert torch.equal(xz.permute(2, 1, 0), x)


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_art_tv_vs_fp64_oracle(tomo_case, storage):
    from helpers import coloured_art_fp64, tv_step_fp64
    from ct2b200 import precision as P
    vol, scan, geom, ind, y16, col, torch = tomo_case
    its = 4
    job = P.ARTTV(y16, geom, storage=storage, reg_fac=0.7)
    for _ in range(its):
        job.iterate()
    got = job.result().float().cpu().numpy()
    x = np.zeros(vol.shape)
    y = y16.double().cpu().numpy()
    for _ in range(its):
        prev = x
        x = coloured_art_fp64(x, y, ind, scan, vol, col, 0.7)
        x = tv_step_fp64(x, prev, 0.002)
    err = rel_l2(got, x)
    floor = rel_l2(torch.tensor(x).to(torch.bfloat16).double().numpy(), x)
    print("ART+TV (%s storage, %d its) rel-L2 vs FP64 oracle: %.3e (BF16 rounding of the FP64 "
          "result itself: %.3e)" % (storage, its, err, floor))
    if storage == "f32":
        assert err <= RECON_TOL
    elif storage == "f16":
        assert err <= 2e-3
    else:
        assert err <= 10.0 * floor


@pytest.mark.parametrize("turn", [0.0, 0.3])
def test_backproject_turned_detector_and_odd_rows(cuda, turn):
    """The backprojector walks detector-adjacent ray pairs together when they
    share the q model; a detector turned about its normal breaks that for
    every pair (each ray then walks alone), and an odd number of rows leaves
    the last thread of a column one ray.  FP32 storage: the arithmetic
    against the FP64 oracle at the plain form's bar, and the adjoint."""
    import math
    import torch
    from ct2b200 import precision as P
    from ct2b200.autograd import ConeGeometry
    from helpers import small_circular
    vol, scan, x = small_circular(n=22, ns=8, nd=20)
    scan = W.Scan(scan.ns, scan.nu, 25, scan.du, scan.dv, scan.u0, -25 * scan.dv / 2,
                  scan.frame_vectors)
    fv = scan.frame_vectors.copy()
    if turn:
        c, s = math.cos(turn), math.sin(turn)
        u, v = fv[:, 9:12].copy(), fv[:, 12:15].copy()
        fv[:, 9:12] = c * u - s * v
        fv[:, 12:15] = s * u + c * v
    scan = W.Scan(scan.ns, scan.nu, scan.nv, scan.du, scan.dv, scan.u0, scan.v0,
                  fv.astype(np.float32))
    geom = ConeGeometry.from_scan(scan, vol, "cuda")
    rng = np.random.default_rng(7)
    y = rng.random(scan.shape, np.float32)
    got = P.back_project(torch.tensor(y, device="cuda"), geom).cpu().numpy()
    ind = np.ones(scan.shape, np.int32)
    ref = oracle.view_proj3D_f64.sinobackproject_linear(y.astype(np.float64), ind,
                                                        scan.frame_vectors, *scan.view, *vol.grid)
    assert np.abs(ref).max() > 0
    assert rel_l2(got, ref) <= F32_TOL, rel_l2(got, ref)
    xt = torch.tensor(x, device="cuda")
    lhs = _dot(P.project(xt, geom).cpu(), y)
    rhs = _dot(x, got)
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
