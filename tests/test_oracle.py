"""The CPU oracle against the reference's own known answers and the
structural identities of its algorithms (no GPU needed).

Pins:
* single-ray ART identity, emil_code/tests/art_test.py:62-70;
* TV gradient vs central finite differences in FP64, emil_code/tests/tpvGrad.py:29-44;
* exact transpose of projector and backprojector (view_proj3D.f:703-1370);
* MLEM fixed point y = A x (view_proj3D.f:2507-2831);
* analytic chord of a sphere (view_proj3D.f:483-603);
* total_var3d of a constant volume is 0 (totalvar.f:35-62).
"""
import math

import numpy as np
import pytest

import oracle
from helpers import rel_l2, small_circular, ray_list_from_scan


@pytest.mark.parametrize("dt", ["f32", "f64"])
@pytest.mark.parametrize("kind", ["linear", "nearest"])
def test_oracle_adjoint(dt, kind):
    vp = oracle.view_proj3D if dt == "f32" else oracle.view_proj3D_f64
    vol, scan, x = small_circular()
    rng = np.random.default_rng(0)
    y = rng.standard_normal(scan.shape)
    ind = np.ones(scan.shape, np.int32)
    Ax = getattr(vp, "sinoproj_" + kind)(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    Aty = getattr(vp, "sinobackproject_" + kind)(y, ind, scan.frame_vectors, *scan.view, *vol.grid)
    lhs = np.dot(Ax.astype(np.float64).ravel(), y.astype(vp.dt).astype(np.float64).ravel())
    rhs = np.dot(x.astype(np.float64).ravel(), Aty.astype(np.float64).ravel())
    tol = 2e-6 if dt == "f32" else 1e-12
    assert abs(lhs - rhs) <= tol * max(abs(lhs), abs(rhs))


def test_oracle_f32_matches_f64():
    vol, scan, x = small_circular()
    ind = np.ones(scan.shape, np.int32)
    a = oracle.view_proj3D.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    b = oracle.view_proj3D_f64.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    assert rel_l2(a, b) < 2e-6


@pytest.mark.parametrize("kind", ["linear", "nearest"])
def test_single_ray_art_identity(kind):
    """emil_code/tests/art_test.py:62-70: after one ART step with only one ray
    enabled and reg_fac = 1, re-projecting that ray returns its datum."""
    vol, scan, x = small_circular()
    for dt, vp, tol in (("f32", oracle.view_proj3D, 2e-5), ("f64", oracle.view_proj3D_f64, 1e-12)):
        ind = np.zeros(scan.shape, np.int32)
        ind[3, scan.nu // 2 + 1, scan.nv // 2 - 2] = 1
        y = np.zeros(scan.shape)
        y[3, scan.nu // 2 + 1, scan.nv // 2 - 2] = 7.5
        x1 = getattr(vp, "artstep_" + kind)(1.0, y, ind, scan.frame_vectors, *scan.view, x,
                                            *vol.grid)
        p = getattr(vp, "sinoproj_" + kind)(ind, scan.frame_vectors, *scan.view, x1, *vol.grid)
        got = p[3, scan.nu // 2 + 1, scan.nv // 2 - 2]
        assert abs(got / 7.5 - 1.0) < tol, (dt, got)


def test_em_fixed_point():
    vol, scan, x = small_circular()
    x = x + 0.1
    ind = np.ones(scan.shape, np.int32)
    y = oracle.view_proj3D_f64.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    x1 = oracle.view_proj3D_f64.emstep_linear(y, ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    ones = oracle.view_proj3D_f64.sinobackproject_linear(np.ones(scan.shape), ind,
                                                         scan.frame_vectors, *scan.view, *vol.grid)
    m = ones > 1e-3
    assert np.max(np.abs(x1[m] - x[m]) / x[m]) < 1e-10


def test_ellipsoid_chord_of_sphere():
    vol, scan, _ = small_circular()
    nu, nv = scan.nu, scan.nv
    fv = scan.frame_vectors[2]
    r, c = 9.0, (1.5, -2.0, 0.5)
    out = oracle.view_proj3D_f64.ellipsoid_proj(np.ones((nu, nv), np.int32), fv, nu, nv, scan.du,
                                                scan.dv, scan.u0, scan.v0, r, r, r, *c, 0.3, 1.1,
                                                2.0)
    S = fv[0:3].astype(np.float64)
    for ju, kv in ((nu // 2, nv // 2), (nu // 2 + 3, nv // 2 - 4), (2, 3)):
        u = scan.u0 + (ju + 0.5) * scan.du
        v = scan.v0 + (kv + 0.5) * scan.dv
        B = fv[6:9] + fv[9:12] * np.float32(u) + fv[12:15] * np.float32(v)
        d = (B - S) / np.linalg.norm(B - S)
        w = np.array(c) - S
        dist2 = np.dot(w, w) - np.dot(w, d) ** 2
        chord = 2 * math.sqrt(max(r * r - dist2, 0.0)) * 2.0
        assert abs(out[ju, kv] - chord) < 1e-6 * max(1.0, chord)


def test_tv_constant_is_zero_and_fd_gradient():
    x = np.full((6, 7, 5), 3.25)
    assert abs(oracle.totalvar_f64.total_var3d(0.0, x, 6, 7, 5)) < 1e-9
    rng = np.random.default_rng(1)
    x = rng.random((6, 7, 5))
    g, bobo = oracle.totalvar_f64.total_var_grad3d(0.0, x, 6, 7, 5, 0)
    h = 1e-6
    for idx in [(1, 1, 1), (3, 4, 2), (5, 6, 4), (0, 0, 0), (2, 0, 3)]:
        xp = x.copy()
        xm = x.copy()
        xp[idx] += h
        xm[idx] -= h
        fd = (oracle.totalvar_f64.total_var3d(0.0, xp, 6, 7, 5) -
              oracle.totalvar_f64.total_var3d(0.0, xm, 6, 7, 5)) / (2 * h)
        assert abs(fd - g[idx]) < 1e-5 * max(1.0, abs(g[idx])), (idx, fd, g[idx])
    assert bobo > 0


def test_tomo_z_projector_matches_general_when_z_driven():
    # isotropic voxels: every ray of this +-25 deg arc is then z-driven under
    # the general rule too (with 0.1 x 1 mm voxels most rays would not be,
    # which is why the tomosynthesis kernels force the z axis)
    from ct2b200 import workloads as W
    vol = W.Volume(40, 32, 24, 0.5, 0.5, 0.5, -10.0, -8.0, -6.0)
    scan = W.tomo_scan(7, 48, 40, 0.5, 0.5, radius=300.0, c2d=20.0)
    x = W.voxelize(vol, W.random_ellipsoids(5, 20.0, seed=5))
    ind = np.ones(scan.shape, np.int32)
    a = oracle.view_proj3D_tomo.sinoprojz(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    b = oracle.view_proj3D.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    # in this geometry every ray is z-driven, so the general projector agrees
    assert rel_l2(a, b) < 1e-7


def test_ray_list_matches_view_geometry():
    vol, scan, x = small_circular(n=12, ns=3, nd=10)
    rv = ray_list_from_scan(scan)
    ind = np.ones(len(rv), np.int32)
    a = oracle.ray_proj3D.sinoproj_linear(ind, rv, len(rv), x, *vol.grid)
    b = oracle.view_proj3D.sinoproj_linear(np.ones(scan.shape, np.int32), scan.frame_vectors,
                                           *scan.view, x, *vol.grid)
    assert np.array_equal(a, b.ravel())


def test_spherical_radon_trace_pins_oracle():
    """The oracle reproduces the reference's recorded first iteration of the
    spherical-Radon ART + TV example (derrEvol.txt row 1) to 1e-3: pins
    radon3D.spherical_radon_linear, radon3D.artstep_linear, totalvar.total_var3d
    and the loop glue."""
    import radon_case
    got = radon_case.first_iteration(oracle.radon3D, oracle.totalvar,
                                     oracle.tomo3Dfort.ellipsoid_embed)
    for g, want in zip(got, radon_case.TRACE_ITER1):
        assert abs(g - want) <= 1e-3 * abs(want), (got, radon_case.TRACE_ITER1)


def test_fdk_oracle_matches_reference_golden():
    """oracle.fdk restates emil_code/FDK.py; the fixture was produced by the
    reference module itself (tests/golden/make_fdk_golden.py)."""
    import os
    from oracle import fdk
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "fdk_small.npz"))
    ns, nu, nv, du, dv, u0, v0, radius, sdd = g["params"]
    ns, nu, nv = int(ns), int(nu), int(nv)
    w = fdk.fdk_sino_weight3D(radius, sdd - radius, ns, g["vu"], g["vv"], g["sino"])
    assert np.array_equal(w, g["weighted"])
    assert np.array_equal(fdk.fdk_sino_filter3D(du, 1, w), g["f_plain"])
    assert np.array_equal(fdk.fdk_sino_filter3D(du, 1, w, 'Hann', L=1), g["f_hann"])
    assert np.array_equal(fdk.fdk_sino_filter3D(du, 1, w, 'Hann', L=0.5), g["f_hann_half"])
    assert np.array_equal(fdk.fdk_sino_filter3D(dv, 2, w), g["f_v"])
    r = fdk.fdk_backproj_linear3D(ns, nu, nv, du, dv, u0, v0, radius, sdd, 0.5, 0.5, g["vs"],
                                  g["vx"], g["vy"], g["vz"], g["f_hann"])
    assert np.array_equal(r, g["recon"])


def test_tv_p_variants_known_answer():
    """The reference's TpV/TpdV check (emil_code/tests/tpvGrad.py:40-80, in
    FP64): along the normalised gradient g/|g| the central difference of the
    value equals |g| (bobo) -- for TpV, TpdV and Lp, several p."""
    tv = oracle.totalvar_f64
    rng = np.random.default_rng(0)
    x = rng.standard_normal((3, 4, 5))
    d = 1e-7
    for p in (1.0, 1.5, 0.8):
        g, b = tv.total_p_var_grad3d(p, x, 3, 4, 5, 1)
        fd = (tv.total_var3d_p(p, x + d * g / 2, 3, 4, 5) -
              tv.total_var3d_p(p, x - d * g / 2, 3, 4, 5)) / d
        assert abs(fd - b) <= 1e-6 * b
        g, b = tv.total_p_dvar_grad3d(p, x, 3, 4, 5, 0.7, 0.9, 1.3, 1)
        fd = (tv.total_dvar3d_p(p, x + d * g / 2, 3, 4, 5, 0.7, 0.9, 1.3) -
              tv.total_dvar3d_p(p, x - d * g / 2, 3, 4, 5, 0.7, 0.9, 1.3)) / d
        assert abs(fd - b) <= 1e-6 * b
        g, b = tv.lp_grad3d(p, x, 3, 4, 5, 1)
        fd = (tv.calc_lp(p, x + d * g / 2, 3, 4, 5) - tv.calc_lp(p, x - d * g / 2, 3, 4, 5)) / d
        assert abs(fd - b) <= 1e-6 * b


def test_tv_p_variants_at_p1_and_p2():
    """TpV at p = 1 is the TV (same value, gradient up to ppp = 1); Lp at p = 2
    is the sum of squares (+ eps)."""
    tv = oracle.totalvar_f64
    rng = np.random.default_rng(1)
    x = rng.standard_normal((5, 6, 7))
    assert abs(tv.total_var3d_p(1.0, x, 5, 6, 7) - tv.total_var3d(0.0, x, 5, 6, 7)) <= 1e-9
    g1, _ = tv.total_p_var_grad3d(1.0, x, 5, 6, 7, 0)
    g0, _ = tv.total_var_grad3d(0.0, x, 5, 6, 7, 0)
    assert np.allclose(g1, g0, rtol=1e-12, atol=1e-12)
    assert abs(tv.calc_lp(2.0, x, 5, 6, 7) - (np.sum(x * x) + x.size * 1e-9)) <= 1e-8
    m = tv.gmi(x, 5, 6, 7)
    assert np.all(m[0] == 0) and np.all(m[:, 0] == 0) and np.all(m[:, :, 0] == 0)


@pytest.mark.parametrize("dt", ["f32", "f64"])
def test_oracle_threaded_pair_equals_serial(dt):
    """The host-threaded projector and backprojector (the CPU baseline, and
    the FP64 checker of large jobs) compute what the serial ones do."""
    vp = oracle.view_proj3D if dt == "f32" else oracle.view_proj3D_f64
    vol, scan, x = small_circular()
    ind = np.ones(scan.shape, np.int32)
    a = vp.sinoproj_linear(ind, scan.frame_vectors, *scan.view, x, *vol.grid)
    b = vp.sinoproj_linear_omp(ind, scan.frame_vectors, *scan.view, x, *vol.grid, 4)
    assert np.array_equal(a, b)
    c = vp.sinobackproject_linear(a, ind, scan.frame_vectors, *scan.view, *vol.grid)
    d = vp.sinobackproject_linear_omp(a, ind, scan.frame_vectors, *scan.view, *vol.grid, 4)
    assert rel_l2(d, c) < (1e-6 if dt == "f32" else 1e-14)
