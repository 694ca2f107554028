"""The oracle's Joseph projector family and the geometry generator against
outputs of the reference's own code (no GPU needed).

tests/golden/joseph.npz holds the reference's numba translation of
emil_code/view_proj3D.f (translatedFortrans/view_proj3D.py: sinoproj_linear
:309, sinobackproject_linear :398, sinoproj_nearest :495,
sinobackproject_nearest :562, ellipsoid_proj :252) run in FP64 on four small
cases -- config 0 reduced with a random indicator, a turned detector with a
close source (x-, y- and z-driven rays), exact x/y driving-axis ties with
rays through voxel faces, and the tomosynthesis slab.
tests/golden/geometry.npz holds the frame vectors of the reference's
emil_code/configs3D.py at the configurations' parameters.  Both were made by
tests/golden/make_joseph_golden.py.
"""
import os

import numpy as np
import pytest

import configs3D
import oracle
from ct2b200 import workloads as W
from helpers import rel_l2

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
J = np.load(os.path.join(GOLD, "joseph.npz"))
G = np.load(os.path.join(GOLD, "geometry.npz"))
CASES = [str(c) for c in J["cases"]]


def case(key):
    view = J[key + "_view"]
    grid = J[key + "_grid"]
    ns, nu, nv = (int(v) for v in view[:3])
    view = (ns, nu, nv) + tuple(float(v) for v in view[3:])
    grid = tuple(float(v) for v in grid[:6]) + tuple(int(v) for v in grid[6:])
    return (J[key + "_fv"], view, grid, J[key + "_ind"].astype(np.int32), J[key + "_vol"],
            J[key + "_sino"])


def f32(vals):
    return tuple(float(np.float32(v)) if isinstance(v, float) else v for v in vals)


@pytest.mark.parametrize("key", CASES)
@pytest.mark.parametrize("kind", ["linear", "nearest"])
def test_fp64_oracle_matches_reference_projection(key, kind):
    fv, view, grid, ind, vol, _ = case(key)
    got = getattr(oracle.view_proj3D_f64, "sinoproj_" + kind)(ind, fv, *view, vol, *grid)
    ref = J[key + "_proj_" + kind]
    assert got.shape == ref.shape
    assert rel_l2(got, ref) < 1e-12, rel_l2(got, ref)
    assert np.max(np.abs(got - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("key", CASES)
@pytest.mark.parametrize("kind", ["linear", "nearest"])
def test_fp64_oracle_matches_reference_backprojection(key, kind):
    fv, view, grid, ind, _, sino = case(key)
    got = getattr(oracle.view_proj3D_f64, "sinobackproject_" + kind)(sino, ind, fv, *view, *grid)
    ref = J[key + "_bp_" + kind]
    assert got.shape == ref.shape
    assert rel_l2(got, ref) < 1e-12, rel_l2(got, ref)
    assert np.max(np.abs(got - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("key", CASES)
@pytest.mark.parametrize("kind", ["linear", "nearest"])
def test_fp32_oracle_near_reference(key, kind):
    """The REAL*4 oracle (the GPU's parity target) is within FP32 rounding
    of the reference's FP64 evaluation on the same inputs."""
    fv, view, grid, ind, vol, sino = case(key)
    vp = oracle.view_proj3D
    p = getattr(vp, "sinoproj_" + kind)(ind, fv, *f32(view), vol, *f32(grid))
    b = getattr(vp, "sinobackproject_" + kind)(sino, ind, fv, *f32(view), *f32(grid))
    # nearest sampling is discontinuous: an FP32 floor may flip at a voxel face
    tol = 1e-5 if kind == "linear" else 5e-3
    assert rel_l2(p, J[key + "_proj_" + kind]) < tol
    assert rel_l2(b, J[key + "_bp_" + kind]) < tol


def test_cases_cover_every_driving_axis_and_ties():
    """The fixture exercises what it claims: x-, y- and z-driven rays, and
    exact |dx| = |dy| ties."""
    seen = set()
    ties = 0
    for key in CASES:
        fv, view, grid, ind, _, _ = case(key)
        ns, nu, nv, du, dv, u0, v0 = view
        d = np.array(grid[:3])
        f = fv.astype(np.float64)
        for s in range(ns):
            for j in range(nu):
                u = u0 + (j + 0.5) * du
                for k in range(nv):
                    v = v0 + (k + 0.5) * dv
                    b = f[s, 6:9] + f[s, 9:12] * u + f[s, 12:15] * v
                    ad = np.abs(b - f[s, 0:3]) / d
                    if ad[0] > ad[1] and ad[0] > ad[2]:
                        seen.add(0)
                    elif ad[1] > ad[2]:
                        seen.add(1)
                        ties += ad[0] == ad[1]
                    else:
                        seen.add(2)
    assert seen == {0, 1, 2}
    assert ties > 0


@pytest.mark.parametrize("key", ["c0r", "turn"])
def test_oracle_ellipsoid_proj_matches_reference(key):
    fv = J[key + "_fv"]
    view = J[key + "_view"]
    nu, nv = int(view[1]), int(view[2])
    du, dv, u0, v0 = (float(v) for v in view[3:])
    ind = J[key + "_ell_ind"].astype(np.int32)
    ref = J[key + "_ell_sino"]
    for i, s in enumerate(J[key + "_ell_views"]):
        for e, (ax, ay, az, cx, cy, cz, al, be, att) in enumerate(J[key + "_ells"]):
            got = oracle.view_proj3D_f64.ellipsoid_proj(ind, fv[s], nu, nv, du, dv, u0, v0, ax,
                                                        ay, az, cx, cy, cz, al, be, att)
            assert rel_l2(got, ref[i, e]) < 1e-12
            g32 = oracle.view_proj3D.ellipsoid_proj(ind, fv[s], nu, nv, *f32((du, dv, u0, v0)),
                                                    *f32((ax, ay, az, cx, cy, cz, al, be, att)))
            assert rel_l2(g32, ref[i, e]) < 1e-5


GEOMETRY = {
    "c0": ("circular_conebeam", {"radius": 300.0, "source_to_detector": 600.0}),
    "c1": ("circular_conebeam", {"radius": 500.0, "source_to_detector": 1000.0}),
    "c2": ("tomosynthesis", {"radius": 603.0, "center_to_detector": 47.0}),
    "c3": ("circular_conebeam", {"radius": 400.0, "source_to_detector": 800.0}),
    "small": ("circular_conebeam", {"radius": 60.0, "source_to_detector": 120.0}),
}


@pytest.mark.parametrize("key", sorted(GEOMETRY))
def test_frame_vectors_equal_reference_configs3D(key):
    name, parms = GEOMETRY[key]
    ns, slen, s0, ep = G[key + "_params"]
    fv = configs3D.frame_vectors(name, parms, int(ns), float(slen), float(s0), int(ep))
    assert fv.dtype == np.float32
    assert np.array_equal(fv, G[key]), np.max(np.abs(fv - G[key]))


def test_workload_geometries_equal_reference_configs3D():
    """The configurations the bench and the workloads run use exactly the
    reference generator's frame vectors."""
    assert np.array_equal(W.config0()[1].frame_vectors, G["c0"])
    assert np.array_equal(W.config1()[1].frame_vectors, G["c1"])
    assert np.array_equal(W.config2()[1].frame_vectors, G["c2"])
    assert np.array_equal(W.config3_single()[1].frame_vectors, G["c3"])
