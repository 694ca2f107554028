"""The CUDA Joseph projectors, matched backprojectors and the analytic
ellipsoid projector, through the f2py-signature drop-ins (C ABI), against
outputs of the reference's own code: tests/golden/joseph.npz, the FP64 run of
the reference's numba translation of emil_code/view_proj3D.f on four small
cases (config 0 reduced with a random indicator, a turned detector with a
close source, exact driving-axis ties, the tomosynthesis slab).

Tolerances: linear projections and backprojections <= 1e-5 relative L2, the
plain-form bar; nearest sampling is discontinuous, and the FP32 arithmetic
the reference itself runs in (the REAL*4 oracle) sits up to 5e-3 from the
FP64 run where a floor lands on a voxel face, so there the GPU is held to the
REAL*4 oracle at 1e-5 and to the FP64 run no farther than the REAL*4 oracle
is, plus 1e-5.
"""
import os

import numpy as np
import pytest

import oracle
import view_proj3D
from helpers import rel_l2

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
J = np.load(os.path.join(GOLD, "joseph.npz"))
CASES = [str(c) for c in J["cases"]]


def case(key):
    view = J[key + "_view"]
    grid = J[key + "_grid"]
    ns, nu, nv = (int(v) for v in view[:3])
    view = (ns, nu, nv) + tuple(float(np.float32(v)) for v in view[3:])
    grid = tuple(float(np.float32(v)) for v in grid[:6]) + tuple(int(v) for v in grid[6:])
    return (J[key + "_fv"], view, grid, J[key + "_ind"].astype(np.int32), J[key + "_vol"],
            J[key + "_sino"])


@pytest.mark.parametrize("key", CASES)
@pytest.mark.parametrize("kind", ["linear", "nearest"])
def test_projector_vs_reference(cuda, key, kind):
    fv, view, grid, ind, vol, _ = case(key)
    got = getattr(view_proj3D, "sinoproj_" + kind)(ind, fv, *view, vol, *grid)
    ref = J[key + "_proj_" + kind]
    if kind == "linear":
        assert rel_l2(got, ref) <= 1e-5
    else:
        o32 = oracle.view_proj3D.sinoproj_nearest(ind, fv, *view, vol, *grid)
        assert rel_l2(got, o32) <= 1e-5
        assert rel_l2(got, ref) <= rel_l2(o32, ref) + 1e-5


@pytest.mark.parametrize("key", CASES)
@pytest.mark.parametrize("kind", ["linear", "nearest"])
def test_backprojector_vs_reference(cuda, key, kind):
    fv, view, grid, ind, _, sino = case(key)
    got = getattr(view_proj3D, "sinobackproject_" + kind)(sino, ind, fv, *view, *grid)
    ref = J[key + "_bp_" + kind]
    if kind == "linear":
        assert rel_l2(got, ref) <= 1e-5
    else:
        o32 = oracle.view_proj3D.sinobackproject_nearest(sino, ind, fv, *view, *grid)
        assert rel_l2(got, o32) <= 1e-5
        assert rel_l2(got, ref) <= rel_l2(o32, ref) + 1e-5


@pytest.mark.parametrize("key", ["c0r", "turn"])
def test_ellipsoid_proj_vs_reference(cuda, key):
    fv = J[key + "_fv"]
    view = J[key + "_view"]
    nu, nv = int(view[1]), int(view[2])
    du, dv, u0, v0 = (float(np.float32(v)) for v in view[3:])
    ind = J[key + "_ell_ind"].astype(np.int32)
    ref = J[key + "_ell_sino"]
    for i, s in enumerate(J[key + "_ell_views"]):
        for e, p in enumerate(J[key + "_ells"]):
            p = [float(np.float32(v)) for v in p]
            got = view_proj3D.ellipsoid_proj(ind, fv[s], nu, nv, du, dv, u0, v0, *p)
            # cosf/sinf of CUDA against the reference's FP64 cos/sin
            assert rel_l2(got, ref[i, e]) <= 1e-4
