"""Generates tests/golden/joseph.npz and tests/golden/geometry.npz from the
reference's own Python code.

joseph.npz -- the Joseph projector family run by the reference's numba
translation of emil_code/view_proj3D.f (emil_code/translatedFortrans/
view_proj3D.py: sinoproj_linear :309, sinobackproject_linear :398,
sinoproj_nearest :495, sinobackproject_nearest :562, ellipsoid_proj :252).
The translation evaluates in FP64 when handed FP64 arrays, so it pins the
FP64 oracle.  Cases (each small enough for the scalar oracle in a second):

* ``c0r``   -- config 0 reduced: 24^3 at 2.5 mm, circular cone beam SID 300 /
  SDD 600, 12 views over 360 deg, 36^2 detector at 3.5 mm, a random
  indicator with about 10 % of the rays off;
* ``turn``  -- a close source (SID 60 / SDD 120) and a detector turned by 30
  degrees in its own plane and taller than it is wide, so every driving axis
  (x, y and z) occurs, and the ray steps cross voxel rows obliquely;
* ``tie``   -- hand-built 45-degree views whose central detector column sees
  |dx| = |dy| exactly (the x/y tie goes to y, view_proj3D.f:811,843) and rays
  that pass through voxel faces, where the nearest-voxel floor sits on a
  boundary;
* ``tomo``  -- the tomosynthesis geometry (source arc over a stationary
  detector), mostly z-driven rays through a thin slab.

Inputs are stored as float32 values (exact in FP64); the translation's FP64
outputs are stored as float64.  ellipsoid_proj is recorded for a handful of
ellipsoids (two rotation angles, as the reference's routine takes) on every
third view of the c0r and turn cases.

geometry.npz -- frame vectors made by the reference's
emil_code/configs3D.py (config_vectors_circular_conebeam :11-49,
config_vectors_tomosynthesis :615-654) at the parameters of configurations
0-3, on the view parameters of sinogram3D.__init__ (emil_code/tomo3D.py:
113-147, get_ds :186-190: s = s0 + ip*ds, ds = slen/(ns-1) with the end
points included, slen/ns without), stored as float32 as sinogram3D does.

The reference root is read at generation time only; the committed .npz files
are what the tests use.

Run: python tests/golden/make_joseph_golden.py <reference root>
     (or set CT2_REFERENCE_ROOT)
"""
import math
import os
import sys
import tempfile

import numpy as np

from refroot import reference_root  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_J = os.path.join(HERE, "joseph.npz")
OUT_G = os.path.join(HERE, "geometry.npz")


# ---------------------------------------------------------------------------
# geometry
# ---------------------------------------------------------------------------

GEOMETRY = {
    # name: (config function, parms, ns, slen, s0, include end points)
    "c0": ("circular_conebeam", {"radius": 300.0, "source_to_detector": 600.0}, 60,
           2 * math.pi, 0.0, 0),
    "c1": ("circular_conebeam", {"radius": 500.0, "source_to_detector": 1000.0}, 360,
           2 * math.pi, 0.0, 0),
    "c2": ("tomosynthesis", {"radius": 603.0, "center_to_detector": 47.0}, 25,
           2 * math.radians(25.0), math.pi / 2 - math.radians(25.0), 1),
    "c3": ("circular_conebeam", {"radius": 400.0, "source_to_detector": 800.0}, 180,
           2 * math.pi, 0.0, 0),
    "small": ("circular_conebeam", {"radius": 60.0, "source_to_detector": 120.0}, 10,
              2 * math.pi, 0.3, 0),
}


def ref_frames(cfg, name, parms, ns, slen, s0, endpoints):
    fn = getattr(cfg, "config_vectors_" + name)
    ds = slen / (ns - 1.0) if endpoints else slen / ns
    fv = np.zeros((ns, 18), np.float32)
    for ip in range(ns):
        fv[ip] = fn(s0 + ip * ds, parms)
    return fv


# ---------------------------------------------------------------------------
# Joseph cases
# ---------------------------------------------------------------------------

def circular_frames(cfg, ns, radius, sdd, s0=0.0):
    return ref_frames(cfg, "circular_conebeam",
                      {"radius": radius, "source_to_detector": sdd}, ns, 2 * math.pi, s0, 0)


def turned(fv, angle):
    """Rotate each view's detector axes (eu, ev) by ``angle`` in the detector
    plane."""
    out = fv.astype(np.float64).copy()
    c, s = math.cos(angle), math.sin(angle)
    eu, ev = out[:, 9:12].copy(), out[:, 12:15].copy()
    out[:, 9:12] = c * eu + s * ev
    out[:, 12:15] = -s * eu + c * ev
    return out.astype(np.float32)


def tie_frames():
    """Views at 45 degrees (and 225, 135) built from exact binary values:
    source (a, a, h), detector centre (-b, -b, h), eu along (-1, 1, 0); the
    central column of an odd-width detector sits at u = 0, where
    xdiff = ydiff exactly."""
    rows = []
    for sx, sy in ((1, 1), (-1, -1), (-1, 1)):
        a, b, h = 64.0, 64.0, 0.0
        src = (sx * a, sy * a, h)
        det = (-sx * b, -sy * b, h)
        eu = (-sy * 0.75, sx * 0.75, 0.0)  # not unit: exact binary, keeps the tie exact
        ev = (0.0, 0.0, 1.0)
        ew = (sx * 0.75, sy * 0.75, 0.0)
        rows.append(src + (0.0, 0.0, 0.0) + det + eu + ev + ew)
    return np.array(rows, np.float32)


def tomo_frames(cfg, ns, radius, c2d, half_deg):
    half = math.radians(half_deg)
    return ref_frames(cfg, "tomosynthesis", {"radius": radius, "center_to_detector": c2d}, ns,
                      2 * half, math.pi / 2 - half, 1)


def make_cases(cfg):
    rng = np.random.default_rng(20261204)
    cases = {}

    # config 0 reduced
    n, d = 24, 2.5
    grid = (d, d, d, -n * d / 2, -n * d / 2, -n * d / 2, n, n, n)
    nu = nv = 36
    du = dv = 3.5
    view = (12, nu, nv, du, dv, -nu * du / 2, -nv * dv / 2)
    ind = (rng.random((12, nu, nv)) > 0.1).astype(np.int32)
    cases["c0r"] = (circular_frames(cfg, 12, 300.0, 600.0), view, grid, ind)

    # close source, turned and tall detector: x-, y- and z-driven rays
    n, d = 20, 2.0
    grid = (d, d * 1.25, d * 0.8, -20.0, -25.0, -16.0, n, n, n + 4)
    nu, nv = 30, 40
    du, dv = 5.0, 6.5
    view = (6, nu, nv, du, dv, -nu * du / 2, -nv * dv / 2)
    ind = np.ones((6, nu, nv), np.int32)
    cases["turn"] = (turned(circular_frames(cfg, 6, 60.0, 120.0, s0=0.2), math.radians(30.0)),
                     view, grid, ind)

    # exact x/y ties and voxel-face crossings
    n, d = 16, 2.0
    grid = (d, d, d, -16.0, -16.0, -16.0, n, n, n)
    nu, nv = 17, 17  # odd: the middle column has u = 0 exactly
    du, dv = 2.0, 2.0
    view = (3, nu, nv, du, dv, -nu * du / 2, -nv * dv / 2)
    ind = np.ones((3, nu, nv), np.int32)
    cases["tie"] = (tie_frames(), view, grid, ind)

    # tomosynthesis slab
    grid = (0.5, 0.5, 2.0, -10.0, -8.0, -12.0, 40, 32, 12)
    nu, nv = 44, 36
    view = (5, nu, nv, 0.55, 0.55, -nu * 0.55 / 2, -nv * 0.55 / 2)
    ind = np.ones((5, nu, nv), np.int32)
    cases["tomo"] = (tomo_frames(cfg, 5, 300.0, 20.0, 25.0), view, grid, ind)
    return cases, rng


def main():
    root = reference_root()
    os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp())
    sys.path.insert(0, os.path.join(root, "emil_code"))
    sys.path.insert(0, os.path.join(root, "emil_code", "translatedFortrans"))
    import configs3D as cfg  # noqa: E402  (the reference's geometry module)
    import view_proj3D as tr  # noqa: E402  (the reference's numba translation)

    geo = {}
    for key, (name, parms, ns, slen, s0, ep) in GEOMETRY.items():
        geo[key] = ref_frames(cfg, name, parms, ns, slen, s0, ep)
        geo[key + "_params"] = np.array([ns, slen, s0, ep], np.float64)
    np.savez_compressed(OUT_G, **geo)
    print("wrote", OUT_G)

    cases, rng = make_cases(cfg)
    out = {"cases": np.array(sorted(cases))}
    for key, (fv, view, grid, ind) in cases.items():
        ns, nu, nv, du, dv, u0, v0 = view
        dx, dy, dz, x0, y0, z0, nx, ny, nz = grid
        vol = rng.random((nx, ny, nz)).astype(np.float32)
        sino = rng.random((ns, nu, nv)).astype(np.float32)
        fv64 = fv.astype(np.float64)
        vol64 = vol.astype(np.float64)
        sino64 = sino.astype(np.float64)
        res = {}
        for kind in ("linear", "nearest"):
            p = np.zeros((ns, nu, nv))
            getattr(tr, "sinoproj_" + kind)(p, ind, fv64, ns, nu, nv, du, dv, u0, v0, vol64,
                                            dx, dy, dz, x0, y0, z0, nx, ny, nz)
            b = np.zeros((nx, ny, nz))
            getattr(tr, "sinobackproject_" + kind)(sino64, ind, fv64, ns, nu, nv, du, dv, u0, v0,
                                                   b, dx, dy, dz, x0, y0, z0, nx, ny, nz)
            res["proj_" + kind] = p
            res["bp_" + kind] = b
        out[key + "_fv"] = fv
        out[key + "_view"] = np.array(view, np.float64)
        out[key + "_grid"] = np.array(grid, np.float64)
        out[key + "_ind"] = ind.astype(np.uint8)
        out[key + "_vol"] = vol
        out[key + "_sino"] = sino
        for k, v in res.items():
            out[key + "_" + k] = v

    # ellipsoid_proj: (ax, ay, az, x0, y0, z0, alpha, beta, att) per ellipsoid
    for key in ("c0r", "turn"):
        fv, view, grid, ind = cases[key]
        ns, nu, nv, du, dv, u0, v0 = view
        fov = grid[6] * grid[0]
        ells = []
        for _ in range(4):
            ax = rng.uniform(0.1, 0.35, 3) * fov
            c = rng.uniform(-0.25, 0.25, 3) * fov
            ang = rng.uniform(0, math.pi, 2)
            ells.append(np.concatenate([ax, c, ang, [rng.uniform(0.2, 1.0)]]))
        ells = np.array(ells)
        views = np.arange(0, ns, 3)
        sino = np.zeros((len(views), len(ells), nu, nv))
        ind1 = np.ones((nu, nv), np.int32)
        ind1[::4, 1::5] = 0
        for i, s in enumerate(views):
            f = fv[s].astype(np.float64)
            for e, (ax, ay, az, cx, cy, cz, al, be, att) in enumerate(ells):
                tr.ellipsoid_proj(sino[i, e], ind1, f, nu, nv, du, dv, u0, v0, ax, ay, az, cx,
                                  cy, cz, al, be, att)
        out[key + "_ells"] = ells
        out[key + "_ell_views"] = views
        out[key + "_ell_ind"] = ind1
        out[key + "_ell_sino"] = sino
    np.savez_compressed(OUT_J, **out)
    print("wrote", OUT_J)


if __name__ == "__main__":
    main()
