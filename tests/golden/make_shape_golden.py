"""Generates tests/golden/shape_roots.npz from the reference's own Python
restatement of the analytic-surface projector,
emil_code/translatedFortrans/view_proj3D.py (numba; a machine translation of
emil_code/view_proj3D.f that its header marks as not yet checked).

What is recorded, all with FP64 inputs:

* root_plane / root_ellipsoid / root_cylinder / root_cone on seeded random
  segments (source outside, bin across the surface), troot as the
  translation returns it (float32);
* gen_shape_proj for objects made of planes and ellipsoids (the only kinds
  the translation's gen_shape_proj covers).  The translation indexes the
  surface arrays from 1 where emil_code/view_proj3D.f starts at the first
  entry, so it is given the arrays with one leading dummy surface; the
  fixture stores the arrays without it, in the layout the Fortran and
  tomo3D.py's gen_object.project_to use.

It reads the reference's sources at generation time only; the committed .npz is
what the tests use.

Run: python tests/golden/make_shape_golden.py <reference root>
     (or set CT2_REFERENCE_ROOT)
"""
import os
import sys
import tempfile

import numpy as np

from refroot import reference_root  # noqa: E402

REF = os.path.join(reference_root(), "emil_code", "translatedFortrans")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "shape_roots.npz")


def frame(alpha, beta, gamma):
    """Rows (xu, yu, zu) of a surface frame as tomo3D.py's surface class
    builds them (gamma about z, beta about y, alpha about z)."""
    def rot(v):
        x, y, z = v
        xp = x * np.cos(gamma) - y * np.sin(gamma)
        yp = x * np.sin(gamma) + y * np.cos(gamma)
        zp = z
        xpp = xp * np.cos(beta) + zp * np.sin(beta)
        ypp = yp
        zpp = -xp * np.sin(beta) + zp * np.cos(beta)
        return (xpp * np.cos(alpha) - ypp * np.sin(alpha),
                ypp * np.cos(alpha) + xpp * np.sin(alpha), zpp)
    return [rot((1.0, 0.0, 0.0)), rot((0.0, 1.0, 0.0)), rot((0.0, 0.0, 1.0))]


def main():
    os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp())
    sys.path.insert(0, REF)
    import view_proj3D as tr  # the translation
    rng = np.random.default_rng(515)
    out = {}

    # ---- the four root routines ----
    n = 256
    seg = np.zeros((4, n, 9))
    roots = np.zeros((4, n, 2), np.float32)
    for i in range(n):
        a, b, c = rng.uniform(0.5, 3.0, 3)
        s = rng.normal(size=3)
        s = s / np.linalg.norm(s) * rng.uniform(6.0, 12.0)
        e = -s * rng.uniform(0.8, 1.2) + rng.normal(scale=1.5, size=3)
        seg[:, i, :6] = np.concatenate([s, e])
        seg[:, i, 6:] = (a, b, c)
        roots[0, i] = tr.root_plane(s[2], e[2])
        roots[1, i] = tr.root_ellipsoid(*s, *e, a, b, c)
        roots[2, i] = tr.root_cylinder(s[0], s[1], e[0], e[1], a, b)
        # cone: start below the apex plane or above it, aim across the axis
        cs = np.array([rng.uniform(-8, 8), rng.uniform(-8, 8), rng.uniform(-4, 10)])
        ce = np.array([rng.uniform(-8, 8), rng.uniform(-8, 8), rng.uniform(-4, 10)])
        seg[3, i, :6] = np.concatenate([cs, ce])
        roots[3, i] = tr.root_cone(*cs, *ce, a, b)
    out["root_inputs"] = seg
    out["roots"] = roots

    # ---- gen_shape_proj: a slab cut by two planes, intersected with one or
    # two rotated ellipsoids, seen from a few cone-beam views ----
    nu, nv, du, dv = 24, 20, 1.25, 1.25
    u0, v0 = -nu * du / 2, -nv * dv / 2
    cases = []
    for case in range(4):
        surf = []
        h = rng.uniform(1.0, 3.0)
        surf.append(("plane", (0.0, 0.0, -h), frame(0.0, 0.0, 0.0), None))
        surf.append(("plane", (0.0, 0.0, h), frame(0.0, np.pi, 0.0), None))
        for k in range(1 + case % 2):
            ang = rng.uniform(0, np.pi, 3)
            ctr = rng.normal(scale=1.0, size=3)
            surf.append(("ellipsoid", tuple(ctr), frame(*ang), tuple(rng.uniform(2.0, 6.0, 3))))
        nsurf = len(surf)
        fr = np.zeros((12, nsurf))
        for i, (_, ctr, rows, _) in enumerate(surf):
            fr[0:3, i], fr[3:6, i], fr[6:9, i] = rows
            fr[9:12, i] = ctr
        ell = [(1.0, 1.0, 1.0)] + [s[3] for s in surf if s[0] == "ellipsoid"]
        ell = np.array(ell).T  # (3, nellipsoid)
        nplane = 1 + sum(s[0] == "plane" for s in surf)
        nell = ell.shape[1]
        att = rng.uniform(0.5, 2.0)
        views = []
        for v in range(3):
            th = 2 * np.pi * v / 3 + 0.3 * case
            src = np.array([30 * np.cos(th), 30 * np.sin(th), rng.uniform(-2, 2)])
            det = -src * (30.0 / 30.0)
            eu = np.array([-np.sin(th), np.cos(th), 0.0])
            ev = np.array([0.0, 0.0, 1.0])
            ew = np.cross(eu, ev)
            fv = np.concatenate([src, eu, det, eu, ev, ew]).astype(np.float32)
            ind = np.ones((nu, nv), np.int32)
            ind[::5, ::3] = 0
            sino = np.zeros((nu, nv), np.float32)
            dummy = lambda a: np.concatenate([[0.0], a])  # noqa: E731
            tr.gen_shape_proj(sino, ind, fv, nu, nv, du, dv, u0, v0, att, nsurf + 1,
                              *[dummy(fr[k]) for k in range(12)], nplane, nell,
                              ell[0].copy(), ell[1].copy(), ell[2].copy())
            views.append((fv, ind, sino))
        cases.append(dict(frames=fr, ell=ell, nplane=nplane, att=att, views=views))
    out["n_cases"] = np.array(len(cases))
    out["detector"] = np.array([nu, nv, du, dv, u0, v0])
    for c, d in enumerate(cases):
        out["c%d_frames" % c] = d["frames"]
        out["c%d_ell" % c] = d["ell"]
        out["c%d_nplane" % c] = np.array(d["nplane"])
        out["c%d_att" % c] = np.array(d["att"])
        out["c%d_fv" % c] = np.stack([v[0] for v in d["views"]])
        out["c%d_ind" % c] = np.stack([v[1] for v in d["views"]])
        out["c%d_sino" % c] = np.stack([v[2] for v in d["views"]])
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
