"""Generates tests/golden/fdk_small.npz by running the reference's own
emil_code/FDK.py (and setFreqrange.py) on a small seeded case.

The reference modules are Python 2 (print statements, tab-indented); this
script loads their source, rewrites only what Python 3 cannot parse or run
(print statements -> print(), tab expansion, `npad/2` indexing ->
`npad//2`, numpy's removed `n.integer` alias -> `int`), and executes them.
It reads the reference's sources at generation time only; the committed .npz is
what the tests use.

Run: python tests/golden/make_fdk_golden.py <reference root>
     (or set CT2_REFERENCE_ROOT)
"""
import os
import re
import types

import numpy as np

from refroot import reference_root  # noqa: E402

REF = os.path.join(reference_root(), "emil_code")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fdk_small.npz")


def load(name, extra_globals=None):
    src = open(os.path.join(REF, name + ".py")).read().expandtabs(8)
    src = re.sub(r"^(\s*)print (.*)$", r"\1print(\2)", src, flags=re.M)
    src = src.replace("hn[npad/2]", "hn[npad//2]").replace("n.integer", "int")
    mod = types.ModuleType(name)
    if extra_globals:
        mod.__dict__.update(extra_globals)
    exec(compile(src, name + ".py", "exec"), mod.__dict__)
    return mod


def main():
    import sys
    setf = load("setFreqrange")
    sys.modules["setFreqrange"] = setf
    fdk = load("FDK")
    rng = np.random.default_rng(2024)
    # circular cone beam: SID 40, SDD 80, 16 views, 24 x 20 detector
    ns, nu, nv = 16, 24, 20
    du, dv = 1.0, 1.1
    u0, v0 = -nu * du / 2.0, -nv * dv / 2.0
    radius, sdd = 40.0, 80.0
    sino = rng.random((ns, nu, nv)).astype(np.float32)
    vs = np.arange(ns) * (2 * np.pi / ns)
    vu = u0 + (np.arange(nu) + 0.5) * du
    vv = v0 + (np.arange(nv) + 0.5) * dv
    vv, vu = np.meshgrid(vv, vu)
    w = fdk.fdk_sino_weight3D(radius, sdd - radius, ns, vu, vv, sino)
    f_plain = fdk.fdk_sino_filter3D(du, 1, w)
    f_hann = fdk.fdk_sino_filter3D(du, 1, w, 'Hann', L=1)
    f_hann_half = fdk.fdk_sino_filter3D(du, 1, w, 'Hann', L=0.5)
    f_v = fdk.fdk_sino_filter3D(dv, 2, w)
    nx = ny = 10
    nz = 6
    dx = 0.8
    x0 = -nx * dx / 2.0
    vx = x0 + (np.arange(nx) + 0.5) * dx
    vy = x0 + (np.arange(ny) + 0.5) * dx
    vz = -nz * dx / 2.0 + (np.arange(nz) + 0.5) * dx
    vx, vy = np.meshgrid(vx, vy)
    vx = vx.flatten()
    vy = vy.flatten()
    import builtins
    _print = builtins.print
    builtins.print = lambda *a, **k: None  # the reference prints a line per z slice
    try:
        recon = fdk.fdk_backproj_linear3D(ns, nu, nv, du, dv, u0, v0, radius, sdd, 0.5, 0.5, vs,
                                          vx, vy, vz, f_hann)
    finally:
        builtins.print = _print
    np.savez_compressed(OUT, sino=sino, vs=vs, vu=vu, vv=vv, vx=vx, vy=vy, vz=vz, weighted=w,
                        f_plain=f_plain, f_hann=f_hann, f_hann_half=f_hann_half, f_v=f_v,
                        recon=recon,
                        params=np.array([ns, nu, nv, du, dv, u0, v0, radius, sdd]))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
