"""CPU oracle for the ct-2 reconstruction hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only as the checker or the timed CPU
baseline; the product (``ct-2_b200/``) never imports it.

It mirrors the reference's f2py modules with the same positional signatures
(intent(out) arguments dropped and returned, intent(in,out) arrays returned):

* ``view_proj3D``, ``view_proj3D_tomo``, ``ray_proj3D``, ``totalvar``,
  ``radon3D``, ``tomo3Dfort`` -- ctypes bindings of ``libct2oracle.so``, the
  C restatement of ``emil_code/*.f`` (see ``ct2_oracle_body.h``).  Each module
  object takes ``dtype=np.float32`` (REAL*4 parity oracle, the default) or
  ``np.float64`` (the FP64 oracle).
* ``fdk`` -- an FP64 NumPy restatement of ``emil_code/FDK.py``.

Arrays are C-ordered over the logical shapes the reference's Python callers
use: volumes (nx, ny, nz), sinograms (ns, nu, nv).
"""
import ctypes

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        _lib = ctypes.CDLL(path)
    return _lib


def _f(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _i(a):
    if a is None:
        return None
    return np.ascontiguousarray(a, dtype=np.int32)


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.c_void_p)


def _shapes(mod, nsurf, frames12, nplane, nellipsoid, ell3, ncyl, cyl2, ncone, cone2):
    """The surface table in the oracle's layout: the twelve frame arrays
    (xu1 .. z0, nsurf each) stacked, and each kind's semi-axis arrays
    concatenated (ax | ay [| az]); see ct2_oracle_body.h."""
    dt = mod.dt
    fr = np.zeros((12, max(int(nsurf), 1)), dt)
    for k, a in enumerate(frames12):
        a = np.asarray(a, dt).reshape(-1)
        fr[k, :a.size] = a
    def cat(arrs, n):
        out = np.zeros((len(arrs), max(int(n), 1)), dt)
        for k, a in enumerate(arrs):
            a = np.asarray(a, dt).reshape(-1)
            out[k, :a.size] = a
        return out
    keep = (fr, cat(ell3, nellipsoid), cat(cyl2, ncyl), cat(cone2, ncone))
    args = (int(nsurf), _p(keep[0]), int(nplane), int(nellipsoid), _p(keep[1]), int(ncyl),
            _p(keep[2]), int(ncone), _p(keep[3]))
    return keep, args


class _Mod:
    """One reference module bound at a given precision."""

    def __init__(self, dtype=np.float32):
        self.dt = np.dtype(dtype)
        self.pre = "ora_f_" if self.dt == np.float32 else "ora_d_"
        self.real = ctypes.c_float if self.dt == np.float32 else ctypes.c_double

    def _fn(self, name, restype=None):
        fn = getattr(lib(), self.pre + name)
        fn.restype = restype
        return fn

    def _r(self, x):
        return self.real(x)


class ViewProj3D(_Mod):
    """view_proj3D (emil_code/view_proj3D.f)."""

    def _proj(self, name, indsino, frame_vectors, ns, nu, nv, du, dv, u0, v0, smat, dx, dy, dz,
              x0, y0, z0, nx, ny, nz):
        out = np.zeros((ns, nu, nv), self.dt)
        ind = _i(indsino)
        fv = _f(frame_vectors, self.dt)
        sm = _f(smat, self.dt)
        r = self._r
        self._fn(name)(_p(out), _p(ind), _p(fv), ns, nu, nv, r(du), r(dv), r(u0), r(v0), _p(sm),
                       r(dx), r(dy), r(dz), r(x0), r(y0), r(z0), nx, ny, nz)
        return out

    def _bp(self, name, sinomat, indsino, frame_vectors, ns, nu, nv, du, dv, u0, v0, dx, dy, dz,
            x0, y0, z0, nx, ny, nz):
        out = np.zeros((nx, ny, nz), self.dt)
        r = self._r
        self._fn(name)(_p(_f(sinomat, self.dt)), _p(_i(indsino)), _p(_f(frame_vectors, self.dt)),
                       ns, nu, nv, r(du), r(dv), r(u0), r(v0), _p(out), r(dx), r(dy), r(dz),
                       r(x0), r(y0), r(z0), nx, ny, nz)
        return out

    def _art(self, name, reg_fac, sinomat, indsino, frame_vectors, ns, nu, nv, du, dv, u0, v0,
             smat, dx, dy, dz, x0, y0, z0, nx, ny, nz):
        x = np.array(smat, dtype=self.dt, order="C", copy=True)
        r = self._r
        self._fn(name)(r(reg_fac), _p(_f(sinomat, self.dt)), _p(_i(indsino)),
                       _p(_f(frame_vectors, self.dt)), ns, nu, nv, r(du), r(dv), r(u0), r(v0),
                       _p(x), r(dx), r(dy), r(dz), r(x0), r(y0), r(z0), nx, ny, nz)
        return x

    def _em(self, name, sinomat, indsino, frame_vectors, ns, nu, nv, du, dv, u0, v0, smat, dx, dy,
            dz, x0, y0, z0, nx, ny, nz):
        x = np.array(smat, dtype=self.dt, order="C", copy=True)
        r = self._r
        self._fn(name)(_p(_f(sinomat, self.dt)), _p(_i(indsino)), _p(_f(frame_vectors, self.dt)),
                       ns, nu, nv, r(du), r(dv), r(u0), r(v0), _p(x), r(dx), r(dy), r(dz), r(x0),
                       r(y0), r(z0), nx, ny, nz)
        return x

    def sinoproj_linear(self, *a):
        return self._proj("sinoproj_linear", *a)

    def sinoproj_nearest(self, *a):
        return self._proj("sinoproj_nearest", *a)

    def sinobackproject_linear(self, *a):
        return self._bp("sinobackproject_linear", *a)

    def sinobackproject_nearest(self, *a):
        return self._bp("sinobackproject_nearest", *a)

    def pd_backproj_linear(self, *a):
        return self._bp("pd_backproj_linear", *a)

    def pd_backproj_nearest(self, *a):
        return self._bp("pd_backproj_nearest", *a)

    def artstep_linear(self, *a):
        return self._art("artstep_linear", *a)

    def artstep_nearest(self, *a):
        return self._art("artstep_nearest", *a)

    def emstep_linear(self, *a):
        return self._em("emstep_linear", *a)

    def emstep_nearest(self, *a):
        return self._em("emstep_nearest", *a)

    def ellipsoid_proj(self, indsino, frame_vectors, nu, nv, du, dv, u0, v0, ax, ay, az, x0, y0,
                       z0, alpha, beta, att):
        out = np.zeros((nu, nv), self.dt)
        r = self._r
        self._fn("ellipsoid_proj")(_p(out), _p(_i(indsino)), _p(_f(frame_vectors, self.dt)), nu,
                                   nv, r(du), r(dv), r(u0), r(v0), r(ax), r(ay), r(az), r(x0),
                                   r(y0), r(z0), r(alpha), r(beta), r(att))
        return out

    def gen_shape_proj(self, indsino, frame_vectors, nu, nv, du, dv, u0, v0, att, nsurf, xu1, xu2,
                       xu3, yu1, yu2, yu3, zu1, zu2, zu3, x0, y0, z0, nplane, nellipsoid, ax_ell,
                       ay_ell, az_ell, ncyl, ax_cyl, ay_cyl, ncone, ax_cone, ay_cone):
        out = np.zeros((nu, nv), self.dt)
        r = self._r
        keep, tab = _shapes(self, nsurf, (xu1, xu2, xu3, yu1, yu2, yu3, zu1, zu2, zu3, x0, y0, z0),
                            nplane, nellipsoid, (ax_ell, ay_ell, az_ell), ncyl, (ax_cyl, ay_cyl),
                            ncone, (ax_cone, ay_cone))
        self._fn("gen_shape_proj")(_p(out), _p(_i(indsino)), _p(_f(frame_vectors, self.dt)), nu,
                                   nv, r(du), r(dv), r(u0), r(v0), r(att), *tab)
        return out

    # the same arithmetic over host threads (the timed CPU baseline in REAL*4;
    # the FP64 checker of served jobs too large for one core)
    def sinoproj_linear_omp(self, indsino, frame_vectors, ns, nu, nv, du, dv, u0, v0, smat, dx,
                            dy, dz, x0, y0, z0, nx, ny, nz, nthreads):
        out = np.zeros((ns, nu, nv), self.dt)
        r = self._r
        self._fn("sinoproj_linear_omp")(
            _p(out), _p(_i(indsino)), _p(_f(frame_vectors, self.dt)), ns, nu, nv, r(du), r(dv),
            r(u0), r(v0), _p(_f(smat, self.dt)), r(dx), r(dy), r(dz), r(x0), r(y0), r(z0), nx,
            ny, nz, nthreads)
        return out

    def sinobackproject_linear_omp(self, sinomat, indsino, frame_vectors, ns, nu, nv, du, dv, u0,
                                   v0, dx, dy, dz, x0, y0, z0, nx, ny, nz, nthreads):
        out = np.zeros((nx, ny, nz), self.dt)
        r = self._r
        self._fn("sinobackproject_linear_omp")(
            _p(_f(sinomat, self.dt)), _p(_i(indsino)), _p(_f(frame_vectors, self.dt)), ns, nu,
            nv, r(du), r(dv), r(u0), r(v0), _p(out), r(dx), r(dy), r(dz), r(x0), r(y0), r(z0),
            nx, ny, nz, nthreads)
        return out

    def matproj_linear(self, projmats, ns, nu, nv, du, dv, u0, v0, smat, dx, dy, dz, x0, y0, z0,
                       nx, ny, nz):
        out = np.zeros((ns, nu, nv), self.dt)
        r = self._r
        self._fn("matproj_linear")(_p(out), _p(_f(projmats, self.dt)), ns, nu, nv, r(du), r(dv),
                                   r(u0), r(v0), _p(_f(smat, self.dt)), r(dx), r(dy), r(dz),
                                   r(x0), r(y0), r(z0), nx, ny, nz)
        return out


class ViewProj3DTomo(ViewProj3D):
    """view_proj3D_tomo (emil_code/view_proj3D_tomo.f)."""

    def sinoprojz(self, *a):
        return self._proj("sinoprojz", *a)

    def artstepz(self, *a):
        return self._art("artstepz", *a)

    def emstep_linearz(self, *a):
        return self._em("emstep_linearz", *a)

    def artstepz2vol(self, reg_fac, sinomat, indsino, frame_vectors, ns, nu, nv, du, dv, u0, v0,
                     smat, dx, dy, dz, x0, y0, z0, nx, ny, nz, smata, dxa, dya, dza, x0a, y0a,
                     z0a, nxa, nya, nza):
        x = np.array(smat, dtype=self.dt, order="C", copy=True)
        xa = np.array(smata, dtype=self.dt, order="C", copy=True)
        r = self._r
        self._fn("artstepz2vol")(r(reg_fac), _p(_f(sinomat, self.dt)), _p(_i(indsino)),
                                 _p(_f(frame_vectors, self.dt)), ns, nu, nv, r(du), r(dv), r(u0),
                                 r(v0), _p(x), r(dx), r(dy), r(dz), r(x0), r(y0), r(z0), nx, ny,
                                 nz, _p(xa), r(dxa), r(dya), r(dza), r(x0a), r(y0a), r(z0a), nxa,
                                 nya, nza)
        return x, xa

    def artstepz_coloured(self, reg_fac, sinomat, indsino, frame_vectors, ns, nu, nv, du, dv, u0,
                          v0, smat, dx, dy, dz, x0, y0, z0, nx, ny, nz, cu, cv, nthreads=None):
        """artstepz swept in colour order, the rays of a colour on host
        threads; see artstepz_coloured in ct2_oracle_body.h."""
        x = np.array(smat, dtype=self.dt, order="C", copy=True)
        r = self._r
        fn = self._fn("artstepz_coloured")
        fn.restype = None
        fn(r(reg_fac), _p(_f(sinomat, self.dt)), _p(_i(indsino)), _p(_f(frame_vectors, self.dt)),
           ns, nu, nv, r(du), r(dv), r(u0), r(v0), _p(x), r(dx), r(dy), r(dz), r(x0), r(y0),
           r(z0), nx, ny, nz, int(cu), int(cv), int(nthreads or max_threads()))
        return x


class RayProj3D(_Mod):
    """ray_proj3D (emil_code/ray_proj3D.f)."""

    def _proj(self, name, indsino, ray_vectors, nr, smat, dx, dy, dz, x0, y0, z0, nx, ny, nz):
        out = np.zeros((nr,), self.dt)
        r = self._r
        self._fn(name)(_p(out), _p(_i(indsino)), _p(_f(ray_vectors, self.dt)), nr,
                       _p(_f(smat, self.dt)), r(dx), r(dy), r(dz), r(x0), r(y0), r(z0), nx, ny, nz)
        return out

    def sinoproj_linear(self, *a):
        return self._proj("ray_sinoproj_linear", *a)

    def sinoproj_nearest(self, *a):
        return self._proj("ray_sinoproj_nearest", *a)

    def sinobackproject_nearest(self, sinomat, indsino, ray_vectors, nr, dx, dy, dz, x0, y0, z0,
                                nx, ny, nz):
        out = np.zeros((nx, ny, nz), self.dt)
        r = self._r
        self._fn("ray_sinobackproject_nearest")(
            _p(_f(sinomat, self.dt)), _p(_i(indsino)), _p(_f(ray_vectors, self.dt)), nr, _p(out),
            r(dx), r(dy), r(dz), r(x0), r(y0), r(z0), nx, ny, nz)
        return out

    def _art(self, name, reg_fac, sinomat, indsino, ray_vectors, nr, smat, dx, dy, dz, x0, y0,
             z0, nx, ny, nz):
        x = np.array(smat, dtype=self.dt, order="C", copy=True)
        r = self._r
        self._fn(name)(r(reg_fac), _p(_f(sinomat, self.dt)), _p(_i(indsino)),
                       _p(_f(ray_vectors, self.dt)), nr, _p(x), r(dx), r(dy), r(dz), r(x0), r(y0),
                       r(z0), nx, ny, nz)
        return x

    def artstep_linear(self, *a):
        return self._art("ray_artstep_linear", *a)

    def artstep_nearest(self, *a):
        return self._art("ray_artstep_nearest", *a)

    def emstep_nearest(self, sinomat, indsino, ray_vectors, nr, smat, dx, dy, dz, x0, y0, z0, nx,
                       ny, nz):
        x = np.array(smat, dtype=self.dt, order="C", copy=True)
        r = self._r
        self._fn("ray_emstep_nearest")(_p(_f(sinomat, self.dt)), _p(_i(indsino)),
                                       _p(_f(ray_vectors, self.dt)), nr, _p(x), r(dx), r(dy),
                                       r(dz), r(x0), r(y0), r(z0), nx, ny, nz)
        return x

    def ellipsoid_proj(self, indsino, ray_vectors, nr, ax, ay, az, x0, y0, z0, alpha, beta, att):
        out = np.zeros((nr,), self.dt)
        r = self._r
        self._fn("ray_ellipsoid_proj")(_p(out), _p(_i(indsino)), _p(_f(ray_vectors, self.dt)), nr,
                                       r(ax), r(ay), r(az), r(x0), r(y0), r(z0), r(alpha),
                                       r(beta), r(att))
        return out

    def gen_shape_proj(self, indsino, ray_vectors, nr, att, nsurf, xu1, xu2, xu3, yu1, yu2, yu3,
                       zu1, zu2, zu3, x0, y0, z0, nplane, nellipsoid, ax_ell, ay_ell, az_ell, ncyl,
                       ax_cyl, ay_cyl, ncone, ax_cone, ay_cone):
        out = np.zeros((nr,), self.dt)
        keep, tab = _shapes(self, nsurf, (xu1, xu2, xu3, yu1, yu2, yu3, zu1, zu2, zu3, x0, y0, z0),
                            nplane, nellipsoid, (ax_ell, ay_ell, az_ell), ncyl, (ax_cyl, ay_cyl),
                            ncone, (ax_cone, ay_cone))
        self._fn("ray_gen_shape_proj")(_p(out), _p(_i(indsino)), _p(_f(ray_vectors, self.dt)), nr,
                                       self._r(att), *tab)
        return out


class TotalVar(_Mod):
    """totalvar (emil_code/totalvar.f)."""

    def total_var3d(self, ambdala, smat, nx, ny, nz):
        fn = self._fn("total_var3d", self.real)
        return float(fn(self._r(ambdala), _p(_f(smat, self.dt)), nx, ny, nz))

    def total_var_grad3d(self, ambdala, smat, nx, ny, nz, normalizeq):
        out = np.zeros((nx, ny, nz), self.dt)
        fn = self._fn("total_var_grad3d", self.real)
        bobo = fn(self._r(ambdala), _p(out), _p(_f(smat, self.dt)), nx, ny, nz, int(normalizeq))
        return out, float(bobo)

    def gmi(self, smat, nx, ny, nz):
        out = np.zeros((nx, ny, nz), self.dt)
        self._fn("gmi")(_p(out), _p(_f(smat, self.dt)), nx, ny, nz)
        return out

    def calc_lp(self, p, smat, nx, ny, nz):
        fn = self._fn("calc_lp", self.real)
        return float(fn(self._r(p), _p(_f(smat, self.dt)), nx, ny, nz))

    def total_var3d_p(self, p, smat, nx, ny, nz):
        fn = self._fn("total_var3d_p", self.real)
        return float(fn(self._r(p), _p(_f(smat, self.dt)), nx, ny, nz))

    def total_dvar3d_p(self, p, smat, nx, ny, nz, dx, dy, dz):
        fn = self._fn("total_dvar3d_p", self.real)
        r = self._r
        return float(fn(r(p), _p(_f(smat, self.dt)), nx, ny, nz, r(dx), r(dy), r(dz)))

    def _pgrad(self, name, ppp, smat, nx, ny, nz, extra, normalizeq):
        out = np.zeros((nx, ny, nz), self.dt)
        fn = self._fn(name, self.real)
        bobo = fn(self._r(ppp), _p(out), _p(_f(smat, self.dt)), nx, ny, nz,
                  *[self._r(v) for v in extra], int(normalizeq))
        return out, float(bobo)

    def lp_grad3d(self, ppp, smat, nx, ny, nz, normalizeq):
        return self._pgrad("lp_grad3d", ppp, smat, nx, ny, nz, (), normalizeq)

    def total_p_var_grad3d(self, ppp, smat, nx, ny, nz, normalizeq):
        return self._pgrad("total_p_var_grad3d", ppp, smat, nx, ny, nz, (), normalizeq)

    def total_p_dvar_grad3d(self, ppp, smat, nx, ny, nz, dx, dy, dz, normalizeq):
        return self._pgrad("total_p_dvar_grad3d", ppp, smat, nx, ny, nz, (dx, dy, dz),
                           normalizeq)


class Radon3D(_Mod):
    """radon3D (emil_code/radon3D.f)."""

    def spherical_radon_linear(self, fov, indradon, source_locations, nsa, nsb, ns, nr, dr, r0,
                               smat, dx, dy, dz, x0, y0, z0, nx, ny, nz):
        out = np.zeros((nsa, nsb, nr), self.dt)
        r = self._r
        self._fn("spherical_radon_linear")(r(fov), _p(out), _p(_i(indradon)),
                                           _p(_f(source_locations, self.dt)), nsa, nsb, ns, nr,
                                           r(dr), r(r0), _p(_f(smat, self.dt)), r(dx), r(dy),
                                           r(dz), r(x0), r(y0), r(z0), nx, ny, nz)
        return out

    def artstep_linear(self, reg_fac, fov, radonmat, indradon, source_locations, nsa, nsb, ns, nr,
                       dr, r0, smat, dx, dy, dz, x0, y0, z0, nx, ny, nz):
        x = np.array(smat, dtype=self.dt, order="C", copy=True)
        r = self._r
        self._fn("radon_artstep_linear")(r(reg_fac), r(fov), _p(_f(radonmat, self.dt)),
                                         _p(_i(indradon)), _p(_f(source_locations, self.dt)), nsa,
                                         nsb, ns, nr, r(dr), r(r0), _p(x), r(dx), r(dy), r(dz),
                                         r(x0), r(y0), r(z0), nx, ny, nz)
        return x


class Tomo3DFort(_Mod):
    """tomo3Dfort (emil_code/tomo3DfortranAux.f)."""

    def ellipsoid_embed(self, nx, ny, nz, dx, dy, dz, x0i, y0i, z0i, att, alpha, beta, x0, y0, z0,
                        ax, ay, az):
        out = np.zeros((nx, ny, nz), self.dt)
        r = self._r
        self._fn("ellipsoid_embed")(_p(out), nx, ny, nz, r(dx), r(dy), r(dz), r(x0i), r(y0i),
                                    r(z0i), r(att), r(alpha), r(beta), r(x0), r(y0), r(z0), r(ax),
                                    r(ay), r(az))
        return out

    def shape_root(self, kind, xs, ys, zs, xb, yb, zb, a=1.0, b=1.0, c=1.0,
                   tr=(-1e8, 1e8)):
        """root_plane / root_ellipsoid / root_cylinder / root_cone (kind 0..3)
        of emil_code/view_proj3D.f:11-170 -> troot (2,)."""
        out = np.array(tr, self.dt)
        r = self._r
        self._fn("shape_root")(int(kind), _p(out), r(xs), r(ys), r(zs), r(xb), r(yb), r(zb), r(a),
                               r(b), r(c))
        return out

    def gen_obj_embed(self, nx, ny, nz, dx, dy, dz, x0i, y0i, z0i, att, nsurf, xu1, xu2, xu3,
                      yu1, yu2, yu3, zu1, zu2, zu3, x0, y0, z0, nplane, nellipsoid, ax_ell, ay_ell,
                      az_ell, ncyl, ax_cyl, ay_cyl, ncone, ax_cone, ay_cone):
        out = np.zeros((nx, ny, nz), self.dt)
        r = self._r
        keep, tab = _shapes(self, nsurf, (xu1, xu2, xu3, yu1, yu2, yu3, zu1, zu2, zu3, x0, y0, z0),
                            nplane, nellipsoid, (ax_ell, ay_ell, az_ell), ncyl, (ax_cyl, ay_cyl),
                            ncone, (ax_cone, ay_cone))
        self._fn("gen_obj_embed")(_p(out), nx, ny, nz, r(dx), r(dy), r(dz), r(x0i), r(y0i),
                                  r(z0i), r(att), *tab)
        return out

    def gen_obj_voxval(self, x, y, z, att, nsurf, alpha, beta, gam, x0, y0, z0, nplane,
                       nellipsoid, ax_ell, ay_ell, az_ell, ncyl, ax_cyl, ay_cyl, ncone, ax_cone,
                       ay_cone):
        r = self._r
        keep, tab = _shapes(self, nsurf, (alpha, beta, gam, x0, y0, z0) + ((),) * 6, nplane,
                            nellipsoid, (ax_ell, ay_ell, az_ell), ncyl, (ax_cyl, ay_cyl), ncone,
                            (ax_cone, ay_cone))
        fr = keep[0]
        rows = [fr[k].ctypes.data_as(ctypes.c_void_p) for k in range(6)]
        fn = self._fn("gen_obj_voxval", self.real)
        return float(fn(r(x), r(y), r(z), r(att), int(nsurf), *rows, int(nplane),
                        int(nellipsoid), tab[4], int(ncyl), tab[6], int(ncone), tab[8]))

    def framer(self, x, y, z, alpha, beta, gam, x0, y0, z0):
        out = np.zeros(3, self.dt)
        r = self._r
        self._fn("framer")(_p(out), r(x), r(y), r(z), r(alpha), r(beta), r(gam), r(x0), r(y0),
                           r(z0))
        return out

    def ellipse_voxval(self, x, y, z, att, alpha, beta, x0, y0, z0, ax, ay, az):
        r = self._r
        fn = self._fn("ellipse_voxval", self.real)
        return float(fn(r(x), r(y), r(z), r(att), r(alpha), r(beta), r(x0), r(y0), r(z0), r(ax),
                        r(ay), r(az)))

    def sinoscale(self, sinomat, frame_vectors, ns, nu, nv, du, dv, u0, v0):
        x = np.array(sinomat, dtype=self.dt, order="C", copy=True)
        r = self._r
        self._fn("sinoscale")(_p(x), _p(_f(frame_vectors, self.dt)), ns, nu, nv, r(du), r(dv),
                              r(u0), r(v0))
        return x

    def sinoave(self, sinomat, ns, nu, nv, nss, nus, nvs, nds, ndu, ndv, nws, nwu, nwv):
        out = np.zeros((nss, nus, nvs), self.dt)
        self._fn("sinoave")(_p(_f(sinomat, self.dt)), _p(out), ns, nu, nv, nss, nus, nvs, nds,
                            ndu, ndv, nws, nwu, nwv)
        return out

    def sinodist(self, sinoin, ns, nu, nv, nss, nus, nvs, nds, ndu, ndv, nws, nwu, nwv):
        out = np.zeros((ns, nu, nv), self.dt)
        self._fn("sinodist")(_p(out), _p(_f(sinoin, self.dt)), ns, nu, nv, nss, nus, nvs, nds,
                             ndu, ndv, nws, nwu, nwv)
        return out


class TomoScale(_Mod):
    """tomoscale (emil_code/tomoscale.f)."""

    def _mag(self, name, smat, nx, ny, nz, x0, y0, z0, xlen, ylen, zlen, xs, ys, zs):
        out = np.zeros((nx, ny, nz), self.dt)
        r = self._r
        self._fn(name)(_p(out), _p(_f(smat, self.dt)), nx, ny, nz, r(x0), r(y0), r(z0), r(xlen),
                       r(ylen), r(zlen), r(xs), r(ys), r(zs))
        return out

    def tomovolmag(self, *a):
        return self._mag("tomovolmag", *a)

    def tomovolmagt(self, *a):
        return self._mag("tomovolmagt", *a)


view_proj3D = ViewProj3D(np.float32)
view_proj3D_tomo = ViewProj3DTomo(np.float32)
ray_proj3D = RayProj3D(np.float32)
totalvar = TotalVar(np.float32)
radon3D = Radon3D(np.float32)
tomo3Dfort = Tomo3DFort(np.float32)
tomo3Dfort_f64 = Tomo3DFort(np.float64)
tomoscale = TomoScale(np.float32)
tomoscale_f64 = TomoScale(np.float64)

view_proj3D_f64 = ViewProj3D(np.float64)
view_proj3D_tomo_f64 = ViewProj3DTomo(np.float64)
ray_proj3D_f64 = RayProj3D(np.float64)
totalvar_f64 = TotalVar(np.float64)
radon3D_f64 = Radon3D(np.float64)


def max_threads():
    return int(lib().ora_max_threads())
