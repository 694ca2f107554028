"""ctypes binding of ``libct2b200.so`` (the C ABI declared in include/ct2b200.h).

Every entry point returns a status code; :func:`call` turns a non-zero code
into the exception the reference's f2py layer would raise for the same class
of problem (``ValueError`` for argument errors) or ``RuntimeError`` for CUDA
failures.  The library must exist: there is no CPU fallback.
"""
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "libct2b200.so")

CT2_OK, CT2_EINVAL, CT2_ECUDA, CT2_ENOMEM, CT2_ETIMEOUT = 0, 1, 2, 3, 4

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_D = ctypes.c_double
_L = ctypes.c_longlong
_CODES = {"P": _P, "i": _I, "f": _F, "d": _D, "l": _L}

# Argument signatures of the C ABI, one letter per argument
# (P pointer, i int, f float, d double, l int64).  The device variant of a
# host entry point takes the same arguments plus a trailing stream pointer.
VIEW = "PPPiiiffff"       # sinomat/indsino/frame_vectors + ns,nu,nv,du,dv,u0,v0
GRID = "ffffffiii"        # dx,dy,dz,x0,y0,z0,nx,ny,nz
# surface table of gen_object: nsurf, xu1..z0, nplane, nellipsoid + 3 semi-axis
# arrays, ncyl + 2, ncone + 2
SHAPES = "i" + "P" * 12 + "i" + "iPPP" + "iPP" + "iPP"
SIGS = {
    "view_proj3D_sinoproj_linear": VIEW + "P" + GRID,
    "view_proj3D_sinoproj_nearest": VIEW + "P" + GRID,
    "view_proj3D_sinobackproject_linear": VIEW + "P" + GRID,
    "view_proj3D_sinobackproject_nearest": VIEW + "P" + GRID,
    "view_proj3D_emstep_linear": VIEW + "P" + GRID,
    "view_proj3D_emstep_nearest": VIEW + "P" + GRID,
    "view_proj3D_tomo_sinoprojz": VIEW + "P" + GRID,
    "view_proj3D_tomo_emstep_linearz": VIEW + "P" + GRID,
    "ray_proj3D_sinoproj_linear": "PPPiP" + GRID,
    "ray_proj3D_sinoproj_nearest": "PPPiP" + GRID,
    "ray_proj3D_sinobackproject_nearest": "PPPiP" + GRID,
    "ray_proj3D_emstep_nearest": "PPPiP" + GRID,
    "view_proj3D_artstep_linear": "f" + VIEW + "P" + GRID,
    "view_proj3D_artstep_nearest": "f" + VIEW + "P" + GRID,
    "view_proj3D_tomo_artstepz": "f" + VIEW + "P" + GRID,
    "view_proj3D_tomo_artstepz2vol": "f" + VIEW + "P" + GRID + "P" + GRID,
    "ray_proj3D_artstep_linear": "fPPPiP" + GRID,
    "ray_proj3D_artstep_nearest": "fPPPiP" + GRID,
    "view_proj3D_pd_backproj_linear": VIEW + "P" + GRID,
    "view_proj3D_pd_backproj_nearest": VIEW + "P" + GRID,
    "view_proj3D_ellipsoid_proj": "PPPiiffff" + "fffffffff",
    "ray_proj3D_ellipsoid_proj": "PPPi" + "fffffffff",
    "tomo3Dfort_ellipsoid_embed": "Piiiffffff" + "fff" + "ffffff",
    "totalvar_total_var_grad3d": "fPPiiiiP",
    "totalvar_total_var3d": "fPiiiP",
    "totalvar_gmi": "PPiii",
    "totalvar_calc_lp": "fPiiiP",
    "totalvar_total_var3d_p": "fPiiiP",
    "totalvar_total_dvar3d_p": "fPiiifffP",
    "totalvar_lp_grad3d": "fPPiiiiP",
    "totalvar_total_p_var_grad3d": "fPPiiiiP",
    "totalvar_total_p_dvar_grad3d": "fPPiiifffiP",
    "radon3D_spherical_radon_linear": "fPPPiiiiffP" + GRID,
    "radon3D_artstep_linear": "ffPPPiiiiffP" + GRID,
    "tomo3Dfort_sinoscale": "PPiiiffff",
    "tomo3Dfort_sinoave": "PPiiiiiiiiiiii",
    "tomo3Dfort_sinodist": "PPiiiiiiiiiiii",
    "tomoscale_tomovolmag": "PPiiifffffffff",
    "tomoscale_tomovolmagt": "PPiiifffffffff",
    "view_proj3D_matproj_linear": "PPiiiffffP" + GRID,
    "view_proj3D_gen_shape_proj": "PPPiiffff" + "f" + SHAPES,
    "ray_proj3D_gen_shape_proj": "PPPi" + "f" + SHAPES,
    "tomo3Dfort_gen_obj_embed": "Piiiffffff" + "f" + SHAPES,
    "fdk_sino_weight": "PPPiii",
    "fdk_sino_filter": "PPPPiiii",
    "fdk_backproj_linear": "PiiiffffffffPPPPiiP",
}

# Entry points with a device form only (no host-pointer twin).
DEV_ONLY = {
    "view_proj3D_emratio_linear": "P" + VIEW + "P" + GRID + "P",
    # several volumes through one geometry (no indicator)
    "view_proj3D_sinoproj_linear_many": "iPP" + "iiiffff" + "P" + GRID + "P",
    "view_proj3D_sinobackproject_linear_many": "iPP" + "iiiffff" + "P" + GRID + "P",
    "totalvar_total_var_grad3d_noalloc": "fPPiiiiPP",
    # precision form: storage-type codes follow each array (CT2_F32/BF16/F16)
    "prec_project": "PiPP" + "iiiffff" + "Pi" + GRID + "iP",
    "prec_emratio": "PPiPP" + "iiiffff" + "Pi" + GRID + "iP",
    "prec_backproject": "PiPP" + "iiiffff" + "PP" + GRID + "iP",
    "prec_em_tv_update": "PiPPiiiffP",
    "prec_art_sweep": "fPiPP" + "iiiffff" + "Pi" + GRID + "iiiP",
    "prec_art_tv_update": "PiPPiiifiP",
    "phantom_project": "PPiPiiiffffP",
}

# Host-only entry points (no device twin).
HOST_ONLY = {
    "prec_art_colouring": "Piiiffff" + GRID + "PP",
    "wait_timeouts": "Pi",
    "launch_count": "Pi",
    "set_backprojector": "i",
    "wait_selftest": "i",
    "tomo3Dfort_ellipse_voxval": "P" + "fffffffffff" + "f",
    "tomo3Dfort_step": "Pf",
    "tomo3Dfort_framer": "P" + "fffffffff",
    "tomo3Dfort_gen_obj_voxval": "Pffff" + "i" + "P" * 6 + "i" + "iPPP" + "iPP" + "iPP",
    # batched MLEM+TV iteration of several reconstructions (ct2b200.batch)
    "batch_create": "iP",
    "batch_destroy": "P",
    "batch_set": "Pi" + "PPPPPP" + "iiiffff" + GRID + "fP",
    "batch_clear": "PiP",
    "batch_commit": "PPP",
    "batch_em_iteration": "PP",
}

_lock = threading.Lock()
_lib = None


class LibraryMissing(RuntimeError):
    pass


def lib():
    """Load the CUDA library (build it first with ct-2_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise LibraryMissing(
                "libct2b200.so is not built (%s); run `python ct-2_b200/build.py` -- the "
                "reconstruction kernels exist only as CUDA code" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        L.ct2_last_error.restype = ctypes.c_char_p
        L.ct2_last_error.argtypes = []
        L.ct2_version.restype = ctypes.c_char_p
        L.ct2_version.argtypes = []
        for name, sig in SIGS.items():
            for prefix, extra in (("ct2_", ""), ("ct2_dev_", "P")):
                fn = getattr(L, prefix + name)
                fn.argtypes = [_CODES[c] for c in sig + extra]
                fn.restype = _I
        for name, sig in DEV_ONLY.items():
            fn = getattr(L, "ct2_dev_" + name)
            fn.argtypes = [_CODES[c] for c in sig]
            fn.restype = _I
        for name, sig in HOST_ONLY.items():
            fn = getattr(L, "ct2_" + name)
            fn.argtypes = [_CODES[c] for c in sig]
            fn.restype = _I
        _lib = L
        return _lib


def register(name, sig, restype=_I, device_variant=True):
    """Declare the signature of an additional entry point (used by modules
    that bind entry points beyond the table above)."""
    SIGS[name] = sig
    L = lib()
    for prefix, extra in (("ct2_", ""), ("ct2_dev_", "P")) if device_variant else (("ct2_", ""),):
        fn = getattr(L, prefix + name)
        fn.argtypes = [_CODES[c] for c in sig + extra]
        fn.restype = restype


def last_error():
    return lib().ct2_last_error().decode(errors="replace")


def check(rc, name):
    if rc == CT2_OK:
        return
    msg = "%s: %s" % (name, last_error())
    if rc == CT2_EINVAL:
        raise ValueError(msg)
    if rc == CT2_ENOMEM:
        raise MemoryError(msg)
    if rc == CT2_ETIMEOUT:
        raise TimeoutError(msg)
    raise RuntimeError(msg)


def call(name, *args):
    """Call ``ct2_<name>`` and raise on a non-zero status."""
    fn = getattr(lib(), "ct2_" + name)
    rc = fn(*args)
    check(rc, "ct2_" + name)


def exported_symbols():
    """Names declared in include/ct2b200.h that the loaded library exports."""
    out = []
    for name in SIGS:
        for prefix in ("ct2_", "ct2_dev_"):
            if hasattr(lib(), prefix + name):
                out.append(prefix + name)
    return out
