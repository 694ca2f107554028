"""Argument marshalling shared by the drop-in modules.

The reference's f2py wrappers take positional arguments in the Fortran order
(intent(out) arrays omitted and returned), convert array arguments to the
Fortran type (REAL*4 / INTEGER) and raise ``ValueError`` when a shape does not
match its dimension arguments.  The drop-ins do the same and then choose the
execution path by where the data lives:

* NumPy (or anything array-like) -> the host C ABI entry point: inputs are
  copied to the GPU, the kernel runs, outputs come back as C-contiguous
  ``float32`` NumPy arrays with the reference's logical indexing;
* CUDA ``torch.Tensor`` -> the ``ct2_dev_`` entry point on the tensor's device
  and current stream, zero-copy; outputs are CUDA tensors.

intent(in,out) arrays are returned as new arrays; the caller's array is not
modified, as with f2py for C-ordered input.
"""
import numpy as np

from . import _lib

try:  # torch is only needed for the device path
    import torch
except Exception:  # pragma: no cover
    torch = None


def is_cuda(x):
    return torch is not None and isinstance(x, torch.Tensor) and x.is_cuda


def _writable(a):
    """torch refuses to wrap read-only NumPy memory; copy only then."""
    return a if a.flags.writeable else a.copy()


class Marshal:
    """Converts one call's arrays for the host or the device entry point."""

    def __init__(self, name, arrays):
        self.name = name
        devs = [a.device for a in arrays if is_cuda(a)]
        self.dev = bool(devs)
        self.device = devs[0] if devs else None
        self.keep = []

    # ---- conversions ---------------------------------------------------
    def _shape_check(self, arr_shape, shape, what):
        if shape is not None and tuple(arr_shape) != tuple(int(s) for s in shape):
            raise ValueError("%s: argument %s has shape %s, expected %s" %
                             (self.name, what, tuple(arr_shape), tuple(int(s) for s in shape)))

    def f32(self, x, shape, what):
        if self.dev:
            if not is_cuda(x):
                x = torch.as_tensor(_writable(np.asarray(x, dtype=np.float32)),
                                    device=self.device)
            t = x.to(device=self.device, dtype=torch.float32).contiguous()
            self._shape_check(t.shape, shape, what)
            self.keep.append(t)
            return t
        a = np.asarray(x, dtype=np.float32)
        # a scalar stands for a one-element array only (ascontiguousarray
        # below turns it into shape (1,))
        if (shape is not None and a.ndim == 0 and len(shape) > 0 and
                int(np.prod([int(s) for s in shape])) != 1):
            raise ValueError("%s: argument %s must be an array" % (self.name, what))
        a = np.ascontiguousarray(a)
        self._shape_check(a.shape, shape, what)
        self.keep.append(a)
        return a

    def i32(self, x, shape, what):
        if x is None:
            return None
        if self.dev:
            if not is_cuda(x):
                x = torch.as_tensor(_writable(np.asarray(x)), device=self.device)
            t = x.to(device=self.device, dtype=torch.int32).contiguous()
            self._shape_check(t.shape, shape, what)
            self.keep.append(t)
            return t
        a = np.ascontiguousarray(np.asarray(x).astype(np.int32, copy=False))
        self._shape_check(a.shape, shape, what)
        self.keep.append(a)
        return a

    def out(self, shape, zero=False):
        shape = tuple(int(s) for s in shape)
        if self.dev:
            t = (torch.zeros if zero else torch.empty)(shape, dtype=torch.float32,
                                                       device=self.device)
            self.keep.append(t)
            return t
        a = np.zeros(shape, np.float32)
        self.keep.append(a)
        return a

    def copy(self, x, shape, what):
        """intent(in,out): a private float32 copy the kernel may update."""
        if self.dev:
            t = self.f32(x, shape, what).clone()
            self.keep.append(t)
            return t
        a = np.array(self.f32(x, shape, what), dtype=np.float32, order="C", copy=True)
        self.keep.append(a)
        return a

    @staticmethod
    def ptr(a):
        if a is None:
            return None
        if torch is not None and isinstance(a, torch.Tensor):
            return a.data_ptr() if a.numel() else None
        return a.ctypes.data if a.size else None

    # ---- the call --------------------------------------------------------
    def run(self, entry, *args):
        conv = [self.ptr(a) if isinstance(a, np.ndarray) or
                (torch is not None and isinstance(a, torch.Tensor)) else a for a in args]
        if self.dev:
            with torch.cuda.device(self.device):
                stream = torch.cuda.current_stream(self.device).cuda_stream
                fn = getattr(_lib.lib(), "ct2_dev_" + entry)
                rc = fn(*conv, stream)
            _lib.check(rc, "ct2_dev_" + entry)
        else:
            fn = getattr(_lib.lib(), "ct2_" + entry)
            rc = fn(*conv)
            _lib.check(rc, "ct2_" + entry)


def ints(*vals):
    return [int(v) for v in vals]


def floats(*vals):
    return [float(v) for v in vals]


SHAPE_FRAMES = ("xu1", "xu2", "xu3", "yu1", "yu2", "yu3", "zu1", "zu2", "zu3", "x0", "y0", "z0")


def shape_table(m, nsurf, frames, nplane, nellipsoid, ell, ncyl, cyl, ncone, cone):
    """The gen_object surface table as the C ABI takes it: the twelve frame
    arrays (nsurf entries each), then each kind's count and semi-axis arrays
    (as many entries as the count).  Shapes are checked as f2py does."""
    nsurf, nplane, nellipsoid, ncyl, ncone = ints(nsurf, nplane, nellipsoid, ncyl, ncone)
    args = [nsurf] + [m.f32(a, (nsurf,), n) for a, n in zip(frames, SHAPE_FRAMES)]
    args += [nplane]
    args += [nellipsoid] + [m.f32(a, (nellipsoid,), n)
                            for a, n in zip(ell, ("ax_ell", "ay_ell", "az_ell"))]
    args += [ncyl] + [m.f32(a, (ncyl,), n) for a, n in zip(cyl, ("ax_cyl", "ay_cyl"))]
    args += [ncone] + [m.f32(a, (ncone,), n) for a, n in zip(cone, ("ax_cone", "ay_cone"))]
    return args

