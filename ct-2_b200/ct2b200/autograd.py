"""torch.autograd functions over the GPU kernels (the differentiable form).

* ``project(x, geom)``: A x with the matched backprojector as its backward
  (exact transpose of the forward: same samples, same weights).
* ``data_fit(x, y, geom)``: ||A x - y||^2.  Keeps only x and y; the backward
  projects again and backprojects the residual, so no projection is held
  between forward and backward.  ``keep_residual=True`` keeps the residual
  instead (one projection fewer per step; the projector is deterministic,
  so the residual is the same bit for bit, and so is the gradient with the
  default gather backprojector -- the scatter form, ct2_set_backprojector(1),
  sums in the order of its L2 reductions).
* ``total_variation(x, lam)``: the reference's smoothed TV
  (totalvar.total_var3d) with the TV-gradient kernel
  (totalvar.total_var_grad3d, unnormalised) as its backward.

Volumes are (nx, ny, nz) or batched (B, nx, ny, nz) float32 CUDA tensors.
"""
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib


@dataclass(frozen=True)
class ConeGeometry:
    """A view geometry (frame vectors + flat detector) and a volume grid."""
    frame_vectors: torch.Tensor  # (ns, 18) float32 on the device
    ns: int
    nu: int
    nv: int
    du: float
    dv: float
    u0: float
    v0: float
    grid: tuple  # (dx, dy, dz, x0, y0, z0, nx, ny, nz)

    @staticmethod
    def from_scan(scan, vol, device):
        fv = torch.as_tensor(np.ascontiguousarray(scan.frame_vectors, np.float32), device=device)
        return ConeGeometry(fv, int(scan.ns), int(scan.nu), int(scan.nv), float(scan.du),
                            float(scan.dv), float(scan.u0), float(scan.v0), tuple(vol.grid))

    @property
    def vol_shape(self):
        return tuple(int(v) for v in self.grid[6:9])

    @property
    def sino_shape(self):
        return (self.ns, self.nu, self.nv)


def _stream(t):
    return torch.cuda.current_stream(t.device).cuda_stream


def _grid_args(g):
    return [float(v) for v in g[:6]] + [int(v) for v in g[6:]]


def _view_args(geom):
    return [geom.ns, geom.nu, geom.nv, geom.du, geom.dv, geom.u0, geom.v0]


def forward_project(x, geom, out=None):
    """A x for one volume (nx, ny, nz) on the device (no autograd)."""
    x = x.contiguous()
    if out is None:
        out = torch.empty(geom.sino_shape, dtype=torch.float32, device=x.device)
    rc = _lib.lib().ct2_dev_view_proj3D_sinoproj_linear(
        out.data_ptr(), None, geom.frame_vectors.data_ptr(), *_view_args(geom), x.data_ptr(),
        *_grid_args(geom.grid), _stream(x))
    _lib.check(rc, "ct2_dev_view_proj3D_sinoproj_linear")
    return out


def back_project(y, geom, out=None):
    """A^T y for one sinogram (ns, nu, nv) on the device (no autograd)."""
    y = y.contiguous()
    if out is None:
        out = torch.empty(geom.vol_shape, dtype=torch.float32, device=y.device)
    rc = _lib.lib().ct2_dev_view_proj3D_sinobackproject_linear(
        y.data_ptr(), None, geom.frame_vectors.data_ptr(), *_view_args(geom), out.data_ptr(),
        *_grid_args(geom.grid), _stream(y))
    _lib.check(rc, "ct2_dev_view_proj3D_sinobackproject_linear")
    return out


def forward_project_many(xs, geom, out=None):
    """A x for a batch of volumes (B, nx, ny, nz) through one geometry, each
    kernel launched once for the whole batch; every volume's projection
    equals forward_project of it bit for bit."""
    xs = xs.contiguous()
    if out is None:
        out = torch.empty((xs.shape[0],) + tuple(geom.sino_shape), dtype=torch.float32,
                          device=xs.device)
    rc = _lib.lib().ct2_dev_view_proj3D_sinoproj_linear_many(
        int(xs.shape[0]), out.data_ptr(), geom.frame_vectors.data_ptr(), *_view_args(geom),
        xs.data_ptr(), *_grid_args(geom.grid), _stream(xs))
    _lib.check(rc, "ct2_dev_view_proj3D_sinoproj_linear_many")
    return out


def back_project_many(ys, geom, out=None):
    """A^T y for a batch of sinograms (B, ns, nu, nv), each kernel launched
    once for the whole batch; every volume equals back_project of its
    sinogram bit for bit."""
    ys = ys.contiguous()
    if out is None:
        out = torch.empty((ys.shape[0],) + tuple(geom.vol_shape), dtype=torch.float32,
                          device=ys.device)
    rc = _lib.lib().ct2_dev_view_proj3D_sinobackproject_linear_many(
        int(ys.shape[0]), ys.data_ptr(), geom.frame_vectors.data_ptr(), *_view_args(geom),
        out.data_ptr(), *_grid_args(geom.grid), _stream(ys))
    _lib.check(rc, "ct2_dev_view_proj3D_sinobackproject_linear_many")
    return out


class _Project(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, geom):
        ctx.geom = geom
        with torch.no_grad():
            if x.dim() == 3:
                return forward_project(x.float(), geom)
            return forward_project_many(x.float(), geom)

    @staticmethod
    def backward(ctx, gy):
        geom = ctx.geom
        if gy.dim() == 3:
            return back_project(gy.float(), geom), None
        return back_project_many(gy.float(), geom), None


def project(x, geom):
    return _Project.apply(x, geom)


class _DataFit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, y, geom, keep_residual):
        ctx.geom = geom
        ctx.keep = keep_residual
        with torch.no_grad():
            xs = x if x.dim() == 4 else x[None]
            ys = y if y.dim() == 4 else y[None]
            total = torch.zeros((), dtype=torch.float64, device=x.device)
            r = forward_project_many(xs.float(), geom) - ys
            for b in range(xs.shape[0]):
                total = total + torch.sum(r[b].double() * r[b].double())
        if keep_residual:
            ctx.save_for_backward(r)
        else:
            ctx.save_for_backward(x, y)
        ctx.batched = x.dim() == 4
        return total  # FP64: a float32 loss would round away small changes

    @staticmethod
    def backward(ctx, g):
        geom = ctx.geom
        if ctx.keep:
            (res,) = ctx.saved_tensors
        else:
            x, y = ctx.saved_tensors
            xs = x if x.dim() == 4 else x[None]
            ys = y if y.dim() == 4 else y[None]
            # projected again: the projector is deterministic (one thread
            # per ray, a fixed sample order), so this equals the forward's
            # residual bit for bit
            res = forward_project_many(xs.float(), geom) - ys
        gx = back_project_many(res, geom) * (2.0 * g).float()
        return (gx if ctx.batched else gx[0]), None, None, None


def data_fit(x, y, geom, keep_residual=False):
    """||A x - y||^2 summed over the batch, accumulated and returned in FP64.

    keep_residual: False (the default) keeps only x and y and projects again
    in the backward, so nothing of the projection is held between forward
    and backward; True keeps A x - y (one sinogram per volume) and the
    backward only backprojects it (one projection fewer per step)."""
    return _DataFit.apply(x, y, geom, keep_residual)


def _tv_value(x, lam):
    nx, ny, nz = (int(v) for v in x.shape)
    out = torch.empty(1, dtype=torch.float32, device=x.device)
    rc = _lib.lib().ct2_dev_totalvar_total_var3d(float(lam), x.data_ptr(), nx, ny, nz,
                                                 out.data_ptr(), _stream(x))
    _lib.check(rc, "ct2_dev_totalvar_total_var3d")
    return out[0]


def _tv_grad(x, lam):
    nx, ny, nz = (int(v) for v in x.shape)
    g = torch.empty_like(x)
    bobo = torch.empty(1, dtype=torch.float32, device=x.device)
    rc = _lib.lib().ct2_dev_totalvar_total_var_grad3d(float(lam), g.data_ptr(), x.data_ptr(), nx,
                                                      ny, nz, 0, bobo.data_ptr(), _stream(x))
    _lib.check(rc, "ct2_dev_totalvar_total_var_grad3d")
    return g


class _TV(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, lam):
        ctx.lam = float(lam)
        ctx.save_for_backward(x)
        with torch.no_grad():
            xs = x if x.dim() == 4 else x[None]
            v = sum(_tv_value(xs[b].float().contiguous(), lam) for b in range(xs.shape[0]))
        return v

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        xs = x if x.dim() == 4 else x[None]
        gx = torch.stack([_tv_grad(xs[b].float().contiguous(), ctx.lam) for b in range(xs.shape[0])])
        gx = gx * g
        return (gx if x.dim() == 4 else gx[0]), None


def total_variation(x, lam=0.0):
    """Smoothed TV (+ lam * L1) summed over the batch, with its gradient kernel."""
    return _TV.apply(x, lam)
