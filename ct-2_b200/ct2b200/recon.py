"""Device-resident MLEM+TV iteration shared by the reconstruction workloads
(the diagnostic pipeline, the served stream).

One iteration: ratio = y / (A x < 1e-5 ? 1 : A x) (emstep_linear's clamp,
emil_code/view_proj3D.f:2801-2827), x_EM = x * A^T ratio / A^T 1 with the
sensitivity A^T 1 cached once per geometry, then the TV step of the
reconstruction drivers x <- max(0, x_EM - w ||x_EM - x|| g / ||g||), g the
TV gradient (totalvar.total_var_grad3d, emil_code/totalvar.f:476-602), the
norms summed in FP64 (||g|| < 1e-5 -> 1).

Kernels per iteration: the projector writes the ratio in its epilogue (the
projection itself is never stored), the matched backprojector, then four
element-wise/stencil passes (x_EM with the FP64 partials of ||x_EM - x||,
the partials of ||g||, the scale, max(0, x_EM - scale * g)).
"""
import torch

from . import _lib
from .autograd import _grid_args, _view_args, back_project, forward_project

CT2_F32 = 0

EM_SMALL = 0.00001  # view_proj3D.f emstep_linear clamp
TV_WEIGHT = 0.002


def tv_grad_normalised(x):
    nx, ny, nz = (int(v) for v in x.shape)
    g = torch.empty_like(x)
    bobo = torch.empty(1, dtype=torch.float32, device=x.device)
    rc = _lib.lib().ct2_dev_totalvar_total_var_grad3d(
        0.0, g.data_ptr(), x.data_ptr(), nx, ny, nz, 1, bobo.data_ptr(),
        torch.cuda.current_stream(x.device).cuda_stream)
    _lib.check(rc, "ct2_dev_totalvar_total_var_grad3d")
    return g


def em_ratio(x, y, geom, out):
    """out = y / (A x < 1e-5 ? 1 : A x), written by the projector."""
    rc = _lib.lib().ct2_dev_view_proj3D_emratio_linear(
        out.data_ptr(), y.data_ptr(), None, geom.frame_vectors.data_ptr(), *_view_args(geom),
        x.data_ptr(), *_grid_args(geom.grid), torch.cuda.current_stream(x.device).cuda_stream)
    _lib.check(rc, "ct2_dev_view_proj3D_emratio_linear")
    return out


def em_tv_update(x, ws, sens, tv_weight):
    """x <- max(0, xe - w ||xe - x|| g / ||g||) with xe = x * ws / sens
    (sens < 1e-5 -> 1), in place; ws is left holding xe."""
    nx, ny, nz = (int(v) for v in x.shape)
    rc = _lib.lib().ct2_dev_prec_em_tv_update(
        x.data_ptr(), CT2_F32, ws.data_ptr(), sens.data_ptr(), nx, ny, nz, EM_SMALL,
        float(tv_weight), torch.cuda.current_stream(x.device).cuda_stream)
    _lib.check(rc, "ct2_dev_prec_em_tv_update")


def sensitivity(geom, device):
    """A^T 1 with the EM clamp applied (values < 1e-5 -> 1)."""
    ones = torch.ones(geom.sino_shape, dtype=torch.float32, device=device)
    sens = back_project(ones, geom)
    return torch.where(sens < EM_SMALL, torch.ones_like(sens), sens)


def graph_replay(state, stream=None):
    """One iteration of ``state`` (an object with ``iterate()``, ``x``,
    ``graph`` and ``graphs_ok``) as a CUDA graph replay, the graph captured
    on first use.  The capture runs on a side stream with
    capture_begin/capture_end: the torch.cuda.graph context manager also
    runs gc.collect() and empty_cache(), host work (and re-allocation
    afterwards) that costs far more than the capture in a busy process.  If
    capture is refused the state runs eagerly from then on."""
    if not state.graphs_ok:
        return state.iterate()
    if state.graph is None:
        cur = torch.cuda.current_stream(state.x.device)
        side = stream if stream is not None else torch.cuda.Stream(state.x.device)
        side.wait_stream(cur)
        g = torch.cuda.CUDAGraph()
        try:
            with torch.cuda.stream(side):
                g.capture_begin()
                try:
                    state.iterate()
                finally:
                    g.capture_end()
            cur.wait_stream(side)
            state.graph = g
        except Exception:  # capture refused: run eagerly from now on
            cur.wait_stream(side)
            state.graphs_ok = False
            return state.iterate()
    state.graph.replay()


class EMTVState:
    """x, y, the cached sensitivity and the projection / backprojection
    scratch of one reconstruction, all resident on the device.  ``iterate``
    enqueues one iteration on the current stream; ``graph_iterate`` replays a
    CUDA graph of it, captured on first use (eagerly from then on if capture
    is refused)."""

    def __init__(self, x, y, geom, tv_weight=TV_WEIGHT):
        self.x = x
        self.y = y
        self.geom = geom
        self.tv_weight = float(tv_weight)
        self.sens = sensitivity(geom, x.device)
        self.ws = torch.empty_like(x)
        self.ratio = torch.empty(geom.sino_shape, dtype=torch.float32, device=x.device)
        self.graph = None
        self.graphs_ok = True

    def iterate(self):
        em_ratio(self.x, self.y, self.geom, self.ratio)
        back_project(self.ratio, self.geom, out=self.ws)
        em_tv_update(self.x, self.ws, self.sens, self.tv_weight)

    def iterate_unfused(self):
        """The same iteration written as separate tensor operations (the
        projection stored, the ratio, update, norms and TV step each a pass
        over HBM): the form the fused iteration is checked against."""
        proj = forward_project(self.x, self.geom)
        ratio = self.y / torch.where(proj < EM_SMALL, torch.ones_like(proj), proj)
        back_project(ratio, self.geom, out=self.ws)
        x_em = self.x * self.ws / self.sens
        dnorm = torch.linalg.vector_norm((x_em - self.x).double()).float()
        g = tv_grad_normalised(x_em)
        self.x.copy_(torch.clamp(x_em - self.tv_weight * dnorm * g, min=0.0))

    def graph_iterate(self, stream=None):
        return graph_replay(self, stream)

    def release(self):
        self.graph = None
        for a in ("y", "sens", "ws", "ratio"):
            if hasattr(self, a):
                delattr(self, a)
