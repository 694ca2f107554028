"""Several FP32 MLEM+TV reconstructions advanced together, one batched
iteration at a time (the served stream's engine; C ABI ct2_batch_*).

An iteration of the batch launches each kernel once for all jobs: a
persistent EM-ratio projector over (job, view, pixel tile) work items, the
gather backprojector's kernels over (job, item) per round of view blocks,
then each job's fused update (ct2b200.recon's iteration, same arithmetic),
so a job's iterate is the same alone and in the batch.  While the set of
jobs is unchanged the iteration is replayed from a CUDA graph; adding or
removing a job re-uploads the job descriptors and captures again.
"""
import ctypes

import torch

from . import _lib
from .autograd import _grid_args, _view_args


class EMBatch:
    """Up to ``max_jobs`` reconstructions in one batch on ``device``.  A job
    is an object with the fields of ``recon.EMTVState`` (x, y, geom, sens,
    ws, ratio, tv_weight); the batch reads and writes those tensors, which
    must stay alive while the job is in the batch."""

    def __init__(self, max_jobs, device="cuda", graphs=True):
        self.device = torch.device(device)
        self.L = _lib.lib()
        self.handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self.L.ct2_batch_create(int(max_jobs), ctypes.byref(self.handle)),
                       "ct2_batch_create")
        self.free = list(range(int(max_jobs)))
        self.jobs = {}           # slot -> job
        self.graphs = graphs
        self.graph = None
        self.committed = False
        self.replays = 0

    def __len__(self):
        return len(self.jobs)

    def full(self):
        return not self.free

    def add(self, job):
        """Adds a job (its buffers stay the caller's); returns its slot."""
        if not self.free:
            raise RuntimeError("batch is full")
        slot = self.free[0]
        g = job.geom
        with torch.cuda.device(self.device):
            rc = self.L.ct2_batch_set(self.handle, slot, job.x.data_ptr(), job.y.data_ptr(),
                                      job.sens.data_ptr(), job.ws.data_ptr(),
                                      job.ratio.data_ptr(), g.frame_vectors.data_ptr(),
                                      *_view_args(g), *_grid_args(g.grid), float(job.tv_weight))
        _lib.check(rc, "ct2_batch_set")
        self.free.pop(0)
        self.jobs[slot] = job
        self.committed = False
        self.graph = None
        return slot

    def remove(self, slot):
        """Takes a job out (synchronous: waits for its work in flight)."""
        self.graph = None
        with torch.cuda.device(self.device):
            _lib.check(self.L.ct2_batch_clear(self.handle, int(slot)), "ct2_batch_clear")
        self.jobs.pop(slot, None)
        self.free.append(slot)
        self.free.sort()
        self.committed = False

    def _commit(self):
        n = ctypes.c_int(0)
        with torch.cuda.device(self.device):
            _lib.check(self.L.ct2_batch_commit(self.handle, ctypes.byref(n)), "ct2_batch_commit")
        self.committed = True

    def _launch(self):
        st = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self.L.ct2_batch_em_iteration(self.handle, ctypes.c_void_p(st)),
                   "ct2_batch_em_iteration")

    def iterate(self):
        """One iteration of every job, enqueued on the current stream."""
        if not self.jobs:
            return
        if not self.committed:
            torch.cuda.current_stream(self.device).synchronize()
            self._commit()
        if not self.graphs:
            return self._launch()
        if self.graph is None:
            cur = torch.cuda.current_stream(self.device)
            side = torch.cuda.Stream(self.device)
            side.wait_stream(cur)
            g = torch.cuda.CUDAGraph()
            try:
                with torch.cuda.stream(side):
                    g.capture_begin()
                    try:
                        self._launch()
                    finally:
                        g.capture_end()
                cur.wait_stream(side)
                self.graph = g
            except Exception:  # capture refused: eager from now on
                cur.wait_stream(side)
                self.graphs = False
                return self._launch()
        self.graph.replay()
        self.replays += 1

    def close(self):
        self.graph = None
        if self.handle:
            with torch.cuda.device(self.device):
                self.L.ct2_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()
        self.jobs = {}

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001  (interpreter shutdown)
            pass
