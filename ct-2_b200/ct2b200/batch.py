"""Several FP32 MLEM+TV reconstructions advanced together, one batched
iteration at a time (the served stream's engine; C ABI ct2_batch_*).

An iteration of the batch launches each kernel once for all jobs: a
persistent EM-ratio projector over (job, view, pixel tile) work items, the
gather backprojector's kernels over (job, item) per round of view blocks,
then each job's fused update (ct2b200.recon's iteration, same arithmetic),
so a job's iterate is the same alone and in the batch.  While the set of
jobs is unchanged the iteration is replayed from a CUDA graph; adding or
removing a job re-uploads the job descriptors and captures again.  All of a
batch's work runs on its own stream (``EMBatch.stream``): adding, removing and
committing wait for that stream only, so other streams' work keeps running.
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
            self.stream = torch.cuda.Stream(self.device)
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

    def _st(self):
        return ctypes.c_void_p(self.stream.cuda_stream)

    def add(self, job, after=None):
        """Adds a job (its buffers stay the caller's); returns its slot.  The
        batch's later work waits for the work queued so far on ``after`` (the
        stream that set the job up; the current stream if None)."""
        if not self.free:
            raise RuntimeError("batch is full")
        slot = self.free[0]
        g = job.geom
        self.stream.wait_stream(after if after is not None
                                else torch.cuda.current_stream(self.device))
        with torch.cuda.device(self.device):
            rc = self.L.ct2_batch_set(self.handle, slot, job.x.data_ptr(), job.y.data_ptr(),
                                      job.sens.data_ptr(), job.ws.data_ptr(),
                                      job.ratio.data_ptr(), g.frame_vectors.data_ptr(),
                                      *_view_args(g), *_grid_args(g.grid), float(job.tv_weight),
                                      self._st())
        _lib.check(rc, "ct2_batch_set")
        self.free.pop(0)
        self.jobs[slot] = job
        self.committed = False
        self.graph = None
        return slot

    def remove(self, slot):
        """Takes a job out, after the batch's work queued so far."""
        self.graph = None
        with torch.cuda.device(self.device):
            _lib.check(self.L.ct2_batch_clear(self.handle, int(slot), self._st()),
                       "ct2_batch_clear")
        self.jobs.pop(slot, None)
        self.free.append(slot)
        self.free.sort()
        self.committed = False

    def _commit(self):
        n = ctypes.c_int(0)
        with torch.cuda.device(self.device):
            _lib.check(self.L.ct2_batch_commit(self.handle, self._st(), ctypes.byref(n)),
                       "ct2_batch_commit")
        self.committed = True

    def _launch(self, stream):
        _lib.check(self.L.ct2_batch_em_iteration(self.handle, ctypes.c_void_p(stream.cuda_stream)),
                   "ct2_batch_em_iteration")

    def iterate(self):
        """One iteration of every job, enqueued on the batch's stream; returns
        an event recorded after it (None for an empty batch)."""
        if not self.jobs:
            return None
        if not self.committed:
            self._commit()
        with torch.cuda.device(self.device):
            if self.graphs and self.graph is None:
                g = torch.cuda.CUDAGraph()
                side = torch.cuda.Stream(self.device)
                side.wait_stream(self.stream)
                try:
                    with torch.cuda.stream(side):
                        g.capture_begin()
                        try:
                            self._launch(side)
                        finally:
                            g.capture_end()
                    self.graph = g
                except Exception:  # capture refused: eager from now on
                    self.graphs = False
                self.stream.wait_stream(side)
            with torch.cuda.stream(self.stream):
                if self.graphs:
                    self.graph.replay()
                    self.replays += 1
                else:
                    self._launch(self.stream)
                ev = torch.cuda.Event()
                ev.record(self.stream)
        return ev

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
