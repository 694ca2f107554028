"""Serving loop: a stream of reconstruction jobs of mixed sizes on one GPU.

Jobs arrive over time (a seeded Poisson process).  A job is admitted when it
has arrived and its device footprint fits in the HBM budget next to the jobs
already running; its measured sinogram is then uploaded from pinned host
memory, and its volume, its cached MLEM sensitivity A^T 1 and its scratch stay
resident on the device until it finishes.  Every running job owns a CUDA
stream, so the projector, backprojector, TV and FDK kernels of different jobs
overlap on the GPU; each EM+TV iteration after the first is replayed from a
CUDA graph captured on the job's stream.  The host loop only admits, enqueues
one unit of work (an FDK reconstruction, or one EM+TV iteration) per idle job,
and retires finished jobs, so a job that arrives while others run starts as
soon as memory and a slot allow (continuous batching).

Job kinds (the mixed stream of the served configuration):
  * "fdk":  cosine weight + Hann-windowed ramp filter + FDK backprojection;
  * "emtv": 20 iterations of MLEM (x <- x * A^T(y / Ax) / A^T 1) followed by a
    TV step x <- max(0, x - 0.002 * ||dx_EM|| * g / ||g||).

The measurements are made before the stream starts (``prepare``: seeded
phantom, projection, Poisson counts, -log, kept in pinned host memory), so a
job's latency -- arrival to result on the device -- covers its upload and
its reconstruction, not the simulation of its scan.

Failures stay with their job: a job whose geometry is invalid, whose
footprint exceeds the whole budget, whose work raises, or that is cancelled
(``cancel={job_id: seconds}``; the job stops between two units of work, with
nothing of it in flight) ends with that status and a message, its memory is
released, and the rest of the stream runs on.

``serve(..., max_active=1)`` admits one job at a time: the same resident,
graph-replayed path without the overlap between jobs, the baseline that
isolates what continuous batching adds.  ``run_plain`` runs jobs one at a
time through the reference-facing drop-in API (NumPy arrays, one call per
Fortran routine, the sensitivity recomputed by every emstep_linear as the
Fortran does).

``serve(..., batched=True)`` (FP32 storage) runs the EM+TV jobs in batches
(ct2b200.batch.EMBatch), one per volume size and cost class (views x detector
pixels within a factor of 2) so that a batch's jobs cost about the same per
iteration: every job of a batch advances one iteration
per batched step, each kernel launched once for all of them -- a persistent
projector over all jobs' pixel tiles, the gather backprojector's kernels
over all jobs' items, then each job's update -- replayed from a CUDA graph
while the batch's jobs are unchanged.  A job joins its batch as soon as it
is set up and leaves when its iterations are done (or it is cancelled),
between two steps.  The batches run on their own streams and overlap with
each other and with the FDK jobs' streams.  A job its batch cannot take runs
on its own stream instead.

``serve(..., storage="f16" | "bf16")`` runs the EM+TV jobs in the precision
form (ct2b200.precision.EMTV: FP16 or BF16 volume, FP16 sinograms, FP64
per-ray setup, Kahan ray sums, FP64 norms); FDK jobs stay FP32.
"""
import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import workloads as W
from .autograd import forward_project, ConeGeometry
from .recon import EM_SMALL, TV_WEIGHT, EMTVState, graph_replay  # noqa: F401  (EM_SMALL re-exported)
PHOTONS = 1e5
MU_SCALE = 0.1  # attenuation per mm -> line integrals in cm^-1 * cm
GATHER_TABLE_BUDGET = 512 << 20  # ray-table scratch of one backprojection (ct2_gather.cu)


@dataclass
class JobSpec:
    job_id: int
    kind: str            # "fdk" or "emtv"
    n: int               # volume n^3
    ns: int              # views
    nd: int              # detector nd x nd
    n_ellipsoids: int
    seed: int
    arrival: float = 0.0  # seconds after the stream starts
    iterations: int = 20
    voxel_mm: float = None  # None: 128 mm field of view over n voxels

    def geometry(self):
        """Circular cone beam in the style of the diagnostic configuration:
        SID 500 / SDD 1000 mm, 128 mm field of view, detector covering the
        volume.  Raises ValueError for a geometry the projectors reject."""
        if self.kind not in ("fdk", "emtv"):
            raise ValueError("job %d: unknown kind %r" % (self.job_id, self.kind))
        if not (self.n >= 1 and self.ns >= 1 and self.nd >= 1):
            raise ValueError("job %d: sizes must be >= 1 (n %d, views %d, detector %d)" %
                             (self.job_id, self.n, self.ns, self.nd))
        dx = 128.0 / self.n if self.voxel_mm is None else self.voxel_mm
        if not (math.isfinite(dx) and dx > 0.0):
            raise ValueError("job %d: voxel size must be finite and > 0 (got %r)" %
                             (self.job_id, dx))
        vol = W.Volume.centered((self.n, self.n, self.n), (dx, dx, dx))
        det = 2.0 * self.n * dx * 1.2 / self.nd  # magnification 2, 20 % margin
        scan = W.circular_scan(self.ns, self.nd, self.nd, det, det, 500.0, 1000.0)
        return vol, scan

    def footprint_bytes(self):
        """Device bytes the job holds at its peak: the data, the ratio and
        the sensitivity's ones sinogram; iterate, sensitivity, backprojection
        and TV volumes; the backprojector's ray table; 64 MiB of headroom."""
        nvox = self.n ** 3
        nrays = self.ns * self.nd * self.nd
        table = min(GATHER_TABLE_BUDGET, nrays * 20 + self.ns * (self.nd * 16 + 64))
        return 4 * (3 * nrays + 6 * nvox) + table + (64 << 20)


def random_jobs(count, rate, seed=0, sizes=(64, 128, 256, 384), views=(60, 720),
                detectors=(128, 768), ellipsoids=(12, 60), iterations=20):
    """The served configuration's mixed stream: Poisson arrivals at ``rate``
    jobs/s; size, views, detector, ellipsoid count and kind drawn uniformly."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        jobs.append(JobSpec(job_id=i, kind="fdk" if rng.random() < 0.5 else "emtv",
                            n=int(rng.choice(sizes)),
                            ns=int(rng.integers(views[0], views[1] + 1)),
                            nd=int(rng.integers(detectors[0], detectors[1] + 1)),
                            n_ellipsoids=int(rng.integers(ellipsoids[0], ellipsoids[1] + 1)),
                            seed=int(seed * 1000 + i), arrival=t, iterations=iterations))
    return jobs


# ---------------------------------------------------------------------------
# measurement simulation (every path uses the same data)
# ---------------------------------------------------------------------------

def simulate_measurement(spec, device):
    """Seeded phantom, its projection, 1e5-photon Poisson counts, -log."""
    vol, scan = spec.geometry()
    ells = W.random_ellipsoids(spec.n_ellipsoids, vol.nx * vol.dx, seed=spec.seed)
    x = W.voxelize(vol, ells, device=device)
    geom = ConeGeometry.from_scan(scan, vol, device)
    p = forward_project(x, geom)
    g = torch.Generator(device=device)
    g.manual_seed(spec.seed)
    counts = torch.poisson(PHOTONS * torch.exp(-MU_SCALE * p.clamp(min=0)), generator=g)
    y = (-torch.log(counts.clamp(min=1.0) / PHOTONS) / MU_SCALE).clamp(min=0).float()
    return vol, scan, geom, x, y


def prepare(specs, device="cuda"):
    """Each job's measured sinogram, made on the device and kept in pinned
    host memory (job_id -> tensor), before any stream is timed.  A job whose
    geometry is invalid gets no data (its reconstruction fails on admission)."""
    device = torch.device(device)
    data = {}
    for spec in specs:
        try:
            vol, scan, geom, truth, y = simulate_measurement(spec, device)
        except ValueError:
            continue
        h = torch.empty(y.shape, dtype=torch.float32, pin_memory=True)
        h.copy_(y)
        data[spec.job_id] = h
        del truth, y
    torch.cuda.synchronize(device)
    return data


def release_cached_memory(device="cuda"):
    """Hands the device memory cached by torch's allocator and by the
    stream-ordered pool the library's scratch comes from back to the driver
    (each cache keeps what it freed, and one cannot use the other's), so a
    following run that allocates through either starts from a clear device."""
    import gc
    device = torch.device(device)
    gc.collect()
    torch.cuda.synchronize(device)
    torch.cuda.empty_cache()
    try:
        rt = ctypes.CDLL("libcudart.so.12")
        pool = ctypes.c_void_p()
        if rt.cudaDeviceGetDefaultMemPool(ctypes.byref(pool), device.index or 0) == 0:
            rt.cudaMemPoolTrimTo(pool, ctypes.c_size_t(0))
    except OSError:
        pass


# ---------------------------------------------------------------------------
# device memory accounting (torch's caching allocator + the stream-ordered
# pool the library's scratch comes from)
# ---------------------------------------------------------------------------

class _PoolMeter:
    RESERVED_HIGH, USED_CURRENT, USED_HIGH = 0x6, 0x7, 0x8

    def __init__(self, device):
        self.device = device
        self.ok = False
        try:
            self.rt = ctypes.CDLL("libcudart.so.12")
            self.pool = ctypes.c_void_p()
            self.ok = self.rt.cudaDeviceGetDefaultMemPool(ctypes.byref(self.pool),
                                                          device.index or 0) == 0
        except OSError:
            pass

    def _get(self, attr):
        v = ctypes.c_uint64()
        if self.rt.cudaMemPoolGetAttribute(self.pool, attr, ctypes.byref(v)) != 0:
            return 0
        return v.value

    def begin(self):
        """A mark: the bytes in use now, in each of the two allocators."""
        torch.cuda.synchronize(self.device)
        torch.cuda.reset_peak_memory_stats(self.device)
        mark = [torch.cuda.memory_allocated(self.device), 0]
        if self.ok:
            zero = ctypes.c_uint64(0)  # the pool's high-water mark resets to zero
            self.rt.cudaMemPoolSetAttribute(self.pool, self.USED_HIGH, ctypes.byref(zero))
            mark[1] = self._get(self.USED_CURRENT)
        return mark

    def peak_since(self, mark):
        """The largest number of bytes in use above the mark since it was
        taken (torch's allocator and the pool, each at its own peak)."""
        torch.cuda.synchronize(self.device)
        extra = torch.cuda.max_memory_allocated(self.device) - mark[0]
        if self.ok:
            extra += max(0, self._get(self.USED_HIGH) - mark[1])
        return extra


# ---------------------------------------------------------------------------
# served job
# ---------------------------------------------------------------------------

class Job:
    def __init__(self, spec, device, data, graphs=True, storage="f32"):
        self.spec = spec
        self.storage = storage
        self.device = device
        self.data = data
        self.graphs = graphs
        self.stream = torch.cuda.Stream(device=device)
        self.units_done = 0
        self.total_units = 1 if spec.kind == "fdk" else spec.iterations
        self.event = None
        self.graph = None
        self.t_admit = None
        self.t_done = None
        self.result = None
        self.batchable = False  # runs its iterations in the served batch
        self.slot = None        # its slot there, once it has joined

    # all work of the job is enqueued on its own stream
    def start(self):
        vol, scan = self.spec.geometry()
        if self.data is None:
            raise ValueError("job %d: no measured data" % self.spec.job_id)
        with torch.cuda.stream(self.stream):
            self.vol, self.scan = vol, scan
            self.geom = ConeGeometry.from_scan(scan, vol, self.device)
            self.y = self.data.to(self.device, non_blocking=True)
            if self.spec.kind == "emtv":
                if self.storage == "f32":
                    x = torch.full(vol.shape, 0.5, dtype=torch.float32, device=self.device)
                    self.state = EMTVState(x, self.y, self.geom)
                else:
                    self.state = _PrecisionState(self.y, self.geom, self.storage)
                self.x = self.state.x

    def _fdk(self):
        import FDK  # the drop-in module, on device tensors
        vs = np.arange(self.scan.ns) * (2 * math.pi / self.scan.ns)
        s = self.scan
        v = self.vol
        self.x = FDK.fdk_reconstruct(self.y, s.ns, s.nu, s.nv, s.du, s.dv, s.u0, s.v0, 500.0,
                                     1000.0, vs, v.nx, v.ny, v.nz, v.dx, v.dy, v.dz, v.x0, v.y0,
                                     v.z0, 'Hann', 1.0)

    def enqueue_next(self):
        with torch.cuda.stream(self.stream):
            if self.spec.kind == "fdk":
                self._fdk()
            elif self.graphs and self.units_done >= 1:
                self.state.graph_iterate(stream=self.stream)
                self.graphs = self.state.graphs_ok
                self.graph = self.state.graph
            else:
                self.state.iterate()
            self.units_done += 1
            self.event = torch.cuda.Event()
            self.event.record(self.stream)

    def idle(self):
        return self.event is None or self.event.query()

    def finished(self):
        return self.units_done >= self.total_units and self.idle()

    def release(self, keep_result=True):
        self.stream.synchronize()
        self.result = self.x if (keep_result and hasattr(self, "x")) else None
        self.graph = None
        if hasattr(self, "state"):
            self.state.release()
            del self.state
        for a in ("y", "geom"):
            if hasattr(self, a):
                delattr(self, a)
        if hasattr(self, "x"):
            del self.x


class _PrecisionState:
    """precision.EMTV behind EMTVState's interface (iterate, graph replay)."""

    def __init__(self, y, geom, storage):
        from .precision import EMTV
        self.job = EMTV(y, geom, storage=storage)
        self.x = self.job.x
        self.graph = None
        self.graphs_ok = True

    def iterate(self):
        self.job.iterate()

    def graph_iterate(self, stream=None):
        return graph_replay(self, stream)

    def release(self):
        self.graph = None
        for a in ("y", "sens", "ratio", "ws"):
            if hasattr(self.job, a):
                delattr(self.job, a)


@dataclass
class ServeReport:
    latencies: dict = field(default_factory=dict)  # job_id -> seconds (arrival -> done)
    wall: float = 0.0
    results: dict = field(default_factory=dict)
    status: dict = field(default_factory=dict)     # job_id -> done|failed|rejected|cancelled
    errors: dict = field(default_factory=dict)     # job_id -> message
    footprint_measured: dict = field(default_factory=dict)  # job_id -> bytes (max_active=1)
    peak_footprint: int = 0
    graph_jobs: int = 0

    def summary(self):
        lat = np.array(sorted(self.latencies.values()))
        counts = {}
        for s in self.status.values():
            counts[s] = counts.get(s, 0) + 1
        return {"jobs": len(lat), "wall_s": self.wall,
                "recon_per_s": len(lat) / self.wall if self.wall > 0 else 0.0,
                "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                "max_s": float(lat[-1]) if len(lat) else None,
                "peak_footprint_gb": self.peak_footprint / 1e9, "graph_jobs": self.graph_jobs,
                "status_counts": counts}


def _lane_key(spec):
    """The batch a job joins: its volume size and the octave of its views x
    detector pixels (jobs of one batch cost about the same per iteration)."""
    return (spec.n, int(math.log2(max(1, spec.ns * spec.nd * spec.nd))))


class _Lane:
    """The served batch of one volume size and cost class: its EMBatch, the
    jobs in it and the event of its last step."""

    def __init__(self, key, max_batch, device, graphs):
        from .batch import EMBatch
        self.batch = EMBatch(max_batch, device=device, graphs=graphs)
        self.members = []
        self.event = None
        self.key = key

    def idle(self):
        return self.event is None or self.event.query()

    def step(self, active, cancel, now, rep, retire, meter, marks, keep_results):
        """Between two steps: members leave, set-up jobs of this size join,
        the next step is enqueued.  Returns whether anything happened."""
        progressed = False
        B = self.batch
        for job in list(self.members):
            jid = job.spec.job_id
            if jid in cancel and cancel[jid] <= now:
                B.remove(job.slot)
                self.members.remove(job)
                retire(job, "cancelled", "cancelled after %d of %d units" %
                       (job.units_done, job.total_units))
                progressed = True
            elif job.units_done >= job.total_units:
                B.remove(job.slot)
                self.members.remove(job)
                job.t_done = now
                rep.latencies[jid] = job.t_done - job.spec.arrival
                if B.graphs:
                    rep.graph_jobs += 1
                if meter is not None:
                    rep.footprint_measured[jid] = meter.peak_since(marks.pop(jid))
                retire(job, "done", keep=True)
                if keep_results:
                    rep.results[jid] = job.result.detach().float().cpu().numpy()
                job.result = None
                progressed = True
        for job in list(active):
            if not job.batchable or job.slot is not None:
                continue
            if _lane_key(job.spec) != self.key:
                continue
            jid = job.spec.job_id
            if jid in cancel and cancel[jid] <= now:
                retire(job, "cancelled", "cancelled before its first iteration")
                progressed = True
                continue
            if B.full():
                continue
            try:
                job.slot = B.add(job.state, after=job.stream)
                self.members.append(job)
            except Exception:  # noqa: BLE001  (outside the batch's range: own stream)
                job.batchable = False
            progressed = True
        if self.members:
            try:
                self.event = B.iterate()
                for job in self.members:
                    job.units_done += 1
            except Exception as e:  # noqa: BLE001  (the step's jobs fail, the stream runs on)
                for job in list(self.members):
                    try:
                        B.remove(job.slot)
                    except Exception:  # noqa: BLE001
                        pass
                    self.members.remove(job)
                    retire(job, "failed", "batched step: %s: %s" % (type(e).__name__, e))
                self.event = None
            progressed = True
        return progressed


def serve(specs, device="cuda", hbm_budget=150e9, graphs=True, keep_results=False,
          time_zero=None, storage="f32", data=None, max_active=None, cancel=None,
          measure_footprint=False, batched=False, max_batch=32):
    """Runs the job stream with continuous batching; returns a ServeReport.

    data: job_id -> pinned host sinogram from ``prepare`` (made here, before
    the clock starts, if None).  max_active: at most this many jobs on the
    device at once (1: one at a time).  cancel: job_id -> seconds after the
    stream starts at which the job is cancelled.  measure_footprint (with
    max_active=1): the device bytes each job held at its peak.  batched (FP32
    storage): the EM+TV jobs of each volume size advance together, one
    batched iteration at a time (``EMBatch``), at most max_batch of them in a
    batch."""
    device = torch.device(device)
    if data is None:
        data = prepare(specs, device)
    cancel = dict(cancel or {})
    if measure_footprint and max_active != 1:
        raise ValueError("measure_footprint needs max_active=1 (one job on the device)")
    meter = _PoolMeter(device) if measure_footprint else None
    use_batches = batched and storage == "f32"
    lanes = {}  # _lane_key -> _Lane
    pending = sorted(specs, key=lambda s: s.arrival)
    active = []
    rep = ServeReport()
    used = 0
    marks = {}
    torch.cuda.synchronize(device)
    t0 = time.perf_counter() if time_zero is None else time_zero

    def retire(job, status, message=None, keep=False):
        nonlocal used
        try:
            job.release(keep_result=keep)
        except Exception as e:  # noqa: BLE001  (release must not stop the stream)
            message = (message + "; " if message else "") + "release: %s" % e
        rep.status[job.spec.job_id] = status
        if message:
            rep.errors[job.spec.job_id] = message
        active.remove(job)
        used -= job.spec.footprint_bytes()

    while pending or active:
        now = time.perf_counter() - t0
        # cancellations of jobs not yet admitted, and arrivals above the budget
        for spec in list(pending):
            if spec.job_id in cancel and cancel[spec.job_id] <= now:
                pending.remove(spec)
                rep.status[spec.job_id] = "cancelled"
                rep.errors[spec.job_id] = "cancelled before admission"
            elif spec.arrival <= now and spec.footprint_bytes() > hbm_budget:
                pending.remove(spec)
                rep.status[spec.job_id] = "rejected"
                rep.errors[spec.job_id] = ("needs %.1f GB, above the %.1f GB budget" %
                                           (spec.footprint_bytes() / 1e9, hbm_budget / 1e9))
        while (pending and pending[0].arrival <= now and
               used + pending[0].footprint_bytes() <= hbm_budget and
               (max_active is None or len(active) < max_active)):
            spec = pending.pop(0)
            job = Job(spec, device, data.get(spec.job_id), graphs=graphs, storage=storage)
            job.batchable = use_batches and spec.kind == "emtv"
            job.t_admit = now
            used += spec.footprint_bytes()
            rep.peak_footprint = max(rep.peak_footprint, used)
            active.append(job)
            if meter is not None:
                marks[spec.job_id] = meter.begin()
            try:
                job.start()
            except Exception as e:  # noqa: BLE001  (a job's failure is its own)
                retire(job, "failed", "%s: %s" % (type(e).__name__, e))
        progressed = False
        for job in list(active):
            jid = job.spec.job_id
            if job.batchable:
                continue  # the batch below drives it
            if jid in cancel and cancel[jid] <= time.perf_counter() - t0 and job.idle():
                retire(job, "cancelled", "cancelled after %d of %d units" %
                       (job.units_done, job.total_units))
                progressed = True
            elif job.finished():
                job.t_done = time.perf_counter() - t0
                rep.latencies[jid] = job.t_done - job.spec.arrival
                if job.graph is not None:
                    rep.graph_jobs += 1
                if meter is not None:
                    rep.footprint_measured[jid] = meter.peak_since(marks.pop(jid))
                retire(job, "done", keep=True)
                if keep_results:
                    rep.results[jid] = job.result.detach().float().cpu().numpy()
                job.result = None
                progressed = True
            elif job.idle() and job.units_done < job.total_units:
                try:
                    job.enqueue_next()
                except Exception as e:  # noqa: BLE001
                    retire(job, "failed", "%s: %s" % (type(e).__name__, e))
                progressed = True
        for job in active:
            if job.batchable and job.slot is None and _lane_key(job.spec) not in lanes:
                lanes[_lane_key(job.spec)] = _Lane(_lane_key(job.spec), max_batch, device,
                                                   graphs)
        for lane in lanes.values():
            if lane.idle():
                progressed |= lane.step(active, cancel, time.perf_counter() - t0, rep, retire,
                                        meter, marks, keep_results)
        if not progressed:
            if active:
                time.sleep(0.0002)
            elif pending:
                time.sleep(max(0.0, min(0.005, pending[0].arrival - (time.perf_counter() - t0))))
    torch.cuda.synchronize(device)
    rep.wall = time.perf_counter() - t0
    for lane in lanes.values():
        lane.batch.close()
    return rep


# ---------------------------------------------------------------------------
# the drop-in path: one job at a time through the reference-facing calls
# ---------------------------------------------------------------------------

def run_plain(specs, device="cuda", keep_results=False, data=None):
    """Each job in arrival order, alone, through the reference-facing calls
    (NumPy in, NumPy out per call, sensitivity recomputed by every
    emstep_linear as the Fortran does).  Latency = completion - arrival."""
    import FDK
    import totalvar
    import view_proj3D
    device = torch.device(device)
    if data is None:
        data = prepare(specs, device)
    rep = ServeReport()
    t0 = time.perf_counter()
    for spec in sorted(specs, key=lambda s: s.arrival):
        now = time.perf_counter() - t0
        if spec.arrival > now:
            time.sleep(spec.arrival - now)
        vol, scan = spec.geometry()
        y = data[spec.job_id].numpy()
        ind = np.ones(scan.shape, np.int32)
        if spec.kind == "fdk":
            vs = np.arange(scan.ns) * (2 * math.pi / scan.ns)
            x = FDK.fdk_reconstruct(y, scan.ns, scan.nu, scan.nv, scan.du, scan.dv, scan.u0,
                                    scan.v0, 500.0, 1000.0, vs, vol.nx, vol.ny, vol.nz, vol.dx,
                                    vol.dy, vol.dz, vol.x0, vol.y0, vol.z0, 'Hann', 1.0)
        else:
            x = np.full(vol.shape, 0.5, np.float32)
            for _ in range(spec.iterations):
                xe = view_proj3D.emstep_linear(y, ind, scan.frame_vectors, *scan.view, x,
                                               *vol.grid)
                dn = float(np.linalg.norm((xe - x).astype(np.float64)))
                g, _ = totalvar.total_var_grad3d(0.0, xe, *vol.shape, 1)
                x = np.maximum(xe - TV_WEIGHT * dn * g, 0.0).astype(np.float32)
        done = time.perf_counter() - t0
        rep.latencies[spec.job_id] = done - spec.arrival
        rep.status[spec.job_id] = "done"
        if keep_results:
            rep.results[spec.job_id] = np.asarray(x)
    rep.wall = time.perf_counter() - t0
    return rep
