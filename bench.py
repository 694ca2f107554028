#!/usr/bin/env python
"""Benchmark of the ct-2 projector / matched-backprojector pair on one B200.

Workload (BASELINE metric "proj/backproj Gvoxel-views/s vs HBM roofline"):
the diagnostic cone-beam configuration -- 256^3 FP32 volume at 0.5 mm holding
a seeded 40-ellipsoid phantom, circular cone beam SID 500 / SDD 1000 mm, 360
views over 360 deg, 384 x 384 detector at 0.8 mm.  One step = one forward
projection (view_proj3D.sinoproj_linear) of the phantom + one matched
backprojection (view_proj3D.sinobackproject_linear) of seeded uniform data
in [0.5, 1.5) -- every ray non-zero, so the backprojector walks every ray
that crosses the volume (it skips zero data, and half the phantom's own
projection is zero; that case is reported beside the headline) -- in that
geometry; its work is 2 * 256^3 * 360 voxel-views.

value: Gvoxel-views/s with inputs resident in HBM (CUDA events on the
launching stream, L2 flushed by a 256 MiB write before every step, the flush
outside the timed interval).  e2e: the same metric through the host C ABI
(ct2_view_proj3D_sinoproj_linear + ct2_view_proj3D_sinobackproject_linear)
from pinned host buffers, every host<->device copy inside the timed region.

Served stream (the metric's second half, reported under "serving"): a seeded
Poisson stream of mixed FDK / EM+TV jobs through ct2b200.serving.serve
(HBM-budget admission, per-job streams, CUDA-graph iterations), with
reconstructions/s and p50/p99 latency, beside the same jobs run one at a time
through the drop-in API.

Multi-GPU: the path does not shard (replicas only) -- each rank runs the same
step on its own GPU, value = all ranks' voxel-views / max rank time.

--impl reference: the reference's CPU path on the host cores.  The Fortran
cannot be built in this image, so it is the C restatement of
emil_code/view_proj3D.f in the oracle, OpenMP over rays/views on every host
thread, on a bounded block of views of the same workload.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "ct-2_b200")
for _p in (PKG, ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "proj/backproj Gvoxel-views/s"
UNIT = "Gvoxel-views/s"
ART_WORKLOAD = ("config 0: 64^3 @1 mm (12 ellipsoids), 60 views, 96x96 @1.5 mm; one ART sweep in "
                "the reference's ray order (view_proj3D.artstep_linear, reg_fac 1, zero start)")
WORKLOAD = ("diagnostic cone beam: 256^3 FP32 @0.5 mm (40 seeded ellipsoids), circular SID 500 / "
            "SDD 1000 mm, 360 views / 360 deg, 384x384 detector @0.8 mm; step = sinoproj_linear "
            "of the phantom + sinobackproject_linear of dense data (every ray non-zero)")


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def _traffic_table():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return {}
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if r[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(value, ws, dev=None):
    """The largest of one scalar over all ranks (the value itself at one
    rank); every rank must call it at the same point."""
    if ws <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, ws, ms):
    """Whole-job rate in G units/s: all ranks' units over the slowest rank's
    time in milliseconds."""
    return units_per_rank * ws / (ms * 1e-3) / 1e9


def _replica_summary(summary, jobs_per_rank, ws, dev):
    """A served-stream summary over all ranks: every rank serves its own
    stream, so reconstructions/s is all ranks' jobs over the slowest wall
    time, and the latency percentiles are the worst rank's."""
    if ws <= 1:
        return summary
    out = dict(summary)
    wall = max_over_ranks(summary["wall_s"], ws, dev)
    out["wall_s"] = wall
    out["recon_per_s"] = jobs_per_rank * ws / wall
    out["p50_s"] = max_over_ranks(summary["p50_s"], ws, dev)
    out["p99_s"] = max_over_ranks(summary["p99_s"], ws, dev)
    if summary.get("max_s") is not None:
        out["max_s"] = max_over_ranks(summary["max_s"], ws, dev)
    return out


def cpu_sample_rate(vol, scan, x, target_s=12.0, nthreads=None):
    """Oracle (C restatement of the Fortran) proj + backproj on a block of
    views with every host thread; returns (Gvv/s, views used, seconds, threads)."""
    import oracle
    nthreads = nthreads or oracle.max_threads()
    vp = oracle.view_proj3D
    nvox = vol.nvox

    def run(nv_views):
        fv = scan.frame_vectors[:nv_views]
        ind = np.ones((nv_views, scan.nu, scan.nv), np.int32)
        t0 = time.perf_counter()
        p = vp.sinoproj_linear_omp(ind, fv, nv_views, scan.nu, scan.nv, scan.du, scan.dv,
                                   scan.u0, scan.v0, x, *vol.grid, nthreads)
        vp.sinobackproject_linear_omp(p, ind, fv, nv_views, scan.nu, scan.nv, scan.du, scan.dv,
                                      scan.u0, scan.v0, *vol.grid, nthreads)
        return time.perf_counter() - t0

    nvw = 1
    dt = run(nvw)
    while dt < target_s / 4 and nvw * 2 <= scan.ns:
        nvw = min(scan.ns, max(nvw * 2, int(nvw * (target_s / 2) / max(dt, 1e-3))))
        dt = run(nvw)
    return 2.0 * nvox * nvw / dt / 1e9, nvw, dt, nthreads


def cpu_art_sweep_ms():
    """The reference-order ART sweep of the ART leg in the oracle (the
    Fortran restatement) on one host core, in ms."""
    import oracle
    from ct2b200 import workloads as W
    vol0, scan0, ells0 = W.config0()
    x0 = W.voxelize(vol0, ells0)
    y0 = oracle.view_proj3D.sinoproj_linear(None, scan0.frame_vectors, *scan0.view, x0,
                                            *vol0.grid)
    start = np.zeros(vol0.shape, np.float32)
    t0 = time.perf_counter()
    oracle.view_proj3D.artstep_linear(1.0, y0, None, scan0.frame_vectors, *scan0.view, start,
                                      *vol0.grid)
    return (time.perf_counter() - t0) * 1e3


def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return
    from ct2b200 import workloads as W
    vol, scan, ells = W.config1()
    x = W.voxelize(vol, ells)
    import oracle
    nthreads = oracle.max_threads()
    # warm-up / sizing: choose a view block of ~10 s of CPU work per step
    rate, nvw, dt, nthreads = cpu_sample_rate(vol, scan, x, target_s=8.0, nthreads=nthreads)
    vp = oracle.view_proj3D
    fv = scan.frame_vectors[:nvw]
    ind = np.ones((nvw, scan.nu, scan.nv), np.int32)
    # the backprojection's input as in the GPU arm: dense data, every ray
    # non-zero (the Fortran's cost does not depend on the values)
    ydense = (np.random.default_rng(7).random((nvw, scan.nu, scan.nv)) + 0.5).astype(np.float32)

    def step():
        vp.sinoproj_linear_omp(ind, fv, nvw, scan.nu, scan.nv, scan.du, scan.dv, scan.u0,
                               scan.v0, x, *vol.grid, nthreads)
        vp.sinobackproject_linear_omp(ydense, ind, fv, nvw, scan.nu, scan.nv, scan.du, scan.dv,
                                      scan.u0, scan.v0, *vol.grid, nthreads)

    for _ in range(max(0, args.warmup - 1)):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    per_step = sum(times) / len(times)
    units = 2.0 * vol.nvox * nvw
    value = units / per_step / 1e9
    sample = ("%d of 360 views per step (proj + backproj of 256^3 over those views), "
              "%d host threads" % (nvw, nthreads))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": WORKLOAD, "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "C restatement of emil_code/view_proj3D.f (Fortran not buildable here), OpenMP",
    }
    print(json.dumps(line), flush=True)


def _event_time(fn, steps, warmup, flush=None):
    """Mean CUDA-event time (ms) of fn() on the current stream; the L2 flush
    (if given) runs before every call, outside the timed interval."""
    import torch
    for _ in range(warmup):
        fn()
    tot = 0.0
    for _ in range(steps):
        if flush is not None:
            flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        tot += e0.elapsed_time(e1)
    return tot / steps


def run_precision(args, dev, vol, scan, x, sino32, flush, proj32, ws):
    import torch
    from ct2b200 import precision as P
    from ct2b200 import tomosynthesis as T
    from ct2b200.autograd import ConeGeometry
    geom = ConeGeometry.from_scan(scan, vol, dev)
    xb = x.to(torch.bfloat16)
    s16 = torch.empty(scan.shape, dtype=torch.float16, device=dev)
    bpp = torch.empty(vol.shape, dtype=torch.float32, device=dev)
    t_p = _event_time(lambda: P.project(xb, geom, out=s16), args.steps, args.warmup, flush)
    gen = torch.Generator(device=dev)
    gen.manual_seed(8)
    y16 = (torch.rand(scan.shape, generator=gen, device=dev) + 0.5).half()  # every ray non-zero
    t_b = _event_time(lambda: P.back_project(y16, geom, out=bpp), args.steps, args.warmup, flush)
    t_p, t_b = max_over_ranks(t_p, ws, dev), max_over_ranks(t_b, ws, dev)
    proj32()
    torch.cuda.synchronize()
    err = float((s16.double() - sino32.double()).norm() / sino32.double().norm())
    units = vol.nvox * scan.ns
    alg = scan.ns * 2.0 * (vol.nvox + scan.nu * scan.nv)  # BF16 volume + FP16 detector row
    peak, kind = _peaks()
    pair = {"storage": "bf16 volume / fp16 sinogram", "proj_ms": t_p, "backproj_ms": t_b,
            "backproj_input": "seeded uniform FP16 data in [0.5, 1.5), every ray non-zero",
            "value": replica_rate(2.0 * units, ws, t_p + t_b), "unit": UNIT,
            "roofline_frac_proj": alg / (t_p * 1e-3) / 1e9 / peak,
            "roofline_frac_backproj": alg / (t_b * 1e-3) / 1e9 / peak,
            "alg_bytes_per_pass": alg, "peak_kind": kind,
            "proj_rel_l2_vs_fp32_path": err}
    del xb, s16, bpp, y16
    # tomosynthesis slab: 15 ART+TV iterations per reconstruction
    vol2, scan2 = T.slab(1)
    geom2, truth2, y2 = T.simulate(vol2, scan2, device=dev)
    col = P.art_colouring(geom2)
    its = 15
    def recon():
        job = P.ARTTV(y2, geom2, storage="bf16", colouring=col)
        for i in range(its):
            if i >= 1:
                job.graph_iterate()
            else:
                job.iterate()
        job.graph = None

    # one whole reconstruction (its graph capture included) untimed, then
    # the mean of three: in a process that has run the other legs the first
    # capture of this graph costs far more than the later ones
    t_r = max_over_ranks(_event_time(recon, 3, 1), ws, dev)
    tomo = {"workload": "tomosynthesis slab 512x384x64 (0.1/0.1/1 mm, 200 seeded ellipsoids in a "
                        "half-ellipsoid background), 25 views +-25 deg, SID 650 mm, 1024x768 @0.1 mm, "
                        "1e4-photon Poisson; 15 x (colour-ordered z-driven ART sweep + TV), "
                        "BF16 volume / FP16 sinogram; iterations 2-15 replayed as a CUDA graph; "
                        "mean of 3 reconstructions after 1 untimed",
            "colouring": list(col), "recon_ms": t_r, "ms_per_iteration": t_r / its,
            "value": replica_rate(2.0 * vol2.nvox * scan2.ns * its, ws, t_r), "unit": UNIT,
            "kernel_launches_per_iteration": scan2.ns * col[0] * col[1] + 4}
    return {"pair": pair, "tomosynthesis": tomo}


def run_workloads(dev, ws):
    """Diagnostic pipeline (FDK + 20 MLEM+TV on 256^3 x 360 views), the
    differentiable batch (50 Adam steps on 8 x 128^3 x 180 views) and one
    reference-order ART sweep of config 0, one warm run each, then one timed
    run (CUDA events)."""
    import torch
    from ct2b200 import diagnostic as D
    from ct2b200 import differentiable as Dm
    vol, scan, ells = D.geometry(1)
    geom, y = D.simulate(vol, scan, ells, device=dev)
    D.reconstruct(y, vol, scan, geom, iterations=2)  # warm-up
    t_pipe = max_over_ranks(_event_time(lambda: D.reconstruct(y, vol, scan, geom), 1, 0), ws, dev)
    vv = vol.nvox * scan.ns
    pipe = {"workload": "256^3 @0.5 mm, 40 ellipsoids, 360 views, 384x384 @0.8 mm, analytic "
                        "1e5-photon data; FDK (Hann) + 20 x (MLEM + TV 0.002)",
            "recon_ms": t_pipe,
            "value": replica_rate((1 + 2 * D.ITERATIONS) * vv, ws, t_pipe), "unit": UNIT}
    del y, geom
    vol3, scan3, geom3, y3, truth3 = Dm.problem(device=dev)
    Dm.fit(y3, geom3, steps=2)  # warm-up
    t_fit = max_over_ranks(_event_time(lambda: Dm.fit(y3, geom3), 1, 0), ws, dev)
    vv3 = vol3.nvox * scan3.ns * Dm.BATCH
    fit = {"workload": "8 x 128^3 @0.9 mm, 180 views, 192x192 @1.2 mm; 50 Adam steps on "
                       "||Ax-y||^2 + 0.01 TV(x) (projection recomputed in backward)",
           "fit_ms": t_fit, "ms_per_step": t_fit / Dm.STEPS,
           "value": replica_rate(3 * vv3 * Dm.STEPS, ws, t_fit), "unit": UNIT}
    # reference-order ART (view_proj3D.artstep_linear) on config 0: one sweep
    # on the device, data from the device projector (the host core's time for
    # the same sweep is reported under cpu_baseline)
    import view_proj3D
    from ct2b200 import workloads as W
    vol0, scan0, ells0 = W.config0()
    x0 = W.voxelize(vol0, ells0, device=dev)
    fd = torch.as_tensor(scan0.frame_vectors, device=dev)
    yd = view_proj3D.sinoproj_linear(None, fd, *scan0.view, x0, *vol0.grid)
    sd = torch.zeros(vol0.shape, dtype=torch.float32, device=dev)

    def art():
        view_proj3D.artstep_linear(1.0, yd, None, fd, *scan0.view, sd, *vol0.grid)

    art()  # warm-up
    t_art = max_over_ranks(_event_time(art, 1, 0), ws, dev)
    art_leg = {"workload": ART_WORKLOAD, "sweep_ms": t_art}
    return {"diagnostic_pipeline": pipe, "differentiable_fit": fit, "art_reference_order": art_leg}


def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    from ct2b200 import _lib, workloads as W
    L = _lib.lib()
    vol, scan, ells = W.config1()
    x = W.voxelize(vol, ells, device=dev).contiguous()
    fv = torch.as_tensor(scan.frame_vectors, device=dev).contiguous()
    sino = torch.empty(scan.shape, dtype=torch.float32, device=dev)
    bp = torch.empty(vol.shape, dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = ctypes.c_void_p(stream.cuda_stream)
    g = [float(v) for v in vol.grid[:6]] + [int(v) for v in vol.grid[6:]]
    view = [int(scan.ns), int(scan.nu), int(scan.nv), float(scan.du), float(scan.dv),
            float(scan.u0), float(scan.v0)]

    def proj():
        rc = L.ct2_dev_view_proj3D_sinoproj_linear(sino.data_ptr(), None, fv.data_ptr(), *view,
                                                   x.data_ptr(), *g, sh)
        _lib.check(rc, "sinoproj_linear")

    # The backprojector's input: seeded uniform data in [0.5, 1.5), so every
    # ray that crosses the volume carries a non-zero datum.  The kernel skips
    # rays whose datum is zero (they add nothing); the phantom's own
    # projection has about half its rays zero (they miss every ellipsoid), so
    # backprojecting it is timed separately below and not used for the
    # headline.
    gen = torch.Generator(device=dev)
    gen.manual_seed(7)
    ydense = torch.rand(scan.shape, generator=gen, device=dev) + 0.5

    def back(src=None):
        src = ydense if src is None else src
        rc = L.ct2_dev_view_proj3D_sinobackproject_linear(src.data_ptr(), None, fv.data_ptr(),
                                                          *view, bp.data_ptr(), *g, sh)
        _lib.check(rc, "sinobackproject_linear")

    for _ in range(args.warmup):
        flush.zero_()
        proj()
        back()
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    nlaunch = ctypes.c_ulonglong(0)
    _lib.check(L.ct2_launch_count(ctypes.byref(nlaunch), 1), "ct2_launch_count")
    for k in range(args.steps):
        flush.zero_()
        ev[k][0].record(stream)
        proj()
        ev[k][1].record(stream)
        back()
        ev[k][2].record(stream)
    _lib.check(L.ct2_launch_count(ctypes.byref(nlaunch), 1), "ct2_launch_count")
    gpu_launches = int(nlaunch.value)  # this library's kernels in the timed steps
    torch.cuda.synchronize()
    t_proj = sum(e[0].elapsed_time(e[1]) for e in ev) / args.steps
    t_back = sum(e[1].elapsed_time(e[2]) for e in ev) / args.steps
    t_step = max_over_ranks(t_proj + t_back, ws, dev)
    clk = clocks.stop()
    # the same backprojection of the phantom's projection (zero rays skipped)
    zero_frac = float((sino == 0).float().mean())
    t_back_phantom = max_over_ranks(_event_time(lambda: back(sino), args.steps, 1, flush), ws,
                                    dev)
    # the ray-driven scatter (L2 reductions) on the same dense data, for comparison
    _lib.check(L.ct2_set_backprojector(1), "ct2_set_backprojector")
    try:
        t_back_scatter = max_over_ranks(_event_time(back, args.steps, 1, flush), ws, dev)
    finally:
        L.ct2_set_backprojector(0)

    units_rank = 2.0 * vol.nvox * scan.ns
    value = replica_rate(units_rank, ws, t_step)

    # roofline of the dominant kernel: algorithmic bytes per pass ns*4*(N+P), each
    # view reading the volume once and writing its detector image once
    peak, peak_kind = _peaks()
    alg_bytes = scan.ns * 4.0 * (vol.nvox + scan.nu * scan.nv)
    dom_name, dom_ms = ("sinobackproject_linear", t_back) if t_back >= t_proj else \
        ("sinoproj_linear", t_proj)
    achieved = alg_bytes / (dom_ms * 1e-3) / 1e9
    traffic = _traffic_table().get(dom_name)

    # e2e: the host C ABI with pinned host buffers, copies inside the timed region
    e2e = None
    if not args.no_e2e:
        hx = torch.empty(vol.shape, dtype=torch.float32).pin_memory()
        hx.copy_(x.cpu())
        hfv = torch.as_tensor(scan.frame_vectors).pin_memory()
        hind = torch.ones(scan.shape, dtype=torch.int32).pin_memory()
        hs = torch.empty(scan.shape, dtype=torch.float32).pin_memory()
        hy = torch.empty(scan.shape, dtype=torch.float32).pin_memory()
        hy.copy_(ydense.cpu())
        hb = torch.empty(vol.shape, dtype=torch.float32).pin_memory()

        def e2e_step():
            rc = L.ct2_view_proj3D_sinoproj_linear(hs.data_ptr(), hind.data_ptr(),
                                                   hfv.data_ptr(), *view, hx.data_ptr(), *g)
            _lib.check(rc, "ct2_view_proj3D_sinoproj_linear")
            rc = L.ct2_view_proj3D_sinobackproject_linear(hy.data_ptr(), hind.data_ptr(),
                                                          hfv.data_ptr(), *view, hb.data_ptr(),
                                                          *g)
            _lib.check(rc, "ct2_view_proj3D_sinobackproject_linear")

        for _ in range(max(1, args.warmup)):
            e2e_step()
        te = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            e2e_step()
            te.append(time.perf_counter() - t0)
        t_e2e = max_over_ranks(sum(te) / len(te), ws, dev)
        nr = scan.nrays
        h2d = (vol.nvox * 4 + scan.ns * 72 + nr * 4) + (nr * 4 + nr * 4 + scan.ns * 72)
        d2h = nr * 4 + vol.nvox * 4
        e2e = {"value": replica_rate(units_rank, ws, t_e2e * 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": t_e2e * 1e3,
               "api": "ct2_view_proj3D_sinoproj_linear + ct2_view_proj3D_sinobackproject_linear "
                      "(host pointers, int32 indicator, pinned buffers)"}

    # served stream (the metric's second half): mixed jobs, Poisson arrivals.
    # The scans are simulated before any clock starts (pinned host memory);
    # a job's latency is arrival -> result on the device, its upload included.
    serving = None
    if not args.no_serving:
        from ct2b200 import serving as S
        warm = [S.JobSpec(900, "emtv", 64, 60, 128, 12, seed=1, iterations=2),
                S.JobSpec(901, "fdk", 64, 60, 128, 12, seed=2)]
        S.serve(warm, device=dev)  # warm-up
        S.serve(warm, device=dev, batched=True)
        jobs = S.random_jobs(args.serve_jobs, args.serve_rate, seed=5 + rank)
        data = S.prepare(jobs, dev)
        nj = len(jobs)
        # every leg starts from a device whose cached memory went back to the driver
        S.release_cached_memory(dev)
        served = _replica_summary(S.serve(jobs, device=dev, data=data).summary(), nj, ws, dev)
        S.release_cached_memory(dev)
        batched = _replica_summary(S.serve(jobs, device=dev, data=data, batched=True).summary(),
                                   nj, ws, dev)
        S.release_cached_memory(dev)
        single_rep = S.serve(jobs, device=dev, data=data, max_active=1, measure_footprint=True)
        single = _replica_summary(single_rep.summary(), nj, ws, dev)
        S.release_cached_memory(dev)
        served_prec = _replica_summary(S.serve(jobs, device=dev, data=data,
                                               storage="f16").summary(), nj, ws, dev)
        ratio = [single_rep.footprint_measured[j.job_id] / j.footprint_bytes() for j in jobs
                 if j.job_id in single_rep.footprint_measured]
        plain = None
        if not args.no_plain:
            sub = jobs[:args.plain_jobs]
            S.release_cached_memory(dev)
            p_sub = _replica_summary(S.run_plain(sub, device=dev, data=data).summary(), len(sub),
                                     ws, dev)
            s_sub = _replica_summary(S.serve(sub, device=dev, data=data).summary(), len(sub), ws,
                                     dev)
            plain = {"jobs": len(sub), "recon_per_s": p_sub["recon_per_s"],
                     "p50_s": p_sub["p50_s"], "p99_s": p_sub["p99_s"],
                     "served_recon_per_s_same_jobs": s_sub["recon_per_s"],
                     "speedup": s_sub["recon_per_s"] / p_sub["recon_per_s"],
                     "path": "drop-in API, NumPy in/out per call, sensitivity recomputed per "
                             "emstep_linear (the Fortran call sequence)"}
        serving = {"jobs": nj, "arrival_rate_per_s": args.serve_rate,
                   "mix": "uniform n^3 in {64,128,256,384}, views [60,720], detector [128,768]^2, "
                          "50% FDK / 50% 20x(EM+TV), seeded 12-60 ellipsoids, 150 GB budget",
                   "recon_per_s": served["recon_per_s"], "p50_s": served["p50_s"],
                   "p99_s": served["p99_s"], "max_latency_s": served["max_s"],
                   "wall_s": served["wall_s"], "graph_replayed_jobs": served["graph_jobs"],
                   "status_counts": served["status_counts"],
                   "one_at_a_time_resident": {
                       "recon_per_s": single["recon_per_s"], "p50_s": single["p50_s"],
                       "p99_s": single["p99_s"], "wall_s": single["wall_s"],
                       "path": "the same device-resident, graph-replayed jobs admitted one at "
                               "a time (max_active=1)"},
                   "speedup_vs_one_at_a_time_resident": (served["recon_per_s"] /
                                                         single["recon_per_s"]),
                   "batched": {
                       "recon_per_s": batched["recon_per_s"], "p50_s": batched["p50_s"],
                       "p99_s": batched["p99_s"], "max_latency_s": batched["max_s"],
                       "wall_s": batched["wall_s"], "status_counts": batched["status_counts"],
                       "speedup_vs_one_at_a_time_resident": (batched["recon_per_s"] /
                                                             single["recon_per_s"]),
                       "path": "EM+TV jobs advanced together, one launch per kernel for all "
                               "of them (persistent projector, batched gather rounds), graph "
                               "replay per job set; FDK jobs on their own streams"},
                   "footprint_measured_over_estimate": {
                       "max": max(ratio) if ratio else None,
                       "median": float(np.median(ratio)) if ratio else None},
                   "drop_in_one_at_a_time": plain,
                   "precision_form": {"storage": "EM+TV jobs FP16 volume / FP16 sinogram "
                                                 "(FDK jobs FP32)",
                                      "recon_per_s": served_prec["recon_per_s"],
                                      "p50_s": served_prec["p50_s"], "p99_s": served_prec["p99_s"],
                                      "speedup_vs_one_at_a_time_resident": (
                                          served_prec["recon_per_s"] / single["recon_per_s"])}}
        del data
        S.release_cached_memory(dev)

    # precision form: the same pair with a BF16 volume / FP16 sinogram, and the
    # tomosynthesis slab's 15 ART+TV iterations (BF16 volume, FP16 data)
    precision = None
    if not args.no_precision:
        precision = run_precision(args, dev, vol, scan, x, sino, flush, proj, ws)

    # the other reconstruction workloads, timed end to end on the device
    workloads = None
    if not args.no_workloads:
        workloads = run_workloads(dev, ws)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        xh = x.cpu().numpy()
        rate, nvw, dt, nth = cpu_sample_rate(vol, scan, xh, target_s=10.0)
        cpu = {"value": rate, "unit": UNIT, "cores": nth, "kind": "port",
               "sample": "%d of 360 views (proj + backproj, %.1f s), C restatement of the "
                         "Fortran, OpenMP" % (nvw, dt)}
        # the Fortran itself runs on one core: the same sample single-threaded
        rate1, nvw1, dt1, _ = cpu_sample_rate(vol, scan, xh, target_s=4.0, nthreads=1)
        cpu["single_thread"] = {"value": rate1, "unit": UNIT, "cores": 1,
                                "sample": "%d of 360 views (proj + backproj, %.1f s)" % (nvw1, dt1)}
        if workloads is not None:
            art_ms = cpu_art_sweep_ms()
            workloads["art_reference_order"]["fortran_restatement_one_core_ms"] = art_ms
            workloads["art_reference_order"]["speedup_vs_one_core"] = (
                art_ms / workloads["art_reference_order"]["sweep_ms"])

    if ws > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "l2": "flushed before every step (256 MiB write)",
                   "parallelism": "replicas" if ws > 1 else "single GPU",
                   "proj_ms": t_proj, "backproj_ms": t_back,
                   "backproj_input": "seeded uniform data in [0.5, 1.5), every ray non-zero",
                   "backproj_kind": "atomic-free voxel-driven gather (ct2_gather.cu)",
                   "backproj_scatter_ms": t_back_scatter,
                   "backproj_ms_on_phantom_projection": t_back_phantom,
                   "phantom_projection_zero_ray_fraction": zero_frac},
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "frac_of_spec_8000": achieved / 8000.0,
                     "traffic": traffic,
                     "alg_bytes_per_launch": alg_bytes},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clk,
        # per step: the projector; the backprojector's ray table, gather and
        # (empty here) scatter of the rays the gather leaves out
        "gpu_launches": gpu_launches,
        "serving": serving,
        "precision": precision,
        "workloads": workloads,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host C ABI (e2e) leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the served-stream leg")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the one-job-at-a-time baseline of the served stream")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the precision-form legs (BF16/FP16 pair, tomosynthesis ART+TV)")
    ap.add_argument("--no-workloads", action="store_true",
                    help="skip the diagnostic-pipeline and Adam-fit timings")
    ap.add_argument("--serve-jobs", type=int, default=100)
    ap.add_argument("--serve-rate", type=float, default=4.0, help="job arrivals per second")
    ap.add_argument("--plain-jobs", type=int, default=10,
                    help="jobs of the stream also run through the drop-in API one at a time")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
