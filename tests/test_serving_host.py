"""Host-side rules of the served stream, without a GPU: the seeded job mix,
a job's geometry and its validation, the HBM footprint the admission control
charges, the batch (lane) a job joins, and the latency summary."""
import math

import pytest

from ct2b200 import serving as S


def test_random_jobs_are_seeded_and_in_range():
    a = S.random_jobs(200, 4.0, seed=7)
    b = S.random_jobs(200, 4.0, seed=7)
    assert a == b
    assert S.random_jobs(200, 4.0, seed=8) != a
    arrivals = [j.arrival for j in a]
    assert all(t1 > t0 for t0, t1 in zip(arrivals, arrivals[1:]))
    # Poisson arrivals at 4/s: 200 jobs span about 50 s
    assert 35.0 < arrivals[-1] < 65.0
    assert [j.job_id for j in a] == list(range(200))
    assert len({j.seed for j in a}) == 200
    for j in a:
        assert j.kind in ("fdk", "emtv")
        assert j.n in (64, 128, 256, 384)
        assert 60 <= j.ns <= 720 and 128 <= j.nd <= 768 and 12 <= j.n_ellipsoids <= 60
        assert j.iterations == 20
    kinds = sum(j.kind == "fdk" for j in a)
    assert 70 < kinds < 130


def test_job_geometry_covers_the_volume():
    spec = S.JobSpec(job_id=0, kind="emtv", n=128, ns=90, nd=200, n_ellipsoids=12, seed=1)
    vol, scan = spec.geometry()
    assert tuple(vol.grid[6:9]) == (128, 128, 128)
    assert math.isclose(vol.grid[0], 1.0)  # 128 mm field of view
    assert (scan.ns, scan.nu, scan.nv) == (90, 200, 200)
    # magnification 2 (SID 500, SDD 1000) with a 20 % margin on each side
    assert math.isclose(scan.nu * scan.du, 2.0 * 128.0 * 1.2, rel_tol=1e-6)
    spec2 = S.JobSpec(job_id=1, kind="fdk", n=64, ns=10, nd=32, n_ellipsoids=12, seed=1,
                      voxel_mm=0.5)
    vol2, _ = spec2.geometry()
    assert math.isclose(vol2.grid[0], 0.5)


@pytest.mark.parametrize("change, words", [
    ({"kind": "art"}, "unknown kind"),
    ({"n": 0}, "sizes must be >= 1"),
    ({"ns": -3}, "sizes must be >= 1"),
    ({"nd": 0}, "sizes must be >= 1"),
    ({"voxel_mm": 0.0}, "voxel size"),
    ({"voxel_mm": float("nan")}, "voxel size"),
])
def test_job_geometry_rejects_bad_specs(change, words):
    fields = dict(job_id=3, kind="emtv", n=32, ns=12, nd=40, n_ellipsoids=12, seed=1)
    fields.update(change)
    with pytest.raises(ValueError, match=words):
        S.JobSpec(**fields).geometry()


def test_footprint_counts_buffers_and_caps_the_ray_table():
    spec = S.JobSpec(job_id=0, kind="emtv", n=64, ns=60, nd=128, n_ellipsoids=12, seed=1)
    nrays, nvox = 60 * 128 * 128, 64 ** 3
    table = nrays * 20 + 60 * (128 * 16 + 64)
    assert spec.footprint_bytes() == 4 * (3 * nrays + 6 * nvox) + table + (64 << 20)
    big = S.JobSpec(job_id=1, kind="emtv", n=64, ns=720, nd=768, n_ellipsoids=12, seed=1)
    nrays = 720 * 768 * 768
    assert big.footprint_bytes() == (4 * (3 * nrays + 6 * nvox) + S.GATHER_TABLE_BUDGET +
                                     (64 << 20))
    # larger in every size
    base = spec.footprint_bytes()
    for change in ({"n": 128}, {"ns": 61}, {"nd": 129}):
        f = dict(job_id=2, kind="emtv", n=64, ns=60, nd=128, n_ellipsoids=12, seed=1)
        f.update(change)
        assert S.JobSpec(**f).footprint_bytes() > base


def test_lane_key_groups_by_size_and_cost_octave():
    def key(n, ns, nd):
        return S._lane_key(S.JobSpec(job_id=0, kind="emtv", n=n, ns=ns, nd=nd,
                                     n_ellipsoids=12, seed=1))
    assert key(128, 100, 256) == (128, int(math.log2(100 * 256 * 256)))
    assert key(128, 100, 256) == key(128, 101, 256)      # same octave of rays
    assert key(128, 100, 256) != key(256, 100, 256)      # other volume size
    assert key(128, 200, 256)[1] == key(128, 100, 256)[1] + 1
    assert key(64, 0, 0) == (64, 0)                      # no rays: the lowest class


def test_report_summary():
    r = S.ServeReport()
    empty = r.summary()
    assert empty["jobs"] == 0 and empty["recon_per_s"] == 0.0
    assert empty["p50_s"] is None and empty["p99_s"] is None and empty["max_s"] is None
    r.latencies = {i: float(i + 1) for i in range(100)}
    r.wall = 50.0
    r.status = {i: "done" for i in range(100)}
    r.status.update({100: "rejected", 101: "failed", 102: "cancelled"})
    r.peak_footprint = 3_000_000_000
    s = r.summary()
    assert s["jobs"] == 100 and s["recon_per_s"] == 2.0
    assert s["p50_s"] == 50.5 and math.isclose(s["p99_s"], 99.01) and s["max_s"] == 100.0
    assert s["status_counts"] == {"done": 100, "rejected": 1, "failed": 1, "cancelled": 1}
    assert s["peak_footprint_gb"] == 3.0
