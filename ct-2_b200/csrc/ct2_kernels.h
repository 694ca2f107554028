// Internal launch interfaces between the C ABI layer and the kernels.
#pragma once

#include <cuda.h>  // CUtensorMap
#include <cuda_runtime.h>

#include "ct2_common.cuh"

namespace ct2 {

// Projector launch description (view geometry or ray list).
struct ProjectArgs {
    Grid G;
    const float* vol;    // volume in the layout described by G.s
    const float* geom;   // frame_vectors (ns*18) or ray_vectors (nrays*6)
    const int* ind;      // indicator (same shape as the sinogram) or nullptr = all rays on
    int ns, nu, nv;      // view geometry
    float du, dv, u0, v0;
    long long nrays;     // ray-list geometry
    float* out;          // sinogram (or EM ratio)
    const float* y;      // EM: measured data
    float em_small;      // EM: raysum clamp
};

// Number of bounded device-side waits (TMA stage mbarriers) that ran out on
// the current device since the last reset (synchronous).
int wait_timeouts(int* count, int reset);
// Runs the bounded-wait self-test on `st` (synchronous); *timed_out = 1 when
// the wait gave up, as it must.
int wait_selftest(int spins, cudaStream_t st, int* timed_out);

// mode: MODE_LINEAR / MODE_NEAREST_LE / MODE_NEAREST_LT; list: ray-list geometry;
// force_z: z-driven only (tomosynthesis); em_ratio: write y / max(Ax, small).
int project(const ProjectArgs& a, int mode, bool list, bool force_z, bool em_ratio,
            cudaStream_t st);

// One job of a batched EM-ratio projection (linear, view geometry): its
// arguments, the index of its first work item (items of earlier jobs come
// first; a job has ns * project_batch_items(a) items) and, for the
// TMA-staged form, its volume's tensor maps (encode_volume_maps).
struct ProjectJob {
    CUtensorMap mapx, mapy;  // 64-byte aligned
    ProjectArgs a;
    long long item0;
};
int project_batch_items(const ProjectArgs& a);
// The x- and y-driven box maps of a's volume; 1 if the volume does not admit
// them (the untiled form then applies).
int encode_volume_maps(const ProjectArgs& a, CUtensorMap* mapx, CUtensorMap* mapy);
// Launches `grid` persistent CTAs over the `total` items of `njobs` jobs
// (device array, sorted by item0): the TMA-staged form (every job has its
// maps; items taken from *counter, zero before the launch) or the untiled one;
// em_ratio: each job writes y / max(Ax, small) instead of Ax.
int project_batch(const ProjectJob* jobs, int njobs, long long total, bool tma, bool em_ratio,
                  int grid, unsigned long long* counter, cudaStream_t st);

// Matched backprojector launch description.
struct BackprojectArgs {
    Grid G;
    const float* sino;   // data backprojected into out
    const int* ind;
    const float* geom;
    int ns, nu, nv;
    float du, dv, u0, v0;
    long long nrays;
    float* out;          // accumulated volume (zero-filled by the caller)
    float* out_ones;     // EM: A^T 1 accumulated alongside, or nullptr
};

int backproject(const BackprojectArgs& a, int mode, bool list, bool force_z, cudaStream_t st);

// Atomic-free voxel-driven gather (ct2_gather.cu) for linear mode, view
// geometry, added into a.out (and a.out_ones); returns 1 if it does not
// apply to these arguments.
int backproject_gather(const BackprojectArgs& a, cudaStream_t st);
// 0: gather where it applies (default), 1: always the ray-driven scatter.
int set_backprojector(int kind);

// Batched gather backprojections (several jobs per launch).  A job is views
// view0 .. view0 + nb - 1 of one backprojection of FP32 data without an
// indicator, added into a.out, with `scratch` (gather_scratch_bytes(nu, nv,
// nb) device bytes, 256-byte aligned) for its ray table.  Its descriptor is
// gather_job_bytes() bytes of host memory filled by gather_job_fill (1: the
// geometry is outside the gather's range); gather_jobs_finalize numbers the
// work items of njobs consecutive descriptors and returns the three item
// totals; gather_batch_round launches the round on a device copy of them,
// its kernels taking work items from counters[0..2] (zeroed by the round).
size_t gather_job_bytes();
// Whether a backprojection with these arguments takes the gather (the
// backprojector switch at its default, the geometry in range, no indicator).
bool gather_batch_applies(const BackprojectArgs& a);
int gather_block_views(int ns, int nu, int nv);
size_t gather_scratch_bytes(int nu, int nv, int vb);
int gather_job_fill(void* desc, const BackprojectArgs& a, int view0, int nb, void* scratch);
void gather_jobs_finalize(void* descs, int njobs, long long totals[3]);
int gather_batch_round(const void* d_descs, int njobs, const long long totals[3], int grid,
                       unsigned long long* counters, cudaStream_t st);

// x <- x * ws / max(ones, small) with the reference's clamp (ones < small -> 1).
int em_update(float* x, const float* ws, const float* ones, long long n, float small,
              cudaStream_t st);

// Ordered ART launch description.
struct ArtArgs {
    Grid G;
    float* x;            // volume updated in place
    Grid GA;             // auxiliary volume (two-volume form)
    float* xa;
    const float* geom;
    const int* ind;
    const float* y;
    int ns, nu, nv;
    float du, dv, u0, v0;
    long long nrays;
    float reg_fac;
};

int art_ordered(const ArtArgs& a, int mode, bool list, bool force_z, bool twovol, cudaStream_t st);

}  // namespace ct2
