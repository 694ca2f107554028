// Internal launch interfaces between the C ABI layer and the kernels.
#pragma once

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
