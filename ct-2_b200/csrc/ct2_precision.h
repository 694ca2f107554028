// Launch interface of the precision form (ct2_precision.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ct2_common.cuh"

namespace ct2 {

// Storage element types (the CT2_F32 / CT2_BF16 / CT2_F16 codes of ct2b200.h).
enum { ST_F32 = 0, ST_BF16 = 1, ST_F16 = 2 };

// Projector / EM-ratio launch (view geometry).  (vol, out/y) types are
// (BF16, F16), (F16, F16) or (F32, F32).
struct PrecProjectArgs {
    Grid G;
    const void* vol;
    int vol_type;
    const float* geom;   // frame_vectors (ns*18)
    const int* ind;      // indicator or nullptr = all rays on
    int ns, nu, nv;
    float du, dv, u0, v0;
    void* out;           // sinogram, or y / max(Ax, small) when y != nullptr
    int sino_type;
    const void* y;       // measured data (sinogram type), EM ratio form only
    float em_small;
    const uint32_t* pairs;  // 16-bit volumes: z-pair words (prec_make_pairs) or nullptr
};

// For a 16-bit C-ordered volume: pairs[i] = bits(v[i]) | bits(v[i+1]) << 16
// (the upper half 0 on the last z of a row), so that the two z-adjacent taps
// of a bilinear sample come in one aligned 4-byte load.
int prec_make_pairs(const void* vol, int vol_type, uint32_t* pairs, long long n, int nz,
                    cudaStream_t st);

int prec_project(const PrecProjectArgs& a, bool force_z, cudaStream_t st);

// Matched backprojector: out (+)= A^T sino, out_ones (+)= A^T 1 (FP32).
struct PrecBackprojectArgs {
    Grid G;
    const void* sino;
    int sino_type;
    const int* ind;
    const float* geom;
    int ns, nu, nv;
    float du, dv, u0, v0;
    float* out;
    float* out_ones;     // or nullptr
};

int prec_backproject(const PrecBackprojectArgs& a, bool force_z, cudaStream_t st);
// The atomic-free gather (ct2_gather.cu) over the precision form's rays,
// added into a.out (and a.out_ones); returns 1 if it does not apply.
int prec_backproject_gather(const PrecBackprojectArgs& a, cudaStream_t st);

// One EM+TV step after the EM backprojection:
//   xe = x * ws / max(sens, small)           (ws overwritten with xe, FP32)
//   x  = max(0, xe - w * ||xe - x|| * g(xe) / ||g(xe)||)   stored in vol_type
// with the norms summed in FP64 in a fixed order (partial: 2 * parts doubles,
// scale: 1 double, both device scratch).
int prec_em_tv_update(void* x, int vol_type, float* ws, const float* sens, int nx, int ny, int nz,
                      float small, float tv_weight, double* partial, double* scale,
                      cudaStream_t st);
int prec_parts(long long n);

// Kaczmarz (ART) sweep of the z-driven linear projector over all views in
// colour order: within a view, the rays whose detector indices are congruent
// to (cu0, cv0) modulo (cu, cv) form one colour; the colouring makes their
// bilinear footprints disjoint on every slice, so a colour is updated in
// parallel and the sweep equals the sequential one in the order
// view -> (cu0, cv0) -> rays.
struct PrecArtArgs {
    Grid G;
    void* x;             // volume, updated in place
    int vol_type;
    const void* y;       // measured data
    int sino_type;
    const int* ind;
    const float* geom;
    int ns, nu, nv;
    float du, dv, u0, v0;
    float reg_fac;
    int cu, cv;          // colour strides along u and v
};

int prec_art_sweep(const PrecArtArgs& a, cudaStream_t st);

// TV step after an ART sweep: x <- max(0, x - w * ||x - prev|| * g(x) / ||g(x)||),
// ws (FP32, n) is scratch; norms in FP64 as in prec_em_tv_update.
// (nx, ny, nz) are the dimensions of the C-ordered array as stored (a z-major
// volume passes (nz, ny, nx): the TV is symmetric in the axes).
int prec_art_tv_update(void* x, int vol_type, const void* prev, float* ws, int nx, int ny, int nz,
                       float tv_weight, double* partial, double* scale, cudaStream_t st);

}  // namespace ct2
