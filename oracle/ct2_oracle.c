/*
 * CPU oracle for the ct-2 reconstruction hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Two instantiations of ct2_oracle_body.h: ora_f_* (REAL*4 restatement of the
 * Fortran, the parity oracle) and ora_d_* (the same algorithm in FP64, the
 * oracle the precision form and the iterated configurations report their
 * error against).  Build: gcc -O2 -ffp-contract=off (no FMA contraction, no
 * fast-math, SSE float evaluation on x86-64), see oracle/build.py.
 *
 * The *_omp entry points at the end spread the same per-ray arithmetic over
 * host threads (rays for the projector; private volumes summed at the end for
 * the backprojector): REAL*4 as the timed CPU baseline, FP64 as the checker
 * of served jobs too large for one core.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- REAL*4 instantiation ---- */
#define REAL float
#define ORA_PREFIX ora_f_
#define FLOOR floorf
#define SQRT sqrtf
#define FABS fabsf
#define COS cosf
#define SIN sinf
#define ASIN asinf
#define ACOS acosf
#define ATAN2 atan2f
#define POW powf
#include "ct2_oracle_body.h"
#undef REAL
#undef ORA_PREFIX
#undef FLOOR
#undef SQRT
#undef FABS
#undef COS
#undef SIN
#undef ASIN
#undef ACOS
#undef ATAN2
#undef POW

/* ---- FP64 instantiation ---- */
#define REAL double
#define ORA_PREFIX ora_d_
#define FLOOR floor
#define SQRT sqrt
#define FABS fabs
#define COS cos
#define SIN sin
#define ASIN asin
#define ACOS acos
#define ATAN2 atan2
#define POW pow
#include "ct2_oracle_body.h"

/* ---- timed CPU baseline: the REAL*4 restatement over host threads ---- */

int ora_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* The projector and backprojector over host threads, at either precision:
 * the same per-ray arithmetic as ora_f_ / ora_d_sinoproj_linear and
 * _sinobackproject_linear; rays split over `nthreads` (the backprojector
 * scatters into one private volume per thread and sums them at the end). */
#ifdef _OPENMP
#define ORA_THREAD_NUM(t) (t) = omp_get_thread_num()
#else
#define ORA_THREAD_NUM(t) (void)(t)
#endif

#define ORA_OMP_PAIR(PFX, REALT)                                                                   \
    void PFX##sinoproj_linear_omp(REALT *sinomat, const int *indsino, const REALT *frame_vectors,  \
                                  int ns, int nu, int nv, REALT du, REALT dv, REALT u0, REALT v0,  \
                                  const REALT *smat, REALT dx, REALT dy, REALT dz, REALT x0,       \
                                  REALT y0, REALT z0, int nx, int ny, int nz, int nthreads)        \
    {                                                                                              \
        PFX##rays_t R = {0, frame_vectors, indsino, ns, nu, nv, du, dv, u0, v0};                   \
        PFX##grid_t G = {dx, dy, dz, x0, y0, z0, nx, ny, nz};                                      \
        long n = PFX##nrays(&R);                                                                   \
        long chunk = (long)nv * 4;                                                                 \
        long nchunks = (n + chunk - 1) / chunk;                                                    \
        _Pragma("omp parallel for schedule(dynamic, 1) num_threads(nthreads)")                     \
        for (long c = 0; c < nchunks; c++) {                                                       \
            long b = c * chunk, e = b + chunk < n ? b + chunk : n;                                 \
            PFX##project_range(&R, &G, smat, ORA_LINEAR, b, e, sinomat);                           \
        }                                                                                          \
    }                                                                                              \
    void PFX##sinobackproject_linear_omp(const REALT *sinomat, const int *indsino,                 \
                                         const REALT *frame_vectors, int ns, int nu, int nv,       \
                                         REALT du, REALT dv, REALT u0, REALT v0, REALT *smat,      \
                                         REALT dx, REALT dy, REALT dz, REALT x0, REALT y0,         \
                                         REALT z0, int nx, int ny, int nz, int nthreads)           \
    {                                                                                              \
        PFX##rays_t R = {0, frame_vectors, indsino, ns, nu, nv, du, dv, u0, v0};                   \
        PFX##grid_t G = {dx, dy, dz, x0, y0, z0, nx, ny, nz};                                      \
        long nvox = (long)nx * ny * nz;                                                            \
        long n = PFX##nrays(&R);                                                                   \
        if (nthreads < 1) nthreads = 1;                                                            \
        REALT **priv = (REALT **)calloc(nthreads, sizeof(REALT *));                                \
        for (int t = 0; t < nthreads; t++) priv[t] = (REALT *)calloc(nvox, sizeof(REALT));         \
        long chunk = (long)nv * 4;                                                                 \
        long nchunks = (n + chunk - 1) / chunk;                                                    \
        _Pragma("omp parallel num_threads(nthreads)")                                              \
        {                                                                                          \
            int tid = 0;                                                                           \
            ORA_THREAD_NUM(tid);                                                                   \
            _Pragma("omp for schedule(dynamic, 1)")                                                \
            for (long c = 0; c < nchunks; c++) {                                                   \
                long b = c * chunk, e = b + chunk < n ? b + chunk : n;                             \
                PFX##backproject_range(&R, &G, sinomat, ORA_LINEAR, -1, b, e, priv[tid]);          \
            }                                                                                      \
        }                                                                                          \
        _Pragma("omp parallel for num_threads(nthreads)")                                          \
        for (long i = 0; i < nvox; i++) {                                                          \
            REALT acc = 0;                                                                         \
            for (int t = 0; t < nthreads; t++) acc += priv[t][i];                                  \
            smat[i] = acc;                                                                         \
        }                                                                                          \
        for (int t = 0; t < nthreads; t++) free(priv[t]);                                          \
        free(priv);                                                                                \
    }

ORA_OMP_PAIR(ora_f_, float)
ORA_OMP_PAIR(ora_d_, double)
