/*
 * ct2b200 -- C ABI of the B200-native reconstruction hot path of taroii/ct-2.
 *
 * Each entry point replaces one Fortran subroutine that the reference binds
 * through f2py (emil_code/Makefile:1-16 builds view_proj3D.so, ray_proj3D.so,
 * view_proj3D_tomo.so, totalvar.so, radon3D.so, tomo3Dfort.so).  Arguments
 * keep the Fortran subroutine's order, including its intent(out) arrays,
 * which the caller allocates here (f2py allocates them and drops them from
 * the Python signature).  Scalars are passed by value.
 *
 * Two families:
 *   ct2_<module>_<routine>(...)      host pointers; copies in, runs on the
 *                                    current CUDA device, copies out, returns
 *                                    when the result is in host memory.
 *   ct2_dev_<module>_<routine>(...)  device pointers, stream-ordered on
 *                                    `stream` (a cudaStream_t; 0 = legacy
 *                                    default stream); returns after enqueueing.
 *
 * Layout: every array is C-ordered over the logical shape the reference's
 * Python callers index, i.e. smat[nx][ny][nz] (z fastest),
 * sinomat[ns][nu][nv] (v fastest), frame_vectors[ns][18],
 * ray_vectors[nr][6].  Indicator arrays are int32 (Fortran INTEGER); a NULL
 * indicator means every ray is enabled.  intent(out) arrays are zero-filled
 * by the callee before use, as f2py does, so the routines that accumulate
 * (sinobackproject_*) return the same values the reference does.
 *
 * Return value: CT2_OK, or an error code with a message from ct2_last_error().
 */
#ifndef CT2B200_H
#define CT2B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CT2_OK 0
#define CT2_EINVAL 1   /* invalid argument (shape, size, spacing, pointer) */
#define CT2_ECUDA 2    /* CUDA runtime error */
#define CT2_ENOMEM 3   /* device allocation failed */
#define CT2_ETIMEOUT 4 /* a bounded device-side wait ran out */

/* Message of the last error on the calling thread ("" if none). */
const char *ct2_last_error(void);
/* Library version string. */
const char *ct2_version(void);
/* Number of bounded device-side waits (the TMA-staged projector's mbarrier
 * waits) that ran out on the current device since the last reset.  A wait
 * that runs out gives up, its chunk is read from global memory instead (the
 * same sum bit for bit), the CTA issues no further copy and, before it ends,
 * waits (bounded) for the copies it has in flight; the host entry points of
 * that projector (sinoproj_linear, emstep_linear) return CT2_ETIMEOUT when
 * the count advanced during the call.  Synchronous; reset != 0 clears the
 * count.  (No counterpart in the reference.) */
int ct2_wait_timeouts(int *count, int reset);
/* Number of kernels this library has launched in the process (every device,
 * every stream, graph captures included) since the last reset; reset != 0
 * returns the count and clears it.  Host-side bookkeeping only: it makes no
 * CUDA call.  (No counterpart in the reference.) */
int ct2_launch_count(unsigned long long *count, int reset);

/* ---- Several volumes through one view geometry ---------------------------
 * (No counterpart in the reference, whose modules take one volume per call.)
 * nvol volumes (nvol, nx, ny, nz), C-ordered and contiguous, and their
 * sinograms (nvol, ns, nu, nv), through the geometry of
 * ct2_dev_view_proj3D_sinoproj_linear / _sinobackproject_linear (no
 * indicator: every ray on), each kernel launched once for all volumes.  Each
 * volume's result equals its own single-volume call bit for bit.  The
 * backprojector zero-fills smat and uses the gather (groups of volumes whose
 * ray tables stay within 2 GB of stream-ordered scratch); with
 * ct2_set_backprojector(1) or a geometry outside the gather's range it runs
 * the single-volume backprojector per volume.  Stream-ordered; the job
 * descriptors are copied from host memory on the stream, so a call cannot be
 * captured in a CUDA graph.  nvol in [0, 4096]. */
int ct2_dev_view_proj3D_sinoproj_linear_many(int nvol, float *sinomat, const float *frame_vectors,
                                             int ns, int nu, int nv, float du, float dv, float u0,
                                             float v0, const float *smat, float dx, float dy,
                                             float dz, float x0, float y0, float z0, int nx,
                                             int ny, int nz, void *stream);
int ct2_dev_view_proj3D_sinobackproject_linear_many(int nvol, const float *sinomat,
                                                    const float *frame_vectors, int ns, int nu,
                                                    int nv, float du, float dv, float u0, float v0,
                                                    float *smat, float dx, float dy, float dz,
                                                    float x0, float y0, float z0, int nx, int ny,
                                                    int nz, void *stream);

/* ---- Batched MLEM+TV iteration of several reconstructions ----------------
 * (No counterpart in the reference, whose drivers reconstruct one volume at a
 * time.)  A batch holds up to max_jobs FP32 reconstructions of any sizes and
 * geometries (circular-family views, the gather backprojector's range) on
 * the current device.  ct2_batch_em_iteration then runs one iteration of
 * every job:
 *   ratio = y / (A x < 1e-5 ? 1 : A x);  ws = A^T ratio;
 *   xe = x * ws / (sens < 1e-5 ? 1 : sens);
 *   x  = max(0, xe - tv_weight * ||xe - x|| * g(xe) / ||g(xe)||)
 * (emstep_linear, view_proj3D.f:2801-2827, then the drivers' TV step with
 * the totalvar gradient g, the norms in FP64) with each kernel launched once
 * for all jobs: a persistent projector over (job, view, pixel tile) items, the
 * gather backprojector's kernels over (job, item) per round of view blocks,
 * then each job's update.  Each job's result equals its own iteration run
 * alone.  The caller owns every buffer: x (nx*ny*nz, updated in place), y and
 * ratio (ns*nu*nv; ratio is scratch), sens = A^T 1 (clamped or not), ws
 * (nx*ny*nz scratch).  Give every call of one batch the same stream (the
 * batch's stream): ct2_batch_set allocates the job's ray-table scratch (up to
 * 512 MB) and ct2_batch_clear frees it, stream-ordered after the iterations
 * already queued there; ct2_batch_commit uploads the job descriptors on that
 * stream and waits for that stream only, and must follow every set/clear
 * before the next iteration, which otherwise fails with CT2_EINVAL.
 * ct2_batch_em_iteration is stream-ordered, allocates nothing and
 * synchronises nothing (it can be captured in a CUDA graph; capture again
 * after a commit).  A handle is used by one thread at a time. */
int ct2_batch_create(int max_jobs, void **handle);
int ct2_batch_destroy(void *handle);
int ct2_batch_set(void *handle, int slot, float *x, const float *y, const float *sens, float *ws,
                  float *ratio, const float *frame_vectors, int ns, int nu, int nv, float du,
                  float dv, float u0, float v0, float dx, float dy, float dz, float x0, float y0,
                  float z0, int nx, int ny, int nz, float tv_weight, void *stream);
int ct2_batch_clear(void *handle, int slot, void *stream);
int ct2_batch_commit(void *handle, void *stream, int *njobs);
int ct2_batch_em_iteration(void *handle, void *stream);
/* Exercises the bounded device-side wait: one thread waits, at most `spins`
 * tries (1 to 2^20), on an mbarrier that nothing completes and no copy
 * targets.  Returns CT2_ETIMEOUT when the wait gives up, as it must; the
 * context stays usable.  Synchronous.  (No counterpart in the reference.) */
int ct2_wait_selftest(int spins);
/* Which matched backprojector the linear view-geometry entry points use:
 * 0 (default) the atomic-free voxel-driven gather for views whose detector v
 * axis is the volume's z axis (other views and z-driven rays still go
 * through the ray-driven scatter), 1 the ray-driven scatter with L2
 * reductions for every view.  Both are the exact transpose of the
 * projector; the gather is also bit-reproducible run to run.  Process-wide;
 * set it while no call is in flight.  (No counterpart in the reference.) */
int ct2_set_backprojector(int kind);

/* ------------------------------------------------------------------ */
/* view_proj3D (emil_code/view_proj3D.f)                               */
/* ------------------------------------------------------------------ */

/* Joseph projector, bilinear: emil_code/view_proj3D.f:703-910 */
int ct2_view_proj3D_sinoproj_linear(float *sinomat, const int32_t *indsino,
                                    const float *frame_vectors, int ns, int nu, int nv, float du,
                                    float dv, float u0, float v0, const float *smat, float dx,
                                    float dy, float dz, float x0, float y0, float z0, int nx,
                                    int ny, int nz);
int ct2_dev_view_proj3D_sinoproj_linear(float *sinomat, const int32_t *indsino,
                                        const float *frame_vectors, int ns, int nu, int nv,
                                        float du, float dv, float u0, float v0, const float *smat,
                                        float dx, float dy, float dz, float x0, float y0, float z0,
                                        int nx, int ny, int nz, void *stream);

/* Joseph projector, nearest voxel: emil_code/view_proj3D.f:915-1092 */
int ct2_view_proj3D_sinoproj_nearest(float *sinomat, const int32_t *indsino,
                                     const float *frame_vectors, int ns, int nu, int nv, float du,
                                     float dv, float u0, float v0, const float *smat, float dx,
                                     float dy, float dz, float x0, float y0, float z0, int nx,
                                     int ny, int nz);
int ct2_dev_view_proj3D_sinoproj_nearest(float *sinomat, const int32_t *indsino,
                                         const float *frame_vectors, int ns, int nu, int nv,
                                         float du, float dv, float u0, float v0, const float *smat,
                                         float dx, float dy, float dz, float x0, float y0,
                                         float z0, int nx, int ny, int nz, void *stream);
/* Voxel-driven bilinear splat through 3x4 projection matrices
 * projmats[ns][3][4] (voxel centres x10, 1-based detector cells):
 * emil_code/view_proj3D.f:607-697 */
int ct2_view_proj3D_matproj_linear(float *sinomat, const float *projmats, int ns, int nu, int nv,
                                   float du, float dv, float u0, float v0, const float *smat,
                                   float dx, float dy, float dz, float x0, float y0, float z0,
                                   int nx, int ny, int nz);
int ct2_dev_view_proj3D_matproj_linear(float *sinomat, const float *projmats, int ns, int nu,
                                       int nv, float du, float dv, float u0, float v0,
                                       const float *smat, float dx, float dy, float dz, float x0,
                                       float y0, float z0, int nx, int ny, int nz, void *stream);

/* Matched (exact-transpose) backprojector, bilinear: emil_code/view_proj3D.f:1096-1370 */
int ct2_view_proj3D_sinobackproject_linear(const float *sinomat, const int32_t *indsino,
                                           const float *frame_vectors, int ns, int nu, int nv,
                                           float du, float dv, float u0, float v0, float *smat,
                                           float dx, float dy, float dz, float x0, float y0,
                                           float z0, int nx, int ny, int nz);
int ct2_dev_view_proj3D_sinobackproject_linear(const float *sinomat, const int32_t *indsino,
                                               const float *frame_vectors, int ns, int nu, int nv,
                                               float du, float dv, float u0, float v0, float *smat,
                                               float dx, float dy, float dz, float x0, float y0,
                                               float z0, int nx, int ny, int nz, void *stream);

/* Matched backprojector, nearest voxel: emil_code/view_proj3D.f:1374-1595 */
int ct2_view_proj3D_sinobackproject_nearest(const float *sinomat, const int32_t *indsino,
                                            const float *frame_vectors, int ns, int nu, int nv,
                                            float du, float dv, float u0, float v0, float *smat,
                                            float dx, float dy, float dz, float x0, float y0,
                                            float z0, int nx, int ny, int nz);
int ct2_dev_view_proj3D_sinobackproject_nearest(const float *sinomat, const int32_t *indsino,
                                                const float *frame_vectors, int ns, int nu, int nv,
                                                float du, float dv, float u0, float v0,
                                                float *smat, float dx, float dy, float dz, float x0,
                                                float y0, float z0, int nx, int ny, int nz,
                                                void *stream);

/* One MLEM step, bilinear (smat in/out): emil_code/view_proj3D.f:2507-2831 */
int ct2_view_proj3D_emstep_linear(const float *sinomat, const int32_t *indsino,
                                  const float *frame_vectors, int ns, int nu, int nv, float du,
                                  float dv, float u0, float v0, float *smat, float dx, float dy,
                                  float dz, float x0, float y0, float z0, int nx, int ny, int nz);
int ct2_dev_view_proj3D_emstep_linear(const float *sinomat, const int32_t *indsino,
                                      const float *frame_vectors, int ns, int nu, int nv, float du,
                                      float dv, float u0, float v0, float *smat, float dx,
                                      float dy, float dz, float x0, float y0, float z0, int nx,
                                      int ny, int nz, void *stream);

/* The first half of that MLEM step on its own: ratio = y / (A smat < 1e-5 ?
 * 1 : A smat) over the rays (emil_code/view_proj3D.f:2801-2810), written by
 * the projector's epilogue.  A loop that caches A^T 1 pairs it with
 * ct2_dev_view_proj3D_sinobackproject_linear of the ratio and a voxel update
 * (for the EM+TV drivers, ct2_dev_prec_em_tv_update with CT2_F32 storage).
 * Disabled rays get ratio 0.  (No counterpart of its own in the reference.) */
int ct2_dev_view_proj3D_emratio_linear(float *ratio, const float *y, const int32_t *indsino,
                                       const float *frame_vectors, int ns, int nu, int nv,
                                       float du, float dv, float u0, float v0, const float *smat,
                                       float dx, float dy, float dz, float x0, float y0, float z0,
                                       int nx, int ny, int nz, void *stream);

/* One MLEM step, nearest voxel (smat in/out): emil_code/view_proj3D.f:2834-3075 */
int ct2_view_proj3D_emstep_nearest(const float *sinomat, const int32_t *indsino,
                                   const float *frame_vectors, int ns, int nu, int nv, float du,
                                   float dv, float u0, float v0, float *smat, float dx, float dy,
                                   float dz, float x0, float y0, float z0, int nx, int ny, int nz);
int ct2_dev_view_proj3D_emstep_nearest(const float *sinomat, const int32_t *indsino,
                                       const float *frame_vectors, int ns, int nu, int nv,
                                       float du, float dv, float u0, float v0, float *smat,
                                       float dx, float dy, float dz, float x0, float y0, float z0,
                                       int nx, int ny, int nz, void *stream);

/* ------------------------------------------------------------------ */
/* view_proj3D_tomo (emil_code/view_proj3D_tomo.f)                     */
/* ------------------------------------------------------------------ */

/* z-driven Joseph projector: emil_code/view_proj3D_tomo.f:4-148 */
int ct2_view_proj3D_tomo_sinoprojz(float *sinomat, const int32_t *indsino,
                                   const float *frame_vectors, int ns, int nu, int nv, float du,
                                   float dv, float u0, float v0, const float *smat, float dx,
                                   float dy, float dz, float x0, float y0, float z0, int nx,
                                   int ny, int nz);
int ct2_dev_view_proj3D_tomo_sinoprojz(float *sinomat, const int32_t *indsino,
                                       const float *frame_vectors, int ns, int nu, int nv,
                                       float du, float dv, float u0, float v0, const float *smat,
                                       float dx, float dy, float dz, float x0, float y0, float z0,
                                       int nx, int ny, int nz, void *stream);

/* One z-driven MLEM step (smat in/out): emil_code/view_proj3D_tomo.f:615-822 */
int ct2_view_proj3D_tomo_emstep_linearz(const float *sinomat, const int32_t *indsino,
                                        const float *frame_vectors, int ns, int nu, int nv,
                                        float du, float dv, float u0, float v0, float *smat,
                                        float dx, float dy, float dz, float x0, float y0, float z0,
                                        int nx, int ny, int nz);
int ct2_dev_view_proj3D_tomo_emstep_linearz(const float *sinomat, const int32_t *indsino,
                                            const float *frame_vectors, int ns, int nu, int nv,
                                            float du, float dv, float u0, float v0, float *smat,
                                            float dx, float dy, float dz, float x0, float y0,
                                            float z0, int nx, int ny, int nz, void *stream);

/* ------------------------------------------------------------------ */
/* ray_proj3D (emil_code/ray_proj3D.f): per-ray endpoints ray_vectors[nr][6] */
/* = (source xyz, bin xyz)                                             */
/* ------------------------------------------------------------------ */

/* emil_code/ray_proj3D.f:514-671 */
int ct2_ray_proj3D_sinoproj_linear(float *sinomat, const int32_t *indsino,
                                   const float *ray_vectors, int nr, const float *smat, float dx,
                                   float dy, float dz, float x0, float y0, float z0, int nx,
                                   int ny, int nz);
int ct2_dev_ray_proj3D_sinoproj_linear(float *sinomat, const int32_t *indsino,
                                       const float *ray_vectors, int nr, const float *smat,
                                       float dx, float dy, float dz, float x0, float y0, float z0,
                                       int nx, int ny, int nz, void *stream);

/* emil_code/ray_proj3D.f:677-804 */
int ct2_ray_proj3D_sinoproj_nearest(float *sinomat, const int32_t *indsino,
                                    const float *ray_vectors, int nr, const float *smat, float dx,
                                    float dy, float dz, float x0, float y0, float z0, int nx,
                                    int ny, int nz);
int ct2_dev_ray_proj3D_sinoproj_nearest(float *sinomat, const int32_t *indsino,
                                        const float *ray_vectors, int nr, const float *smat,
                                        float dx, float dy, float dz, float x0, float y0, float z0,
                                        int nx, int ny, int nz, void *stream);

/* emil_code/ray_proj3D.f:809-980 (bounds `lt n-1`, as the reference) */
int ct2_ray_proj3D_sinobackproject_nearest(const float *sinomat, const int32_t *indsino,
                                           const float *ray_vectors, int nr, float *smat,
                                           float dx, float dy, float dz, float x0, float y0,
                                           float z0, int nx, int ny, int nz);
int ct2_dev_ray_proj3D_sinobackproject_nearest(const float *sinomat, const int32_t *indsino,
                                               const float *ray_vectors, int nr, float *smat,
                                               float dx, float dy, float dz, float x0, float y0,
                                               float z0, int nx, int ny, int nz, void *stream);

/* emil_code/ray_proj3D.f:1454-1652 (smat in/out) */
int ct2_ray_proj3D_emstep_nearest(const float *sinomat, const int32_t *indsino,
                                  const float *ray_vectors, int nr, float *smat, float dx,
                                  float dy, float dz, float x0, float y0, float z0, int nx, int ny,
                                  int nz);
int ct2_dev_ray_proj3D_emstep_nearest(const float *sinomat, const int32_t *indsino,
                                      const float *ray_vectors, int nr, float *smat, float dx,
                                      float dy, float dz, float x0, float y0, float z0, int nx,
                                      int ny, int nz, void *stream);

/* ------------------------------------------------------------------ */
/* ART (sequential Kaczmarz; the reference's ray order is kept exactly) */
/* ------------------------------------------------------------------ */

/* emil_code/view_proj3D.f:1950-2271 (smat in/out) */
int ct2_view_proj3D_artstep_linear(float reg_fac, const float *sinomat, const int32_t *indsino,
                                   const float *frame_vectors, int ns, int nu, int nv, float du,
                                   float dv, float u0, float v0, float *smat, float dx, float dy,
                                   float dz, float x0, float y0, float z0, int nx, int ny, int nz);
int ct2_dev_view_proj3D_artstep_linear(float reg_fac, const float *sinomat,
                                       const int32_t *indsino, const float *frame_vectors, int ns,
                                       int nu, int nv, float du, float dv, float u0, float v0,
                                       float *smat, float dx, float dy, float dz, float x0,
                                       float y0, float z0, int nx, int ny, int nz, void *stream);
/* emil_code/view_proj3D.f:2275-2503 (smat in/out) */
int ct2_view_proj3D_artstep_nearest(float reg_fac, const float *sinomat, const int32_t *indsino,
                                    const float *frame_vectors, int ns, int nu, int nv, float du,
                                    float dv, float u0, float v0, float *smat, float dx, float dy,
                                    float dz, float x0, float y0, float z0, int nx, int ny,
                                    int nz);
int ct2_dev_view_proj3D_artstep_nearest(float reg_fac, const float *sinomat,
                                        const int32_t *indsino, const float *frame_vectors, int ns,
                                        int nu, int nv, float du, float dv, float u0, float v0,
                                        float *smat, float dx, float dy, float dz, float x0,
                                        float y0, float z0, int nx, int ny, int nz, void *stream);
/* emil_code/view_proj3D_tomo.f:154-347 (smat in/out) */
int ct2_view_proj3D_tomo_artstepz(float reg_fac, const float *sinomat, const int32_t *indsino,
                                  const float *frame_vectors, int ns, int nu, int nv, float du,
                                  float dv, float u0, float v0, float *smat, float dx, float dy,
                                  float dz, float x0, float y0, float z0, int nx, int ny, int nz);
int ct2_dev_view_proj3D_tomo_artstepz(float reg_fac, const float *sinomat,
                                      const int32_t *indsino, const float *frame_vectors, int ns,
                                      int nu, int nv, float du, float dv, float u0, float v0,
                                      float *smat, float dx, float dy, float dz, float x0,
                                      float y0, float z0, int nx, int ny, int nz, void *stream);
/* emil_code/view_proj3D_tomo.f:352-612 (smat and smata in/out) */
int ct2_view_proj3D_tomo_artstepz2vol(float reg_fac, const float *sinomat, const int32_t *indsino,
                                      const float *frame_vectors, int ns, int nu, int nv, float du,
                                      float dv, float u0, float v0, float *smat, float dx,
                                      float dy, float dz, float x0, float y0, float z0, int nx,
                                      int ny, int nz, float *smata, float dxa, float dya,
                                      float dza, float x0a, float y0a, float z0a, int nxa,
                                      int nya, int nza);
int ct2_dev_view_proj3D_tomo_artstepz2vol(float reg_fac, const float *sinomat,
                                          const int32_t *indsino, const float *frame_vectors,
                                          int ns, int nu, int nv, float du, float dv, float u0,
                                          float v0, float *smat, float dx, float dy, float dz,
                                          float x0, float y0, float z0, int nx, int ny, int nz,
                                          float *smata, float dxa, float dya, float dza, float x0a,
                                          float y0a, float z0a, int nxa, int nya, int nza,
                                          void *stream);
/* emil_code/ray_proj3D.f:987-1268 (smat in/out) */
int ct2_ray_proj3D_artstep_linear(float reg_fac, const float *sinomat, const int32_t *indsino,
                                  const float *ray_vectors, int nr, float *smat, float dx,
                                  float dy, float dz, float x0, float y0, float z0, int nx, int ny,
                                  int nz);
int ct2_dev_ray_proj3D_artstep_linear(float reg_fac, const float *sinomat, const int32_t *indsino,
                                      const float *ray_vectors, int nr, float *smat, float dx,
                                      float dy, float dz, float x0, float y0, float z0, int nx,
                                      int ny, int nz, void *stream);
/* emil_code/ray_proj3D.f:1272-1450 (smat in/out; bounds `lt n-1`) */
int ct2_ray_proj3D_artstep_nearest(float reg_fac, const float *sinomat, const int32_t *indsino,
                                   const float *ray_vectors, int nr, float *smat, float dx,
                                   float dy, float dz, float x0, float y0, float z0, int nx, int ny,
                                   int nz);
int ct2_dev_ray_proj3D_artstep_nearest(float reg_fac, const float *sinomat,
                                       const int32_t *indsino, const float *ray_vectors, int nr,
                                       float *smat, float dx, float dy, float dz, float x0,
                                       float y0, float z0, int nx, int ny, int nz, void *stream);

/* ------------------------------------------------------------------ */
/* Voxel-driven (unmatched) backprojection; indsino is ignored, as in   */
/* the reference                                                        */
/* ------------------------------------------------------------------ */

/* emil_code/view_proj3D.f:1769-1944 */
int ct2_view_proj3D_pd_backproj_linear(const float *sinomat, const int32_t *indsino,
                                       const float *frame_vectors, int ns, int nu, int nv, float du,
                                       float dv, float u0, float v0, float *smat, float dx,
                                       float dy, float dz, float x0, float y0, float z0, int nx,
                                       int ny, int nz);
int ct2_dev_view_proj3D_pd_backproj_linear(const float *sinomat, const int32_t *indsino,
                                           const float *frame_vectors, int ns, int nu, int nv,
                                           float du, float dv, float u0, float v0, float *smat,
                                           float dx, float dy, float dz, float x0, float y0,
                                           float z0, int nx, int ny, int nz, void *stream);
/* emil_code/view_proj3D.f:1598-1766 */
int ct2_view_proj3D_pd_backproj_nearest(const float *sinomat, const int32_t *indsino,
                                        const float *frame_vectors, int ns, int nu, int nv,
                                        float du, float dv, float u0, float v0, float *smat,
                                        float dx, float dy, float dz, float x0, float y0, float z0,
                                        int nx, int ny, int nz);
int ct2_dev_view_proj3D_pd_backproj_nearest(const float *sinomat, const int32_t *indsino,
                                            const float *frame_vectors, int ns, int nu, int nv,
                                            float du, float dv, float u0, float v0, float *smat,
                                            float dx, float dy, float dz, float x0, float y0,
                                            float z0, int nx, int ny, int nz, void *stream);

/* ------------------------------------------------------------------ */
/* Analytic ellipsoid projection and voxeliser                          */
/* ------------------------------------------------------------------ */

/* One view (indsino[nu][nv], frame_vectors[18]): emil_code/view_proj3D.f:483-603 */
int ct2_view_proj3D_ellipsoid_proj(float *sinomat, const int32_t *indsino,
                                   const float *frame_vectors, int nu, int nv, float du, float dv,
                                   float u0, float v0, float ax, float ay, float az, float x0,
                                   float y0, float z0, float alpha, float beta, float att);
int ct2_dev_view_proj3D_ellipsoid_proj(float *sinomat, const int32_t *indsino,
                                       const float *frame_vectors, int nu, int nv, float du,
                                       float dv, float u0, float v0, float ax, float ay, float az,
                                       float x0, float y0, float z0, float alpha, float beta,
                                       float att, void *stream);
/* emil_code/ray_proj3D.f:435-506 */
int ct2_ray_proj3D_ellipsoid_proj(float *sinomat, const int32_t *indsino,
                                  const float *ray_vectors, int nr, float ax, float ay, float az,
                                  float x0, float y0, float z0, float alpha, float beta, float att);
int ct2_dev_ray_proj3D_ellipsoid_proj(float *sinomat, const int32_t *indsino,
                                      const float *ray_vectors, int nr, float ax, float ay,
                                      float az, float x0, float y0, float z0, float alpha,
                                      float beta, float att, void *stream);
/* emil_code/tomo3DfortranAux.f:212-264 (smat out) */
int ct2_tomo3Dfort_ellipsoid_embed(float *smat, int nx, int ny, int nz, float dx, float dy,
                                   float dz, float x0i, float y0i, float z0i, float att,
                                   float alpha, float beta, float x0, float y0, float z0, float ax,
                                   float ay, float az);
int ct2_dev_tomo3Dfort_ellipsoid_embed(float *smat, int nx, int ny, int nz, float dx, float dy,
                                       float dz, float x0i, float y0i, float z0i, float att,
                                       float alpha, float beta, float x0, float y0, float z0,
                                       float ax, float ay, float az, void *stream);

/* ------------------------------------------------------------------ */
/* Analytic surface objects (tomo3D.py gen_object)                     */
/* ------------------------------------------------------------------ */
/* The object is the intersection of the interiors of planes (z >= 0),
 * ellipsoids, cylinders (axis z) and cones (nappe z > 0), each in its own
 * frame p -> U (p - c).  The surface table is the f2py argument list:
 * xu1..zu3 (U's rows) and x0, y0, z0 (c), nsurf entries each, surfaces
 * ordered planes, ellipsoids, cylinders, cones; nplane, nellipsoid, ncyl,
 * ncone are one more than the surfaces of each kind, and the semi-axis
 * arrays (nellipsoid, ncyl, ncone entries) carry an unused first entry.
 * EINVAL when the counts need more than nsurf surfaces.  Arithmetic is the
 * Fortran's REAL*4 expression order without FMA contraction. */
#define CT2_SHAPE_TABLE                                                                   \
    int nsurf, const float *xu1, const float *xu2, const float *xu3, const float *yu1,   \
        const float *yu2, const float *yu3, const float *zu1, const float *zu2,           \
        const float *zu3, const float *x0, const float *y0, const float *z0, int nplane, \
        int nellipsoid, const float *ax_ell, const float *ay_ell, const float *az_ell,    \
        int ncyl, const float *ax_cyl, const float *ay_cyl, int ncone,                    \
        const float *ax_cone, const float *ay_cone
/* One view: path length through the object x source-bin distance x att per
 * ray (indsino[nu][nv], frame_vectors[18]): emil_code/view_proj3D.f:11-479 */
int ct2_view_proj3D_gen_shape_proj(float *sinomat, const int32_t *indsino,
                                   const float *frame_vectors, int nu, int nv, float du, float dv,
                                   float u0, float v0, float att, CT2_SHAPE_TABLE);
int ct2_dev_view_proj3D_gen_shape_proj(float *sinomat, const int32_t *indsino,
                                       const float *frame_vectors, int nu, int nv, float du,
                                       float dv, float u0, float v0, float att, CT2_SHAPE_TABLE,
                                       void *stream);
/* Ray list (ray_vectors[nr][6]): emil_code/ray_proj3D.f:11-431 */
int ct2_ray_proj3D_gen_shape_proj(float *sinomat, const int32_t *indsino,
                                  const float *ray_vectors, int nr, float att, CT2_SHAPE_TABLE);
int ct2_dev_ray_proj3D_gen_shape_proj(float *sinomat, const int32_t *indsino,
                                      const float *ray_vectors, int nr, float att,
                                      CT2_SHAPE_TABLE, void *stream);
/* Voxeliser: att at voxel centres inside every surface, att * 0 elsewhere
 * (smat out): emil_code/tomo3DfortranAux.f:420-581 */
int ct2_tomo3Dfort_gen_obj_embed(float *smat, int nx, int ny, int nz, float dx, float dy, float dz,
                                 float x0i, float y0i, float z0i, float att, CT2_SHAPE_TABLE);
int ct2_dev_tomo3Dfort_gen_obj_embed(float *smat, int nx, int ny, int nz, float dx, float dy,
                                     float dz, float x0i, float y0i, float z0i, float att,
                                     CT2_SHAPE_TABLE, void *stream);
/* Host-only scalar helpers of tomo3Dfort (one point, host arrays; the
 * reference evaluates them per point from Python):
 * ellipse_voxval tomo3DfortranAux.f:179-208, step :270-278, framer :281-306
 * (xyz[3] out), gen_obj_voxval :311-416 (surfaces by Euler angles alpha, beta,
 * gam and centres, the same count/semi-axis conventions as above). */
int ct2_tomo3Dfort_ellipse_voxval(float *value, float x, float y, float z, float att, float alpha,
                                  float beta, float x0, float y0, float z0, float ax, float ay,
                                  float az);
int ct2_tomo3Dfort_step(float *value, float x);
int ct2_tomo3Dfort_framer(float *xyz, float x, float y, float z, float alpha, float beta,
                          float gam, float x0, float y0, float z0);
int ct2_tomo3Dfort_gen_obj_voxval(float *value, float x, float y, float z, float att, int nsurf,
                                  const float *alpha, const float *beta, const float *gam,
                                  const float *x0, const float *y0, const float *z0, int nplane,
                                  int nellipsoid, const float *ax_ell, const float *ay_ell,
                                  const float *az_ell, int ncyl, const float *ax_cyl,
                                  const float *ay_cyl, int ncone, const float *ax_cone,
                                  const float *ay_cone);

/* Each ray divided by its source-bin distance (in place): tomo3DfortranAux.f:1-68 */
int ct2_tomo3Dfort_sinoscale(float *sinomat, const float *frame_vectors, int ns, int nu, int nv,
                             float du, float dv, float u0, float v0);
int ct2_dev_tomo3Dfort_sinoscale(float *sinomat, const float *frame_vectors, int ns, int nu,
                                 int nv, float du, float dv, float u0, float v0, void *stream);
/* Window averages sinoout[nss][nus][nvs] (stride nd*, window nw*, the windows
 * inside the sinogram): tomo3DfortranAux.f:71-122 */
int ct2_tomo3Dfort_sinoave(const float *sinomat, float *sinoout, int ns, int nu, int nv, int nss,
                           int nus, int nvs, int nds, int ndu, int ndv, int nws, int nwu, int nwv);
int ct2_dev_tomo3Dfort_sinoave(const float *sinomat, float *sinoout, int ns, int nu, int nv,
                               int nss, int nus, int nvs, int nds, int ndu, int ndv, int nws,
                               int nwu, int nwv, void *stream);
/* The windows' values spread back (later windows overwrite, uncovered rays 0):
 * tomo3DfortranAux.f:125-208 */
int ct2_tomo3Dfort_sinodist(float *sinomat, const float *sinoin, int ns, int nu, int nv, int nss,
                            int nus, int nvs, int nds, int ndu, int ndv, int nws, int nwu, int nwv);
int ct2_dev_tomo3Dfort_sinodist(float *sinomat, const float *sinoin, int ns, int nu, int nv,
                                int nss, int nus, int nvs, int nds, int ndu, int ndv, int nws,
                                int nwu, int nwv, void *stream);

/* ------------------------------------------------------------------ */
/* tomoscale (emil_code/tomoscale.f)                                   */
/* ------------------------------------------------------------------ */
/* Per-slice bilinear magnification towards the source (xs, ys, zs): tomoscale.f:1-64 */
int ct2_tomoscale_tomovolmag(float *smatout, const float *smat, int nx, int ny, int nz, float x0,
                             float y0, float z0, float xlen, float ylen, float zlen, float xs,
                             float ys, float zs);
int ct2_dev_tomoscale_tomovolmag(float *smatout, const float *smat, int nx, int ny, int nz,
                                 float x0, float y0, float z0, float xlen, float ylen, float zlen,
                                 float xs, float ys, float zs, void *stream);
/* Its transpose: tomoscale.f:67-137 */
int ct2_tomoscale_tomovolmagt(float *smatout, const float *smat, int nx, int ny, int nz, float x0,
                              float y0, float z0, float xlen, float ylen, float zlen, float xs,
                              float ys, float zs);
int ct2_dev_tomoscale_tomovolmagt(float *smatout, const float *smat, int nx, int ny, int nz,
                                  float x0, float y0, float z0, float xlen, float ylen,
                                  float zlen, float xs, float ys, float zs, void *stream);

/* ------------------------------------------------------------------ */
/* totalvar (emil_code/totalvar.f)                                     */
/* ------------------------------------------------------------------ */

/* emil_code/totalvar.f:476-602: tvgmat out, *bobo out (device pointer in the
 * ct2_dev_ form) */
int ct2_totalvar_total_var_grad3d(float ambdala, float *tvgmat, const float *smat, int nx, int ny,
                                  int nz, int normalizeq, float *bobo);
int ct2_dev_totalvar_total_var_grad3d(float ambdala, float *tvgmat, const float *smat, int nx,
                                      int ny, int nz, int normalizeq, float *bobo, void *stream);
/* emil_code/totalvar.f:35-62 (a FUNCTION: the value is written to *result) */
int ct2_totalvar_total_var3d(float ambdala, const float *smat, int nx, int ny, int nz,
                             float *result);
int ct2_dev_totalvar_total_var3d(float ambdala, const float *smat, int nx, int ny, int nz,
                                 float *result, void *stream);

/* The p-variants (emil_code/totalvar.f:4-471); x**y of the Fortran is powf. */
/* Gradient magnitude image sqrt(eps + |forward differences|^2): totalvar.f:4-30 */
int ct2_totalvar_gmi(float *smatout, const float *smat, int nx, int ny, int nz);
int ct2_dev_totalvar_gmi(float *smatout, const float *smat, int nx, int ny, int nz, void *stream);
/* sum of sqrt(eps + s^2)^p: totalvar.f:65-88 */
int ct2_totalvar_calc_lp(float p, const float *smat, int nx, int ny, int nz, float *result);
int ct2_dev_totalvar_calc_lp(float p, const float *smat, int nx, int ny, int nz, float *result,
                             void *stream);
/* TpV value: totalvar.f:91-118 */
int ct2_totalvar_total_var3d_p(float p, const float *smat, int nx, int ny, int nz, float *result);
int ct2_dev_totalvar_total_var3d_p(float p, const float *smat, int nx, int ny, int nz,
                                   float *result, void *stream);
/* TpdV value (differences over the spacings): totalvar.f:121-147 */
int ct2_totalvar_total_dvar3d_p(float p, const float *smat, int nx, int ny, int nz, float dx,
                                float dy, float dz, float *result);
int ct2_dev_totalvar_total_dvar3d_p(float p, const float *smat, int nx, int ny, int nz, float dx,
                                    float dy, float dz, float *result, void *stream);
/* Lp gradient: totalvar.f:150-216 */
int ct2_totalvar_lp_grad3d(float ppp, float *tvgmat, const float *smat, int nx, int ny, int nz,
                           int normalizeq, float *bobo);
int ct2_dev_totalvar_lp_grad3d(float ppp, float *tvgmat, const float *smat, int nx, int ny, int nz,
                               int normalizeq, float *bobo, void *stream);
/* TpV gradient: totalvar.f:219-344 */
int ct2_totalvar_total_p_var_grad3d(float ppp, float *tvgmat, const float *smat, int nx, int ny,
                                    int nz, int normalizeq, float *bobo);
int ct2_dev_totalvar_total_p_var_grad3d(float ppp, float *tvgmat, const float *smat, int nx,
                                        int ny, int nz, int normalizeq, float *bobo, void *stream);
/* TpdV gradient: totalvar.f:347-471 */
int ct2_totalvar_total_p_dvar_grad3d(float ppp, float *tvgmat, const float *smat, int nx, int ny,
                                     int nz, float dx, float dy, float dz, int normalizeq,
                                     float *bobo);
int ct2_dev_totalvar_total_p_dvar_grad3d(float ppp, float *tvgmat, const float *smat, int nx,
                                         int ny, int nz, float dx, float dy, float dz,
                                         int normalizeq, float *bobo, void *stream);

/* ------------------------------------------------------------------ */
/* radon3D (emil_code/radon3D.f); indradon/radonmat[nsa][nsb][nr],      */
/* source_locations[ns][3]                                              */
/* ------------------------------------------------------------------ */

/* emil_code/radon3D.f:2-129 */
int ct2_radon3D_spherical_radon_linear(float fov, float *radonmat, const int32_t *indradon,
                                       const float *source_locations, int nsa, int nsb, int ns,
                                       int nr, float dr, float r0, const float *smat, float dx,
                                       float dy, float dz, float x0, float y0, float z0, int nx,
                                       int ny, int nz);
int ct2_dev_radon3D_spherical_radon_linear(float fov, float *radonmat, const int32_t *indradon,
                                           const float *source_locations, int nsa, int nsb, int ns,
                                           int nr, float dr, float r0, const float *smat, float dx,
                                           float dy, float dz, float x0, float y0, float z0,
                                           int nx, int ny, int nz, void *stream);
/* emil_code/radon3D.f:134-327 (smat in/out) */
int ct2_radon3D_artstep_linear(float reg_fac, float fov, const float *radonmat,
                               const int32_t *indradon, const float *source_locations, int nsa,
                               int nsb, int ns, int nr, float dr, float r0, float *smat, float dx,
                               float dy, float dz, float x0, float y0, float z0, int nx, int ny,
                               int nz);
int ct2_dev_radon3D_artstep_linear(float reg_fac, float fov, const float *radonmat,
                                   const int32_t *indradon, const float *source_locations, int nsa,
                                   int nsb, int ns, int nr, float dr, float r0, float *smat,
                                   float dx, float dy, float dz, float x0, float y0, float z0,
                                   int nx, int ny, int nz, void *stream);

/* ------------------------------------------------------------------ */
/* FDK (the reference's NumPy stages, emil_code/FDK.py)                 */
/* ------------------------------------------------------------------ */

/* out[s][u][v] = sinomat[s][u][v] * weight[u][v]: the cosine pre-weight of
 * fdk_sino_weight3D, emil_code/FDK.py:10-23 (weight table from the caller) */
int ct2_fdk_sino_weight(float *out, const float *sinomat, const float *weight, int ns, int nu,
                        int nv);
int ct2_dev_fdk_sino_weight(float *out, const float *sinomat, const float *weight, int ns, int nu,
                            int nv, void *stream);
/* Ramp filtering of fdk_sino_filter3D, emil_code/FDK.py:25-103: each line along
 * u (dim 1) or v (dim 2) convolved with the 2n-1 taps of the reference's
 * zero-padded FFT filter (lag -(n-1) first); weight[nu][nv] (or NULL) is
 * applied to the input first.  out must not alias sinomat. */
int ct2_fdk_sino_filter(float *out, const float *sinomat, const float *weight, const float *taps,
                        int ns, int nu, int nv, int dim);
int ct2_dev_fdk_sino_filter(float *out, const float *sinomat, const float *weight,
                            const float *taps, int ns, int nu, int nv, int dim, void *stream);
/* Voxel-driven FDK backprojection, emil_code/FDK.py:130-208: recon[nxy][nz],
 * vs[ns] view angles (FP64), vx/vy[nxy] and vz[nz] point coordinates */
int ct2_fdk_backproj_linear(float *recon, int ns, int nu, int nv, float du, float dv, float u0,
                            float v0, float radius, float source2detector, float uoffset,
                            float voffset, const double *vs, const float *vx, const float *vy,
                            const float *vz, int nxy, int nz, const float *sinomat);
int ct2_dev_fdk_backproj_linear(float *recon, int ns, int nu, int nv, float du, float dv,
                                float u0, float v0, float radius, float source2detector,
                                float uoffset, float voffset, const double *vs, const float *vx,
                                const float *vy, const float *vz, int nxy, int nz,
                                const float *sinomat, void *stream);

/* ------------------------------------------------------------------ */
/* Allocation-free variant                                             */
/* ------------------------------------------------------------------ */

/* No counterpart in the reference.  Same result as
 * ct2_dev_totalvar_total_var_grad3d, for callers that may not let a library
 * allocate device memory (a service that reserves its whole budget up front
 * and forbids allocation while work is in flight; a host application whose
 * own allocator owns the device memory).  Its only scratch, the per-block
 * FP64 partial sums, lives in a fixed 4096-entry (32 KiB) array in the
 * library's device memory, held by every GPU that loads the library until
 * exit; volumes that would need more than 4096 reduction blocks (more than
 * 512 SMs) are rejected with CT2_EINVAL.  The first call on each device looks
 * up that array's address, so make it before any stream capture.  All calls
 * on a device share the array: calls that overlap on the GPU (different
 * streams, not ordered) race and must not be issued. */
int ct2_dev_totalvar_total_var_grad3d_noalloc(float ambdala, float *tvgmat, const float *smat,
                                              int nx, int ny, int nz, int normalizeq, float *bobo,
                                              void *stream);

/* ------------------------------------------------------------------ */
/* Precision form (no counterpart in the reference: an addition)       */
/* ------------------------------------------------------------------ */
/*
 * The linear Joseph projector, its matched backprojector and one MLEM+TV
 * step at reduced storage precision: volumes in BF16, sinograms (data,
 * projections, EM ratios) in FP16, with every per-ray geometry quantity
 * (source, detector bin, direction, driving axis, slopes, travelled length,
 * sample model) in FP64, ray sums in FP32 with Kahan compensation and the
 * EM+TV norms in FP64.  (CT2_F16, CT2_F16) storage keeps the volume in FP16
 * (three more mantissa bits than BF16, for iterations that make many small
 * in-place updates such as ART); with (CT2_F32, CT2_F32) storage the same
 * arithmetic runs on FP32 arrays.  The algorithm is that of
 * ct2_view_proj3D_sinoproj_linear / _sinobackproject_linear /
 * _emstep_linear (z_driven = 1: view_proj3D_tomo's z-driven form); the
 * result is compared with an FP64 evaluation of it, not with the REAL*4
 * Fortran.  Device pointers only, stream-ordered.
 */
#define CT2_F32 0
#define CT2_BF16 1
#define CT2_F16 2

/* sinomat = A smat; (vol_type, sino_type) is (CT2_BF16, CT2_F16), (CT2_F16, CT2_F16)
 * or (CT2_F32, CT2_F32). */
int ct2_dev_prec_project(void *sinomat, int sino_type, const int32_t *indsino,
                         const float *frame_vectors, int ns, int nu, int nv, float du, float dv,
                         float u0, float v0, const void *smat, int vol_type, float dx, float dy,
                         float dz, float x0, float y0, float z0, int nx, int ny, int nz,
                         int z_driven, void *stream);
/* ratio = y / (A smat < 1e-5 ? 1 : A smat), the MLEM ratio of emstep_linear
 * (emil_code/view_proj3D.f:2801-2827); ratio and y have sino_type. */
int ct2_dev_prec_emratio(void *ratio, const void *y, int sino_type, const int32_t *indsino,
                         const float *frame_vectors, int ns, int nu, int nv, float du, float dv,
                         float u0, float v0, const void *smat, int vol_type, float dx, float dy,
                         float dz, float x0, float y0, float z0, int nx, int ny, int nz,
                         int z_driven, void *stream);
/* out = A^T sinomat (FP32, zero-filled first); if out_ones is not NULL it
 * receives A^T 1 over the enabled rays in the same pass. */
int ct2_dev_prec_backproject(const void *sinomat, int sino_type, const int32_t *indsino,
                             const float *frame_vectors, int ns, int nu, int nv, float du,
                             float dv, float u0, float v0, float *out, float *out_ones, float dx,
                             float dy, float dz, float x0, float y0, float z0, int nx, int ny,
                             int nz, int z_driven, void *stream);
/* After ws = A^T ratio: xe = smat * ws / (sens < em_small ? 1 : sens) (left in
 * ws), then smat = max(0, xe - tv_weight * ||xe - smat|| * g / ||g||), g the
 * TV gradient of xe (totalvar.total_var_grad3d, ambdala = 0), the norms in
 * FP64 (||g|| < 1e-5 -> 1). */
int ct2_dev_prec_em_tv_update(void *smat, int vol_type, float *ws, const float *sens, int nx,
                              int ny, int nz, float em_small, float tv_weight, void *stream);

/* One Kaczmarz (ART) sweep of view_proj3D_tomo.artstepz
 * (emil_code/view_proj3D_tomo.f:154-347) in colour order: views in order;
 * within a view the colours (cu0, cv0) in 0..cu-1 x 0..cv-1 in order, a colour
 * being the rays whose detector indices are congruent to (cu0, cv0) modulo
 * (cu, cv).  With strides from ct2_prec_art_colouring the rays of a colour
 * share no voxel, so they are updated in parallel and the sweep equals the
 * sequential Fortran sweep over the rays taken in that order.  zmajor = 1:
 * smat is stored smat[nz][ny][nx] (x fastest), which makes the z-driven
 * rays' loads coalesce; zmajor = 0: the C order smat[nx][ny][nz]. */
int ct2_dev_prec_art_sweep(float reg_fac, const void *sinomat, int sino_type,
                           const int32_t *indsino, const float *frame_vectors, int ns, int nu,
                           int nv, float du, float dv, float u0, float v0, void *smat,
                           int vol_type, float dx, float dy, float dz, float x0, float y0,
                           float z0, int nx, int ny, int nz, int cu, int cv, int zmajor,
                           void *stream);
/* The TV step after an ART sweep (prev = the volume before the sweep; ws is
 * FP32 scratch of the volume's size): smat = max(0, smat - tv_weight *
 * ||smat - prev|| * g / ||g||), g the TV gradient of smat, norms in FP64;
 * zmajor as in ct2_dev_prec_art_sweep. */
int ct2_dev_prec_art_tv_update(void *smat, int vol_type, const void *prev, float *ws, int nx,
                               int ny, int nz, float tv_weight, int zmajor, void *stream);
/* Host-only: colour strides (cu, cv) for ct2_dev_prec_art_sweep such that two
 * rays of one colour are at least 2.05 voxels apart (max norm over x, y) on
 * every slice of the z-driven geometry; frame_vectors is a HOST array. */
int ct2_prec_art_colouring(const float *frame_vectors, int ns, int nu, int nv, float du,
                           float dv, float u0, float v0, float dx, float dy, float dz, float x0,
                           float y0, float z0, int nx, int ny, int nz, int *cu, int *cv);

/* ------------------------------------------------------------------ */
/* Analytic phantom projection (an addition: the data generator)       */
/* ------------------------------------------------------------------ */
/* sinomat[ns][nu][nv] = sum over ellipsoids of att * chord length of the
 * source-bin line, in FP64 (stored FP32).  table[n_ellipsoids][16]: center(3),
 * 1/semi-axes(3), rotation R row-major (9), att; the ellipsoid is
 * {p : sum_k (((p - c) . R[:, k]) / a_k)^2 < 1}.  A superset of
 * view_proj3D.ellipsoid_proj (emil_code/view_proj3D.f:483-603), which has
 * two rotation angles; device pointers, stream-ordered. */
int ct2_dev_phantom_project(float *sinomat, const double *table, int n_ellipsoids,
                            const float *frame_vectors, int ns, int nu, int nv, float du,
                            float dv, float u0, float v0, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CT2B200_H */
