// C ABI, second part: ART, voxel-driven backprojection, analytic ellipsoid
// projection, voxeliser, total variation and the spherical Radon transform.
#include <cuda_runtime.h>

#include <cmath>

#include "ct2_capi_util.h"
#include "ct2_exact.h"
#include "ct2_kernels.h"

using namespace ct2;

#define ST(stream) ((cudaStream_t)(stream))
#define GRID_ARGS_DECL \
    float dx, float dy, float dz, float x0, float y0, float z0, int nx, int ny, int nz
#define GRID_ARGS dx, dy, dz, x0, y0, z0, nx, ny, nz

int ct2::check_vol(int nx, int ny, int nz)
{
    CT2_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, "volume dimensions must be >= 0");
    CT2_REQUIRE((long long)nx * ny * nz < (1ll << 40), "volume too large");
    return CT2_OK;
}

static int check_finite(float v, const char* what)
{
    CT2_REQUIRE(std::isfinite(v), "%s must be finite", what);
    return CT2_OK;
}

// ---------------------------------------------------------------------
// ART (ordered)
// ---------------------------------------------------------------------

static int dev_art(int mode, bool list, bool force_z, float reg_fac, const float* sinomat,
                   const int32_t* indsino, const float* geom, int ns, int nu, int nv, float du,
                   float dv, float u0, float v0, long long nr, float* smat, const Grid& G,
                   float* smata, const Grid* GA, cudaStream_t st)
{
    int rc = check_finite(reg_fac, "reg_fac");
    if (rc) return rc;
    const long long nrays = list ? nr : (long long)ns * nu * nv;
    if ((long long)G.n[0] * G.n[1] * G.n[2] == 0 || nrays == 0) return CT2_OK;
    CT2_REQUIRE(sinomat && geom && smat, "null array argument");
    ArtArgs a{};
    a.G = G;
    a.x = smat;
    if (GA) {
        a.GA = *GA;
        a.xa = smata;
    }
    a.geom = geom;
    a.ind = indsino;
    a.y = sinomat;
    a.ns = ns; a.nu = nu; a.nv = nv;
    a.du = du; a.dv = dv; a.u0 = u0; a.v0 = v0;
    a.nrays = nr;
    a.reg_fac = reg_fac;
    return art_ordered(a, mode, list, force_z, GA != nullptr, st);
}

static int host_art_view(int mode, bool force_z, float reg_fac, const float* sinomat,
                         const int32_t* indsino, const float* fv, int ns, int nu, int nv, float du,
                         float dv, float u0, float v0, float* smat, GRID_ARGS_DECL)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    if ((rc = check_grid(GRID_ARGS))) return rc;
    const size_t nrays = (size_t)ns * nu * nv, nvox = (size_t)nx * ny * nz;
    HostCall H;
    int32_t* d_ind = nullptr;
    float *d_fv = nullptr, *d_sino = nullptr, *d_x = nullptr;
    if ((rc = H.upload((void**)&d_ind, indsino, nrays * 4))) return rc;
    if ((rc = H.upload((void**)&d_fv, fv, (size_t)ns * 72))) return rc;
    if ((rc = H.upload((void**)&d_sino, sinomat, nrays * 4))) return rc;
    if ((rc = H.upload((void**)&d_x, smat, nvox * 4))) return rc;
    const Grid G = make_grid(GRID_ARGS);
    if ((rc = dev_art(mode, false, force_z, reg_fac, d_sino, d_ind, d_fv, ns, nu, nv, du, dv, u0,
                      v0, 0, d_x, G, nullptr, nullptr, H.st)))
        return rc;
    if ((rc = H.download(smat, d_x, nvox * 4))) return rc;
    return H.finish();
}

extern "C" {

int ct2_dev_view_proj3D_artstep_linear(float reg_fac, const float* sinomat, const int32_t* indsino,
                                       const float* frame_vectors, int ns, int nu, int nv,
                                       float du, float dv, float u0, float v0, float* smat,
                                       GRID_ARGS_DECL, void* stream)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc || (rc = check_grid(GRID_ARGS))) return rc;
    return dev_art(MODE_LINEAR, false, false, reg_fac, sinomat, indsino, frame_vectors, ns, nu, nv,
                   du, dv, u0, v0, 0, smat, make_grid(GRID_ARGS), nullptr, nullptr, ST(stream));
}
int ct2_view_proj3D_artstep_linear(float reg_fac, const float* sinomat, const int32_t* indsino,
                                   const float* frame_vectors, int ns, int nu, int nv, float du,
                                   float dv, float u0, float v0, float* smat, GRID_ARGS_DECL)
{
    return host_art_view(MODE_LINEAR, false, reg_fac, sinomat, indsino, frame_vectors, ns, nu, nv,
                         du, dv, u0, v0, smat, GRID_ARGS);
}
int ct2_dev_view_proj3D_artstep_nearest(float reg_fac, const float* sinomat,
                                        const int32_t* indsino, const float* frame_vectors, int ns,
                                        int nu, int nv, float du, float dv, float u0, float v0,
                                        float* smat, GRID_ARGS_DECL, void* stream)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc || (rc = check_grid(GRID_ARGS))) return rc;
    return dev_art(MODE_NEAREST_LE, false, false, reg_fac, sinomat, indsino, frame_vectors, ns, nu,
                   nv, du, dv, u0, v0, 0, smat, make_grid(GRID_ARGS), nullptr, nullptr,
                   ST(stream));
}
int ct2_view_proj3D_artstep_nearest(float reg_fac, const float* sinomat, const int32_t* indsino,
                                    const float* frame_vectors, int ns, int nu, int nv, float du,
                                    float dv, float u0, float v0, float* smat, GRID_ARGS_DECL)
{
    return host_art_view(MODE_NEAREST_LE, false, reg_fac, sinomat, indsino, frame_vectors, ns, nu,
                         nv, du, dv, u0, v0, smat, GRID_ARGS);
}
int ct2_dev_view_proj3D_tomo_artstepz(float reg_fac, const float* sinomat, const int32_t* indsino,
                                      const float* frame_vectors, int ns, int nu, int nv, float du,
                                      float dv, float u0, float v0, float* smat, GRID_ARGS_DECL,
                                      void* stream)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc || (rc = check_grid(GRID_ARGS))) return rc;
    return dev_art(MODE_LINEAR, false, true, reg_fac, sinomat, indsino, frame_vectors, ns, nu, nv,
                   du, dv, u0, v0, 0, smat, make_grid(GRID_ARGS), nullptr, nullptr, ST(stream));
}
int ct2_view_proj3D_tomo_artstepz(float reg_fac, const float* sinomat, const int32_t* indsino,
                                  const float* frame_vectors, int ns, int nu, int nv, float du,
                                  float dv, float u0, float v0, float* smat, GRID_ARGS_DECL)
{
    return host_art_view(MODE_LINEAR, true, reg_fac, sinomat, indsino, frame_vectors, ns, nu, nv,
                         du, dv, u0, v0, smat, GRID_ARGS);
}

int ct2_dev_view_proj3D_tomo_artstepz2vol(float reg_fac, const float* sinomat,
                                          const int32_t* indsino, const float* frame_vectors,
                                          int ns, int nu, int nv, float du, float dv, float u0,
                                          float v0, float* smat, GRID_ARGS_DECL, float* smata,
                                          float dxa, float dya, float dza, float x0a, float y0a,
                                          float z0a, int nxa, int nya, int nza, void* stream)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc || (rc = check_grid(GRID_ARGS))) return rc;
    if ((rc = check_grid(dxa, dya, dza, x0a, y0a, z0a, nxa, nya, nza))) return rc;
    const Grid GA = make_grid(dxa, dya, dza, x0a, y0a, z0a, nxa, nya, nza);
    if ((long long)nxa * nya * nza == 0) {
        // an empty auxiliary volume contributes nothing: the single-volume step
        return dev_art(MODE_LINEAR, false, true, reg_fac, sinomat, indsino, frame_vectors, ns, nu,
                       nv, du, dv, u0, v0, 0, smat, make_grid(GRID_ARGS), nullptr, nullptr,
                       ST(stream));
    }
    CT2_REQUIRE(smata != nullptr, "null smata");
    return dev_art(MODE_LINEAR, false, true, reg_fac, sinomat, indsino, frame_vectors, ns, nu, nv,
                   du, dv, u0, v0, 0, smat, make_grid(GRID_ARGS), smata, &GA, ST(stream));
}
int ct2_view_proj3D_tomo_artstepz2vol(float reg_fac, const float* sinomat, const int32_t* indsino,
                                      const float* frame_vectors, int ns, int nu, int nv, float du,
                                      float dv, float u0, float v0, float* smat, GRID_ARGS_DECL,
                                      float* smata, float dxa, float dya, float dza, float x0a,
                                      float y0a, float z0a, int nxa, int nya, int nza)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc || (rc = check_grid(GRID_ARGS))) return rc;
    if ((rc = check_grid(dxa, dya, dza, x0a, y0a, z0a, nxa, nya, nza))) return rc;
    const size_t nrays = (size_t)ns * nu * nv, nvox = (size_t)nx * ny * nz,
                 nvoxa = (size_t)nxa * nya * nza;
    HostCall H;
    int32_t* d_ind = nullptr;
    float *d_fv = nullptr, *d_sino = nullptr, *d_x = nullptr, *d_xa = nullptr;
    if ((rc = H.upload((void**)&d_ind, indsino, nrays * 4))) return rc;
    if ((rc = H.upload((void**)&d_fv, frame_vectors, (size_t)ns * 72))) return rc;
    if ((rc = H.upload((void**)&d_sino, sinomat, nrays * 4))) return rc;
    if ((rc = H.upload((void**)&d_x, smat, nvox * 4))) return rc;
    if ((rc = H.upload((void**)&d_xa, smata, nvoxa * 4))) return rc;
    if ((rc = ct2_dev_view_proj3D_tomo_artstepz2vol(reg_fac, d_sino, d_ind, d_fv, ns, nu, nv, du,
                                                    dv, u0, v0, d_x, GRID_ARGS, d_xa, dxa, dya, dza,
                                                    x0a, y0a, z0a, nxa, nya, nza, H.st)))
        return rc;
    if ((rc = H.download(smat, d_x, nvox * 4))) return rc;
    if ((rc = H.download(smata, d_xa, nvoxa * 4))) return rc;
    return H.finish();
}

// --- ray_proj3D ART ---

int ct2_dev_ray_proj3D_artstep_linear(float reg_fac, const float* sinomat, const int32_t* indsino,
                                      const float* ray_vectors, int nr, float* smat,
                                      GRID_ARGS_DECL, void* stream)
{
    clear_error();
    CT2_REQUIRE(nr >= 0, "nr must be >= 0");
    int rc = check_grid(GRID_ARGS);
    if (rc) return rc;
    return dev_art(MODE_LINEAR, true, false, reg_fac, sinomat, indsino, ray_vectors, 0, 0, 0, 0,
                   0, 0, 0, nr, smat, make_grid(GRID_ARGS), nullptr, nullptr, ST(stream));
}
int ct2_dev_ray_proj3D_artstep_nearest(float reg_fac, const float* sinomat,
                                       const int32_t* indsino, const float* ray_vectors, int nr,
                                       float* smat, GRID_ARGS_DECL, void* stream)
{
    clear_error();
    CT2_REQUIRE(nr >= 0, "nr must be >= 0");
    int rc = check_grid(GRID_ARGS);
    if (rc) return rc;
    return dev_art(MODE_NEAREST_LT, true, false, reg_fac, sinomat, indsino, ray_vectors, 0, 0, 0,
                   0, 0, 0, 0, nr, smat, make_grid(GRID_ARGS), nullptr, nullptr, ST(stream));
}

static int host_art_list(bool linear, float reg_fac, const float* sinomat, const int32_t* indsino,
                         const float* rv, int nr, float* smat, GRID_ARGS_DECL)
{
    clear_error();
    CT2_REQUIRE(nr >= 0, "nr must be >= 0");
    int rc = check_grid(GRID_ARGS);
    if (rc) return rc;
    const size_t nvox = (size_t)nx * ny * nz;
    HostCall H;
    int32_t* d_ind = nullptr;
    float *d_rv = nullptr, *d_sino = nullptr, *d_x = nullptr;
    if ((rc = H.upload((void**)&d_ind, indsino, (size_t)nr * 4))) return rc;
    if ((rc = H.upload((void**)&d_rv, rv, (size_t)nr * 24))) return rc;
    if ((rc = H.upload((void**)&d_sino, sinomat, (size_t)nr * 4))) return rc;
    if ((rc = H.upload((void**)&d_x, smat, nvox * 4))) return rc;
    rc = linear ? ct2_dev_ray_proj3D_artstep_linear(reg_fac, d_sino, d_ind, d_rv, nr, d_x,
                                                    GRID_ARGS, H.st)
                : ct2_dev_ray_proj3D_artstep_nearest(reg_fac, d_sino, d_ind, d_rv, nr, d_x,
                                                     GRID_ARGS, H.st);
    if (rc) return rc;
    if ((rc = H.download(smat, d_x, nvox * 4))) return rc;
    return H.finish();
}

int ct2_ray_proj3D_artstep_linear(float reg_fac, const float* sinomat, const int32_t* indsino,
                                  const float* ray_vectors, int nr, float* smat, GRID_ARGS_DECL)
{
    return host_art_list(true, reg_fac, sinomat, indsino, ray_vectors, nr, smat, GRID_ARGS);
}
int ct2_ray_proj3D_artstep_nearest(float reg_fac, const float* sinomat, const int32_t* indsino,
                                   const float* ray_vectors, int nr, float* smat, GRID_ARGS_DECL)
{
    return host_art_list(false, reg_fac, sinomat, indsino, ray_vectors, nr, smat, GRID_ARGS);
}

// ---------------------------------------------------------------------
// Voxel-driven backprojection
// ---------------------------------------------------------------------

static int dev_pd(bool linear, const float* sinomat, const float* fv, int ns, int nu, int nv,
                  float du, float dv, float u0, float v0, float* smat, GRID_ARGS_DECL,
                  cudaStream_t st)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc || (rc = check_grid(GRID_ARGS))) return rc;
    CT2_REQUIRE(du != 0.f && dv != 0.f, "du, dv must be non-zero");
    const long long nvox = (long long)nx * ny * nz;
    if (nvox == 0) return CT2_OK;
    CT2_REQUIRE(smat != nullptr, "null smat");
    if ((long long)ns * nu * nv == 0) {
        CT2_CUDA(cudaMemsetAsync(smat, 0, nvox * 4, st));
        return CT2_OK;
    }
    CT2_REQUIRE(sinomat && fv, "null sinomat/frame_vectors");
    Scratch S(st);
    float* pv = nullptr;
    if ((rc = S.get((void**)&pv, (size_t)ns * 16 * 4, false))) return rc;
    return pd_backproject(sinomat, fv, ns, nu, nv, du, dv, u0, v0, smat, make_grid(GRID_ARGS),
                          linear, pv, st);
}

static int host_pd(bool linear, const float* sinomat, const float* fv, int ns, int nu, int nv,
                   float du, float dv, float u0, float v0, float* smat, GRID_ARGS_DECL)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc || (rc = check_grid(GRID_ARGS))) return rc;
    const size_t nrays = (size_t)ns * nu * nv, nvox = (size_t)nx * ny * nz;
    HostCall H;
    float *d_fv = nullptr, *d_sino = nullptr, *d_x = nullptr;
    if ((rc = H.upload((void**)&d_fv, fv, (size_t)ns * 72))) return rc;
    if ((rc = H.upload((void**)&d_sino, sinomat, nrays * 4))) return rc;
    if ((rc = H.alloc((void**)&d_x, nvox * 4, false))) return rc;
    if ((rc = dev_pd(linear, d_sino, d_fv, ns, nu, nv, du, dv, u0, v0, d_x, GRID_ARGS, H.st)))
        return rc;
    if ((rc = H.download(smat, d_x, nvox * 4))) return rc;
    return H.finish();
}

int ct2_dev_view_proj3D_pd_backproj_linear(const float* sinomat, const int32_t* indsino,
                                           const float* frame_vectors, int ns, int nu, int nv,
                                           float du, float dv, float u0, float v0, float* smat,
                                           GRID_ARGS_DECL, void* stream)
{
    (void)indsino;  // ignored by the reference (view_proj3D.f:1918-1920 commented out)
    return dev_pd(true, sinomat, frame_vectors, ns, nu, nv, du, dv, u0, v0, smat, GRID_ARGS,
                  ST(stream));
}
int ct2_view_proj3D_pd_backproj_linear(const float* sinomat, const int32_t* indsino,
                                       const float* frame_vectors, int ns, int nu, int nv, float du,
                                       float dv, float u0, float v0, float* smat, GRID_ARGS_DECL)
{
    (void)indsino;
    return host_pd(true, sinomat, frame_vectors, ns, nu, nv, du, dv, u0, v0, smat, GRID_ARGS);
}
int ct2_dev_view_proj3D_pd_backproj_nearest(const float* sinomat, const int32_t* indsino,
                                            const float* frame_vectors, int ns, int nu, int nv,
                                            float du, float dv, float u0, float v0, float* smat,
                                            GRID_ARGS_DECL, void* stream)
{
    (void)indsino;  // ignored by the reference (view_proj3D.f:1748-1750 commented out)
    return dev_pd(false, sinomat, frame_vectors, ns, nu, nv, du, dv, u0, v0, smat, GRID_ARGS,
                  ST(stream));
}
int ct2_view_proj3D_pd_backproj_nearest(const float* sinomat, const int32_t* indsino,
                                        const float* frame_vectors, int ns, int nu, int nv,
                                        float du, float dv, float u0, float v0, float* smat,
                                        GRID_ARGS_DECL)
{
    (void)indsino;
    return host_pd(false, sinomat, frame_vectors, ns, nu, nv, du, dv, u0, v0, smat, GRID_ARGS);
}

// ---------------------------------------------------------------------
// Analytic ellipsoid projection
// ---------------------------------------------------------------------

int ct2_dev_view_proj3D_ellipsoid_proj(float* sinomat, const int32_t* indsino,
                                       const float* frame_vectors, int nu, int nv, float du,
                                       float dv, float u0, float v0, float ax, float ay, float az,
                                       float x0, float y0, float z0, float alpha, float beta,
                                       float att, void* stream)
{
    clear_error();
    int rc = check_view(1, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    if ((long long)nu * nv == 0) return CT2_OK;
    CT2_REQUIRE(sinomat && frame_vectors, "null sinomat/frame_vectors");
    EllipsoidAB e{ax, ay, az, x0, y0, z0, alpha, beta, att};
    return ellipsoid_proj_view(sinomat, indsino, frame_vectors, nu, nv, du, dv, u0, v0, e,
                               ST(stream));
}
int ct2_view_proj3D_ellipsoid_proj(float* sinomat, const int32_t* indsino,
                                   const float* frame_vectors, int nu, int nv, float du, float dv,
                                   float u0, float v0, float ax, float ay, float az, float x0,
                                   float y0, float z0, float alpha, float beta, float att)
{
    clear_error();
    int rc = check_view(1, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    const size_t n = (size_t)nu * nv;
    HostCall H;
    int32_t* d_ind = nullptr;
    float *d_fv = nullptr, *d_out = nullptr;
    if ((rc = H.upload((void**)&d_ind, indsino, n * 4))) return rc;
    if ((rc = H.upload((void**)&d_fv, frame_vectors, 72))) return rc;
    if ((rc = H.alloc((void**)&d_out, n * 4, false))) return rc;
    if ((rc = ct2_dev_view_proj3D_ellipsoid_proj(d_out, d_ind, d_fv, nu, nv, du, dv, u0, v0, ax,
                                                 ay, az, x0, y0, z0, alpha, beta, att, H.st)))
        return rc;
    if ((rc = H.download(sinomat, d_out, n * 4))) return rc;
    return H.finish();
}

int ct2_dev_ray_proj3D_ellipsoid_proj(float* sinomat, const int32_t* indsino,
                                      const float* ray_vectors, int nr, float ax, float ay,
                                      float az, float x0, float y0, float z0, float alpha,
                                      float beta, float att, void* stream)
{
    clear_error();
    CT2_REQUIRE(nr >= 0, "nr must be >= 0");
    if (nr == 0) return CT2_OK;
    CT2_REQUIRE(sinomat && ray_vectors, "null sinomat/ray_vectors");
    EllipsoidAB e{ax, ay, az, x0, y0, z0, alpha, beta, att};
    return ellipsoid_proj_list(sinomat, indsino, ray_vectors, nr, e, ST(stream));
}
int ct2_ray_proj3D_ellipsoid_proj(float* sinomat, const int32_t* indsino, const float* ray_vectors,
                                  int nr, float ax, float ay, float az, float x0, float y0,
                                  float z0, float alpha, float beta, float att)
{
    clear_error();
    CT2_REQUIRE(nr >= 0, "nr must be >= 0");
    int rc;
    HostCall H;
    int32_t* d_ind = nullptr;
    float *d_rv = nullptr, *d_out = nullptr;
    if ((rc = H.upload((void**)&d_ind, indsino, (size_t)nr * 4))) return rc;
    if ((rc = H.upload((void**)&d_rv, ray_vectors, (size_t)nr * 24))) return rc;
    if ((rc = H.alloc((void**)&d_out, (size_t)nr * 4, false))) return rc;
    if ((rc = ct2_dev_ray_proj3D_ellipsoid_proj(d_out, d_ind, d_rv, nr, ax, ay, az, x0, y0, z0,
                                                alpha, beta, att, H.st)))
        return rc;
    if ((rc = H.download(sinomat, d_out, (size_t)nr * 4))) return rc;
    return H.finish();
}

// ---------------------------------------------------------------------
// tomo3Dfort.ellipsoid_embed
// ---------------------------------------------------------------------

int ct2_dev_tomo3Dfort_ellipsoid_embed(float* smat, int nx, int ny, int nz, float dx, float dy,
                                       float dz, float x0i, float y0i, float z0i, float att,
                                       float alpha, float beta, float x0, float y0, float z0,
                                       float ax, float ay, float az, void* stream)
{
    clear_error();
    int rc = check_grid(dx, dy, dz, x0i, y0i, z0i, nx, ny, nz);
    if (rc) return rc;
    if ((long long)nx * ny * nz == 0) return CT2_OK;
    CT2_REQUIRE(smat != nullptr, "null smat");
    return ellipsoid_embed(smat, make_grid(dx, dy, dz, x0i, y0i, z0i, nx, ny, nz), att, alpha,
                           beta, x0, y0, z0, ax, ay, az, ST(stream));
}
int ct2_tomo3Dfort_ellipsoid_embed(float* smat, int nx, int ny, int nz, float dx, float dy,
                                   float dz, float x0i, float y0i, float z0i, float att,
                                   float alpha, float beta, float x0, float y0, float z0, float ax,
                                   float ay, float az)
{
    clear_error();
    int rc = check_grid(dx, dy, dz, x0i, y0i, z0i, nx, ny, nz);
    if (rc) return rc;
    const size_t nvox = (size_t)nx * ny * nz;
    HostCall H;
    float* d_x = nullptr;
    if ((rc = H.alloc((void**)&d_x, nvox * 4, false))) return rc;
    if ((rc = ct2_dev_tomo3Dfort_ellipsoid_embed(d_x, nx, ny, nz, dx, dy, dz, x0i, y0i, z0i, att,
                                                 alpha, beta, x0, y0, z0, ax, ay, az, H.st)))
        return rc;
    if ((rc = H.download(smat, d_x, nvox * 4))) return rc;
    return H.finish();
}

// ---------------------------------------------------------------------
// totalvar
// ---------------------------------------------------------------------


int ct2_dev_totalvar_total_var_grad3d(float ambdala, float* tvgmat, const float* smat, int nx,
                                      int ny, int nz, int normalizeq, float* bobo, void* stream)
{
    clear_error();
    int rc = check_vol(nx, ny, nz);
    if (rc) return rc;
    CT2_REQUIRE(bobo != nullptr, "null bobo");
    const long long n = (long long)nx * ny * nz;
    if (n > 0) CT2_REQUIRE(tvgmat && smat, "null tvgmat/smat");
    cudaStream_t st = ST(stream);
    Scratch S(st);
    double* partial = nullptr;
    if ((rc = S.get((void**)&partial, sizeof(double) * tv_parts(n), false))) return rc;
    return tv_grad(smat, tvgmat, nx, ny, nz, ambdala, normalizeq, bobo, partial, st);
}
int ct2_totalvar_total_var_grad3d(float ambdala, float* tvgmat, const float* smat, int nx, int ny,
                                  int nz, int normalizeq, float* bobo)
{
    clear_error();
    int rc = check_vol(nx, ny, nz);
    if (rc) return rc;
    const size_t n = (size_t)nx * ny * nz;
    HostCall H;
    float *d_s = nullptr, *d_t = nullptr, *d_b = nullptr;
    if ((rc = H.upload((void**)&d_s, smat, n * 4))) return rc;
    if ((rc = H.alloc((void**)&d_t, n * 4, false))) return rc;
    if ((rc = H.alloc((void**)&d_b, 4, false))) return rc;
    if ((rc = ct2_dev_totalvar_total_var_grad3d(ambdala, d_t, d_s, nx, ny, nz, normalizeq, d_b,
                                                H.st)))
        return rc;
    if ((rc = H.download(tvgmat, d_t, n * 4))) return rc;
    if ((rc = H.download(bobo, d_b, 4))) return rc;
    return H.finish();
}

int ct2_dev_totalvar_total_var3d(float ambdala, const float* smat, int nx, int ny, int nz,
                                 float* result, void* stream)
{
    clear_error();
    int rc = check_vol(nx, ny, nz);
    if (rc) return rc;
    CT2_REQUIRE(result != nullptr, "null result");
    const long long n = (long long)nx * ny * nz;
    if (n > 0) CT2_REQUIRE(smat != nullptr, "null smat");
    cudaStream_t st = ST(stream);
    Scratch S(st);
    double* partial = nullptr;
    if ((rc = S.get((void**)&partial, sizeof(double) * tv_parts(n), false))) return rc;
    return tv_value(smat, nx, ny, nz, ambdala, result, partial, st);
}
int ct2_totalvar_total_var3d(float ambdala, const float* smat, int nx, int ny, int nz,
                             float* result)
{
    clear_error();
    int rc = check_vol(nx, ny, nz);
    if (rc) return rc;
    const size_t n = (size_t)nx * ny * nz;
    HostCall H;
    float *d_s = nullptr, *d_r = nullptr;
    if ((rc = H.upload((void**)&d_s, smat, n * 4))) return rc;
    if ((rc = H.alloc((void**)&d_r, 4, false))) return rc;
    if ((rc = ct2_dev_totalvar_total_var3d(ambdala, d_s, nx, ny, nz, d_r, H.st))) return rc;
    if ((rc = H.download(result, d_r, 4))) return rc;
    return H.finish();
}

// --- the p-variants (totalvar.f:4-471) ---

static int dev_tvp_grad(int kind, float ppp, float* tvgmat, const float* smat, int nx, int ny,
                        int nz, float dx, float dy, float dz, int normalizeq, float* bobo,
                        cudaStream_t st)
{
    clear_error();
    int rc = check_vol(nx, ny, nz);
    if (rc) return rc;
    CT2_REQUIRE(bobo != nullptr, "null bobo");
    CT2_REQUIRE(std::isfinite(ppp), "p must be finite");
    if (kind == 1)
        CT2_REQUIRE(std::isfinite(dx) && std::isfinite(dy) && std::isfinite(dz) && dx != 0.f &&
                        dy != 0.f && dz != 0.f,
                    "spacings must be finite and nonzero");
    const long long n = (long long)nx * ny * nz;
    if (n > 0) CT2_REQUIRE(tvgmat && smat, "null tvgmat/smat");
    Scratch S(st);
    double* partial = nullptr;
    if ((rc = S.get((void**)&partial, sizeof(double) * tv_parts(n), false))) return rc;
    return tvp_grad(kind, ppp, dx, dy, dz, smat, tvgmat, nx, ny, nz, normalizeq, bobo, partial, st);
}

static int host_tvp_grad(int kind, float ppp, float* tvgmat, const float* smat, int nx, int ny,
                         int nz, float dx, float dy, float dz, int normalizeq, float* bobo)
{
    clear_error();
    int rc = check_vol(nx, ny, nz);
    if (rc) return rc;
    const size_t n = (size_t)nx * ny * nz;
    HostCall H;
    float *d_s = nullptr, *d_t = nullptr, *d_b = nullptr;
    if ((rc = H.upload((void**)&d_s, smat, n * 4))) return rc;
    if ((rc = H.alloc((void**)&d_t, n * 4, false))) return rc;
    if ((rc = H.alloc((void**)&d_b, 4, false))) return rc;
    if ((rc = dev_tvp_grad(kind, ppp, d_t, d_s, nx, ny, nz, dx, dy, dz, normalizeq, d_b, H.st)))
        return rc;
    if ((rc = H.download(tvgmat, d_t, n * 4))) return rc;
    if ((rc = H.download(bobo, d_b, 4))) return rc;
    return H.finish();
}

static int dev_tvp_value(int kind, float p, const float* smat, int nx, int ny, int nz, float dx,
                         float dy, float dz, float* result, cudaStream_t st)
{
    clear_error();
    int rc = check_vol(nx, ny, nz);
    if (rc) return rc;
    CT2_REQUIRE(result != nullptr, "null result");
    CT2_REQUIRE(std::isfinite(p), "p must be finite");
    const long long n = (long long)nx * ny * nz;
    if (n > 0) CT2_REQUIRE(smat != nullptr, "null smat");
    // total_var3d_p subtracts (nx-1)(ny-1)(nz-1) sqrt(eps)**p in REAL*4 (totalvar.f:115)
    const float eps = 0.000000001f;
    const float shift = kind == 0 ? ((float)nx - 1.f) * ((float)ny - 1.f) * ((float)nz - 1.f) *
                                        powf(sqrtf(eps), p)
                                  : 0.f;
    Scratch S(st);
    double* partial = nullptr;
    if ((rc = S.get((void**)&partial, sizeof(double) * tv_parts(n), false))) return rc;
    return tvp_value(kind, p, dx, dy, dz, smat, nx, ny, nz, shift, result, partial, st);
}

static int host_tvp_value(int kind, float p, const float* smat, int nx, int ny, int nz, float dx,
                          float dy, float dz, float* result)
{
    clear_error();
    int rc = check_vol(nx, ny, nz);
    if (rc) return rc;
    const size_t n = (size_t)nx * ny * nz;
    HostCall H;
    float *d_s = nullptr, *d_r = nullptr;
    if ((rc = H.upload((void**)&d_s, smat, n * 4))) return rc;
    if ((rc = H.alloc((void**)&d_r, 4, false))) return rc;
    if ((rc = dev_tvp_value(kind, p, d_s, nx, ny, nz, dx, dy, dz, d_r, H.st))) return rc;
    if ((rc = H.download(result, d_r, 4))) return rc;
    return H.finish();
}

int ct2_dev_totalvar_gmi(float* smatout, const float* smat, int nx, int ny, int nz, void* stream)
{
    clear_error();
    int rc = check_vol(nx, ny, nz);
    if (rc) return rc;
    if ((long long)nx * ny * nz > 0) CT2_REQUIRE(smatout && smat, "null smatout/smat");
    return gmi(smat, smatout, nx, ny, nz, ST(stream));
}
int ct2_totalvar_gmi(float* smatout, const float* smat, int nx, int ny, int nz)
{
    clear_error();
    int rc = check_vol(nx, ny, nz);
    if (rc) return rc;
    const size_t n = (size_t)nx * ny * nz;
    HostCall H;
    float *d_s = nullptr, *d_o = nullptr;
    if ((rc = H.upload((void**)&d_s, smat, n * 4))) return rc;
    if ((rc = H.alloc((void**)&d_o, n * 4, false))) return rc;
    if ((rc = ct2_dev_totalvar_gmi(d_o, d_s, nx, ny, nz, H.st))) return rc;
    if ((rc = H.download(smatout, d_o, n * 4))) return rc;
    return H.finish();
}

int ct2_dev_totalvar_calc_lp(float p, const float* smat, int nx, int ny, int nz, float* result,
                             void* stream)
{
    return dev_tvp_value(2, p, smat, nx, ny, nz, 1.f, 1.f, 1.f, result, ST(stream));
}
int ct2_totalvar_calc_lp(float p, const float* smat, int nx, int ny, int nz, float* result)
{
    return host_tvp_value(2, p, smat, nx, ny, nz, 1.f, 1.f, 1.f, result);
}
int ct2_dev_totalvar_total_var3d_p(float p, const float* smat, int nx, int ny, int nz,
                                   float* result, void* stream)
{
    return dev_tvp_value(0, p, smat, nx, ny, nz, 1.f, 1.f, 1.f, result, ST(stream));
}
int ct2_totalvar_total_var3d_p(float p, const float* smat, int nx, int ny, int nz, float* result)
{
    return host_tvp_value(0, p, smat, nx, ny, nz, 1.f, 1.f, 1.f, result);
}
int ct2_dev_totalvar_total_dvar3d_p(float p, const float* smat, int nx, int ny, int nz, float dx,
                                    float dy, float dz, float* result, void* stream)
{
    return dev_tvp_value(1, p, smat, nx, ny, nz, dx, dy, dz, result, ST(stream));
}
int ct2_totalvar_total_dvar3d_p(float p, const float* smat, int nx, int ny, int nz, float dx,
                                float dy, float dz, float* result)
{
    return host_tvp_value(1, p, smat, nx, ny, nz, dx, dy, dz, result);
}
int ct2_dev_totalvar_lp_grad3d(float ppp, float* tvgmat, const float* smat, int nx, int ny, int nz,
                               int normalizeq, float* bobo, void* stream)
{
    return dev_tvp_grad(2, ppp, tvgmat, smat, nx, ny, nz, 1.f, 1.f, 1.f, normalizeq, bobo,
                        ST(stream));
}
int ct2_totalvar_lp_grad3d(float ppp, float* tvgmat, const float* smat, int nx, int ny, int nz,
                           int normalizeq, float* bobo)
{
    return host_tvp_grad(2, ppp, tvgmat, smat, nx, ny, nz, 1.f, 1.f, 1.f, normalizeq, bobo);
}
int ct2_dev_totalvar_total_p_var_grad3d(float ppp, float* tvgmat, const float* smat, int nx,
                                        int ny, int nz, int normalizeq, float* bobo, void* stream)
{
    return dev_tvp_grad(0, ppp, tvgmat, smat, nx, ny, nz, 1.f, 1.f, 1.f, normalizeq, bobo,
                        ST(stream));
}
int ct2_totalvar_total_p_var_grad3d(float ppp, float* tvgmat, const float* smat, int nx, int ny,
                                    int nz, int normalizeq, float* bobo)
{
    return host_tvp_grad(0, ppp, tvgmat, smat, nx, ny, nz, 1.f, 1.f, 1.f, normalizeq, bobo);
}
int ct2_dev_totalvar_total_p_dvar_grad3d(float ppp, float* tvgmat, const float* smat, int nx,
                                         int ny, int nz, float dx, float dy, float dz,
                                         int normalizeq, float* bobo, void* stream)
{
    return dev_tvp_grad(1, ppp, tvgmat, smat, nx, ny, nz, dx, dy, dz, normalizeq, bobo, ST(stream));
}
int ct2_totalvar_total_p_dvar_grad3d(float ppp, float* tvgmat, const float* smat, int nx, int ny,
                                     int nz, float dx, float dy, float dz, int normalizeq,
                                     float* bobo)
{
    return host_tvp_grad(1, ppp, tvgmat, smat, nx, ny, nz, dx, dy, dz, normalizeq, bobo);
}

// ---------------------------------------------------------------------
// radon3D
// ---------------------------------------------------------------------

static int radon_check(float fov, int nsa, int nsb, int ns, int nr, float dr, float r0,
                       GRID_ARGS_DECL)
{
    CT2_REQUIRE(nsa >= 0 && nsb >= 0 && nr >= 0 && ns >= 0, "radon dimensions must be >= 0");
    CT2_REQUIRE((long long)nsa * nsb <= (long long)ns, "source_locations has %d rows, need %d",
                ns, nsa * nsb);
    CT2_REQUIRE(std::isfinite(fov) && std::isfinite(dr) && std::isfinite(r0), "non-finite radon "
                "parameter");
    return check_grid(GRID_ARGS);
}

int ct2_dev_radon3D_spherical_radon_linear(float fov, float* radonmat, const int32_t* indradon,
                                           const float* source_locations, int nsa, int nsb, int ns,
                                           int nr, float dr, float r0, const float* smat,
                                           GRID_ARGS_DECL, void* stream)
{
    clear_error();
    int rc = radon_check(fov, nsa, nsb, ns, nr, dr, r0, GRID_ARGS);
    if (rc) return rc;
    const long long nm = (long long)nsa * nsb * nr;
    if (nm == 0) return CT2_OK;
    CT2_REQUIRE(radonmat && source_locations, "null radonmat/source_locations");
    if ((long long)nx * ny * nz == 0) {
        CT2_CUDA(cudaMemsetAsync(radonmat, 0, nm * 4, ST(stream)));
        return CT2_OK;
    }
    CT2_REQUIRE(smat != nullptr, "null smat");
    RadonArgs a{};
    a.G = make_grid(GRID_ARGS);
    a.fov = fov;
    a.src = source_locations;
    a.ind = indradon;
    a.nsa = nsa; a.nsb = nsb; a.nr = nr;
    a.dr = dr; a.r0 = r0;
    a.x = const_cast<float*>(smat);
    a.out = radonmat;
    return radon_forward(a, ST(stream));
}
int ct2_radon3D_spherical_radon_linear(float fov, float* radonmat, const int32_t* indradon,
                                       const float* source_locations, int nsa, int nsb, int ns,
                                       int nr, float dr, float r0, const float* smat,
                                       GRID_ARGS_DECL)
{
    clear_error();
    int rc = radon_check(fov, nsa, nsb, ns, nr, dr, r0, GRID_ARGS);
    if (rc) return rc;
    const size_t nm = (size_t)nsa * nsb * nr, nvox = (size_t)nx * ny * nz;
    HostCall H;
    int32_t* d_ind = nullptr;
    float *d_src = nullptr, *d_x = nullptr, *d_out = nullptr;
    if ((rc = H.upload((void**)&d_ind, indradon, nm * 4))) return rc;
    if ((rc = H.upload((void**)&d_src, source_locations, (size_t)ns * 12))) return rc;
    if ((rc = H.upload((void**)&d_x, smat, nvox * 4))) return rc;
    if ((rc = H.alloc((void**)&d_out, nm * 4, false))) return rc;
    if ((rc = ct2_dev_radon3D_spherical_radon_linear(fov, d_out, d_ind, d_src, nsa, nsb, ns, nr,
                                                     dr, r0, d_x, GRID_ARGS, H.st)))
        return rc;
    if ((rc = H.download(radonmat, d_out, nm * 4))) return rc;
    return H.finish();
}

int ct2_dev_radon3D_artstep_linear(float reg_fac, float fov, const float* radonmat,
                                   const int32_t* indradon, const float* source_locations, int nsa,
                                   int nsb, int ns, int nr, float dr, float r0, float* smat,
                                   GRID_ARGS_DECL, void* stream)
{
    clear_error();
    int rc = radon_check(fov, nsa, nsb, ns, nr, dr, r0, GRID_ARGS);
    if (rc || (rc = check_finite(reg_fac, "reg_fac"))) return rc;
    const long long nm = (long long)nsa * nsb * nr, nvox = (long long)nx * ny * nz;
    if (nm == 0 || nvox == 0) return CT2_OK;
    CT2_REQUIRE(radonmat && source_locations && smat, "null array argument");
    cudaStream_t st = ST(stream);
    Scratch S(st);
    float* wmat = nullptr;
    if ((rc = S.get((void**)&wmat, nvox * 4, true))) return rc;
    RadonArgs a{};
    a.G = make_grid(GRID_ARGS);
    a.fov = fov;
    a.src = source_locations;
    a.ind = indradon;
    a.nsa = nsa; a.nsb = nsb; a.nr = nr;
    a.dr = dr; a.r0 = r0;
    a.x = smat;
    a.y = radonmat;
    a.reg_fac = reg_fac;
    return radon_art(a, wmat, st);
}
int ct2_radon3D_artstep_linear(float reg_fac, float fov, const float* radonmat,
                               const int32_t* indradon, const float* source_locations, int nsa,
                               int nsb, int ns, int nr, float dr, float r0, float* smat,
                               GRID_ARGS_DECL)
{
    clear_error();
    int rc = radon_check(fov, nsa, nsb, ns, nr, dr, r0, GRID_ARGS);
    if (rc) return rc;
    const size_t nm = (size_t)nsa * nsb * nr, nvox = (size_t)nx * ny * nz;
    HostCall H;
    int32_t* d_ind = nullptr;
    float *d_src = nullptr, *d_x = nullptr, *d_y = nullptr;
    if ((rc = H.upload((void**)&d_ind, indradon, nm * 4))) return rc;
    if ((rc = H.upload((void**)&d_src, source_locations, (size_t)ns * 12))) return rc;
    if ((rc = H.upload((void**)&d_y, radonmat, nm * 4))) return rc;
    if ((rc = H.upload((void**)&d_x, smat, nvox * 4))) return rc;
    if ((rc = ct2_dev_radon3D_artstep_linear(reg_fac, fov, d_y, d_ind, d_src, nsa, nsb, ns, nr, dr,
                                             r0, d_x, GRID_ARGS, H.st)))
        return rc;
    if ((rc = H.download(smat, d_x, nvox * 4))) return rc;
    return H.finish();
}

}  // extern "C"
