// Several volumes through one view geometry, one launch per kernel for all of
// them (the differentiable workload's batch of volumes).  No counterpart in
// the reference, whose modules project one volume per call.
//
// ct2_dev_view_proj3D_sinoproj_linear_many: the projector of every volume as
// one persistent launch over (volume, view, 32 x 8 pixel tile) work items --
// the TMA-staged form where a volume admits tensor maps, the untiled form
// otherwise -- every pixel computed exactly as the single-volume projector
// computes it.
// ct2_dev_view_proj3D_sinobackproject_linear_many: the gather backprojector
// of every sinogram, per round of view blocks, as the batched table, tile and
// residual kernels over all volumes' items (groups of volumes whose ray
// tables together stay within kGroupScratch); with the scatter backprojector
// selected (ct2_set_backprojector(1)) or outside the gather's range, one
// single-volume backprojection per volume.  Each volume's result equals its
// own single-volume call bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "ct2_capi_util.h"
#include "ct2_kernels.h"

namespace ct2 {
namespace {

constexpr size_t kGroupScratch = 2ull << 30;  // ray tables of one group of volumes

int num_sms()
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    return sms;
}

int check_many(int nvol, int ns, int nu, int nv, float du, float dv, float u0, float v0,
               float dx, float dy, float dz, float x0, float y0, float z0, int nx, int ny, int nz)
{
    CT2_REQUIRE(nvol >= 0 && nvol <= 4096, "nvol must be in [0, 4096] (got %d)", nvol);
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    return check_grid(dx, dy, dz, x0, y0, z0, nx, ny, nz);
}

}  // namespace
}  // namespace ct2

using namespace ct2;

extern "C" {

int ct2_dev_view_proj3D_sinoproj_linear_many(int nvol, float* sinomat,
                                             const float* frame_vectors, int ns, int nu, int nv,
                                             float du, float dv, float u0, float v0,
                                             const float* smat, float dx, float dy, float dz,
                                             float x0, float y0, float z0, int nx, int ny, int nz,
                                             void* stream)
{
    clear_error();
    int rc = check_many(nvol, ns, nu, nv, du, dv, u0, v0, dx, dy, dz, x0, y0, z0, nx, ny, nz);
    if (rc) return rc;
    const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const long long nrays = (long long)ns * nu * nv, nvox = (long long)nx * ny * nz;
    if (nvol == 0 || nrays == 0) return CT2_OK;
    CT2_REQUIRE(sinomat && frame_vectors, "null sinomat/frame_vectors");
    if (nvox == 0) {
        CT2_CUDA(cudaMemsetAsync(sinomat, 0, sizeof(float) * nrays * nvol, st));
        return CT2_OK;
    }
    CT2_REQUIRE(smat != nullptr, "null smat");
    const Grid G = make_grid(dx, dy, dz, x0, y0, z0, nx, ny, nz);
    std::vector<ProjectJob> tma, plain;
    long long tma_total = 0, plain_total = 0;
    for (int b = 0; b < nvol; b++) {
        ProjectJob J;
        memset(&J, 0, sizeof(J));
        ProjectArgs& a = J.a;
        a.G = G;
        a.vol = smat + b * nvox;
        a.geom = frame_vectors;
        a.ns = ns;
        a.nu = nu;
        a.nv = nv;
        a.du = du;
        a.dv = dv;
        a.u0 = u0;
        a.v0 = v0;
        a.out = sinomat + b * nrays;
        const long long items = (long long)ns * project_batch_items(a);
        if (encode_volume_maps(a, &J.mapx, &J.mapy) == CT2_OK) {
            J.item0 = tma_total;
            tma_total += items;
            tma.push_back(J);
        } else {
            J.item0 = plain_total;
            plain_total += items;
            plain.push_back(J);
        }
    }
    std::vector<ProjectJob> all(tma);
    all.insert(all.end(), plain.begin(), plain.end());
    Scratch S(st);
    ProjectJob* d_jobs = nullptr;
    unsigned long long* counter = nullptr;
    if ((rc = S.get((void**)&d_jobs, sizeof(ProjectJob) * all.size(), false))) return rc;
    if ((rc = S.get((void**)&counter, sizeof(unsigned long long), true))) return rc;
    CT2_CUDA(cudaMemcpyAsync(d_jobs, all.data(), sizeof(ProjectJob) * all.size(),
                             cudaMemcpyHostToDevice, st));
    const int sms = num_sms();
    rc = project_batch(d_jobs, (int)tma.size(), tma_total, true, false, sms * 4, counter, st);
    if (rc) return rc;
    return project_batch(d_jobs + tma.size(), (int)plain.size(), plain_total, false, false,
                         sms * 8, nullptr, st);
}

int ct2_dev_view_proj3D_sinobackproject_linear_many(int nvol, const float* sinomat,
                                                    const float* frame_vectors, int ns, int nu,
                                                    int nv, float du, float dv, float u0,
                                                    float v0, float* smat, float dx, float dy,
                                                    float dz, float x0, float y0, float z0,
                                                    int nx, int ny, int nz, void* stream)
{
    clear_error();
    int rc = check_many(nvol, ns, nu, nv, du, dv, u0, v0, dx, dy, dz, x0, y0, z0, nx, ny, nz);
    if (rc) return rc;
    const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const long long nrays = (long long)ns * nu * nv, nvox = (long long)nx * ny * nz;
    if (nvol == 0 || nvox == 0) return CT2_OK;
    CT2_REQUIRE(smat != nullptr, "null smat");
    CT2_CUDA(cudaMemsetAsync(smat, 0, sizeof(float) * nvox * nvol, st));
    if (nrays == 0) return CT2_OK;
    CT2_REQUIRE(sinomat && frame_vectors, "null sinomat/frame_vectors");
    BackprojectArgs a{};
    a.G = make_grid(dx, dy, dz, x0, y0, z0, nx, ny, nz);
    a.geom = frame_vectors;
    a.ns = ns;
    a.nu = nu;
    a.nv = nv;
    a.du = du;
    a.dv = dv;
    a.u0 = u0;
    a.v0 = v0;
    a.sino = sinomat;
    a.out = smat;
    if (!gather_batch_applies(a)) {
        // the scatter (or a geometry outside the gather's range): volume by volume
        for (int b = 0; b < nvol; b++) {
            a.sino = sinomat + b * nrays;
            a.out = smat + b * nvox;
            if ((rc = backproject(a, MODE_LINEAR, false, false, st))) return rc;
        }
        return CT2_OK;
    }
    const int vb = gather_block_views(ns, nu, nv);
    const size_t scratch = gather_scratch_bytes(nu, nv, vb);
    const int group = (int)std::max<size_t>(1, std::min<size_t>(nvol, kGroupScratch / scratch));
    const size_t jb = gather_job_bytes();
    const int grid = num_sms() * 8;
    Scratch S(st);
    char* tables = nullptr;
    char* d_desc = nullptr;
    unsigned long long* counters = nullptr;
    if ((rc = S.get((void**)&tables, scratch * group, false))) return rc;
    if ((rc = S.get((void**)&d_desc, jb * group, false))) return rc;
    if ((rc = S.get((void**)&counters, 3 * sizeof(unsigned long long), false))) return rc;
    std::vector<char> desc(jb * group);
    for (int b0 = 0; b0 < nvol; b0 += group) {
        const int m = std::min(group, nvol - b0);
        for (int view0 = 0; view0 < ns; view0 += vb) {
            const int nb = std::min(vb, ns - view0);
            for (int j = 0; j < m; j++) {
                a.sino = sinomat + (b0 + j) * nrays;
                a.out = smat + (b0 + j) * nvox;
                if (gather_job_fill(desc.data() + j * jb, a, view0, nb, tables + j * scratch) !=
                    CT2_OK)
                    return set_error(CT2_EINVAL, "geometry outside the gather's range");
            }
            long long totals[3];
            gather_jobs_finalize(desc.data(), m, totals);
            // the descriptors of the previous round are read by kernels queued
            // before this copy on the same stream
            CT2_CUDA(cudaMemcpyAsync(d_desc, desc.data(), jb * m, cudaMemcpyHostToDevice, st));
            if ((rc = gather_batch_round(d_desc, m, totals, grid, counters, st))) return rc;
        }
    }
    return CT2_OK;
}

}  // extern "C"
