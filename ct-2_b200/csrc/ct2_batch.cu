// Batched MLEM+TV iteration of several reconstructions at once (the served
// stream's engine).  No counterpart in the reference: its drivers reconstruct
// one volume at a time.
//
// Each job of the batch (a slot) is one FP32 reconstruction with its own
// geometry and sizes, whose buffers the caller owns: the iterate x, the
// measured data y, the cached sensitivity A^T 1, a volume and a sinogram of
// scratch.  One call of the iteration launches, for all jobs together:
//  * the EM-ratio projection (ratio = y / max(A x, 1e-5), the reference's
//    clamp) as one persistent kernel over (job, view, 32 x 8 pixel tile)
//    work items: the TMA-staged form for every job whose volume admits
//    tensor maps (k_project_tma_batch, the maps in the job's descriptor), the
//    untiled form for the others (k_project_batch);
//  * the matched gather backprojection of the ratios, per round of view
//    blocks (a job's views split into blocks of its ray-table budget; round r
//    holds block r of every job that has one) as five launches over all
//    jobs' items: reset, ray table, x-driven tiles, y-driven tiles, residual
//    rays (ct2_gather.cu);
//  * each job's fused update x <- max(0, xe - w ||xe - x|| g / ||g||) with
//    xe = x * A^T ratio / A^T 1 (four passes per job).
// Every work item runs the code of the single-job kernels, so a job's result
// is the same alone and in the batch.  The per-job descriptors live in device
// memory written by ct2_batch_commit; the iteration itself allocates nothing
// and synchronises nothing, so a caller can capture it in a CUDA graph and
// replay it while the batch is unchanged.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "ct2_capi_util.h"
#include "ct2_kernels.h"
#include "ct2_precision.h"

namespace ct2 {
namespace {

constexpr float kEmSmall = 0.00001f;  // emstep_linear's clamp (view_proj3D.f:2801-2827)

struct Slot {
    bool used = false;
    float* x = nullptr;
    const float* y = nullptr;
    const float* sens = nullptr;
    float* ws = nullptr;
    float* ratio = nullptr;
    const float* geom = nullptr;
    int ns = 0, nu = 0, nv = 0;
    float du = 0.f, dv = 0.f, u0 = 0.f, v0 = 0.f;
    Grid G{};
    float tv_weight = 0.f;
    int vb = 0, nblocks = 0;
    void* table = nullptr;      // one view block's ray table
    double* partial = nullptr;  // FP64 norm partials of the update
    int parts = 0;
};

struct Engine {
    int dev = 0;
    int sms = 0;
    std::vector<Slot> slots;
    ProjectJob* d_proj = nullptr;  // the TMA-staged jobs, then the untiled ones
    int cap_proj = 0;
    int nproj = 0;
    int ntma = 0;
    long long tma_total = 0, plain_total = 0;
    unsigned long long* d_counters = nullptr;  // 1 (projector) + 3 per round
    int cap_counters = 0;
    char* d_gather = nullptr;
    size_t cap_gather = 0;
    std::vector<int> round_jobs;
    std::vector<long long> round_totals;  // 3 per round
    std::vector<size_t> round_offset;     // bytes into d_gather
    bool committed = false;
};

// Stream-ordered: after the work already queued on st.
void free_slot(Slot& s, cudaStream_t st)
{
    if (s.table) cudaFreeAsync(s.table, st);
    if (s.partial) cudaFreeAsync(s.partial, st);
    s = Slot{};
}

}  // namespace
}  // namespace ct2

using namespace ct2;

extern "C" {

int ct2_batch_create(int max_jobs, void** handle)
{
    clear_error();
    CT2_REQUIRE(handle != nullptr, "null handle");
    *handle = nullptr;
    CT2_REQUIRE(max_jobs >= 1 && max_jobs <= 256, "max_jobs must be in [1, 256] (got %d)",
                max_jobs);
    int dev = 0, sms = 0;
    CT2_CUDA(cudaGetDevice(&dev));
    CT2_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    Engine* E = new (std::nothrow) Engine();
    if (E == nullptr) return set_error(CT2_ENOMEM, "batch engine");
    E->dev = dev;
    E->sms = sms;
    E->slots.resize(max_jobs);
    *handle = E;
    return CT2_OK;
}

int ct2_batch_destroy(void* handle)
{
    clear_error();
    if (handle == nullptr) return CT2_OK;
    Engine* E = reinterpret_cast<Engine*>(handle);
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(E->dev);
    cudaDeviceSynchronize();
    for (Slot& s : E->slots) free_slot(s, nullptr);
    if (E->d_proj) cudaFreeAsync(E->d_proj, nullptr);
    if (E->d_counters) cudaFreeAsync(E->d_counters, nullptr);
    if (E->d_gather) cudaFreeAsync(E->d_gather, nullptr);
    cudaDeviceSynchronize();
    cudaSetDevice(prev);
    delete E;
    return CT2_OK;
}

int ct2_batch_set(void* handle, int slot, float* x, const float* y, const float* sens, float* ws,
                  float* ratio, const float* frame_vectors, int ns, int nu, int nv, float du,
                  float dv, float u0, float v0, float dx, float dy, float dz, float x0, float y0,
                  float z0, int nx, int ny, int nz, float tv_weight, void* stream)
{
    clear_error();
    CT2_REQUIRE(handle != nullptr, "null handle");
    Engine* E = reinterpret_cast<Engine*>(handle);
    CT2_REQUIRE(slot >= 0 && slot < (int)E->slots.size(), "slot %d outside [0, %d)", slot,
                (int)E->slots.size());
    CT2_REQUIRE(x && y && sens && ws && ratio && frame_vectors, "null buffer");
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    rc = check_grid(dx, dy, dz, x0, y0, z0, nx, ny, nz);
    if (rc) return rc;
    CT2_REQUIRE(ns >= 1 && nu >= 1 && nv >= 1 && nx >= 2 && ny >= 2 && nz >= 2,
                "a batched job needs views, detector pixels and at least 2 voxels per axis");
    CT2_REQUIRE(std::isfinite(tv_weight) && tv_weight >= 0.f, "tv_weight must be finite and >= 0");
    int cur = 0;
    CT2_CUDA(cudaGetDevice(&cur));
    CT2_REQUIRE(cur == E->dev, "the batch lives on device %d; the current device is %d", E->dev,
                cur);
    Slot S;
    S.used = true;
    S.x = x;
    S.y = y;
    S.sens = sens;
    S.ws = ws;
    S.ratio = ratio;
    S.geom = frame_vectors;
    S.ns = ns;
    S.nu = nu;
    S.nv = nv;
    S.du = du;
    S.dv = dv;
    S.u0 = u0;
    S.v0 = v0;
    S.G = make_grid(dx, dy, dz, x0, y0, z0, nx, ny, nz);
    S.tv_weight = tv_weight;
    S.vb = gather_block_views(ns, nu, nv);
    S.nblocks = (ns + S.vb - 1) / S.vb;
    // the gather must apply to every view block of the job
    {
        std::vector<char> probe(gather_job_bytes());
        BackprojectArgs b{};
        b.G = S.G;
        b.sino = ratio;
        b.geom = frame_vectors;
        b.ns = ns;
        b.nu = nu;
        b.nv = nv;
        b.du = du;
        b.dv = dv;
        b.u0 = u0;
        b.v0 = v0;
        b.out = ws;
        if (gather_job_fill(probe.data(), b, 0, S.vb, nullptr) != CT2_OK)
            return set_error(CT2_EINVAL, "geometry outside the gather backprojector's range");
    }
    S.parts = prec_parts((long long)nx * ny * nz);
    const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMallocAsync(&S.table, gather_scratch_bytes(nu, nv, S.vb), st);
    if (e == cudaSuccess)
        e = cudaMallocAsync((void**)&S.partial, sizeof(double) * (2 * S.parts + 1), st);
    if (e != cudaSuccess) {
        free_slot(S, st);
        cudaGetLastError();
        return set_error(e == cudaErrorMemoryAllocation ? CT2_ENOMEM : CT2_ECUDA,
                         "batch slot scratch: %s", cudaGetErrorString(e));
    }
    if (E->slots[slot].used) free_slot(E->slots[slot], st);
    E->slots[slot] = S;
    E->committed = false;
    return CT2_OK;
}

int ct2_batch_clear(void* handle, int slot, void* stream)
{
    clear_error();
    CT2_REQUIRE(handle != nullptr, "null handle");
    Engine* E = reinterpret_cast<Engine*>(handle);
    CT2_REQUIRE(slot >= 0 && slot < (int)E->slots.size(), "slot %d outside [0, %d)", slot,
                (int)E->slots.size());
    if (E->slots[slot].used) {
        free_slot(E->slots[slot], reinterpret_cast<cudaStream_t>(stream));
        E->committed = false;
    }
    return CT2_OK;
}

int ct2_batch_commit(void* handle, void* stream, int* njobs)
{
    clear_error();
    CT2_REQUIRE(handle != nullptr, "null handle");
    Engine* E = reinterpret_cast<Engine*>(handle);
    std::vector<const Slot*> jobs;
    for (const Slot& s : E->slots)
        if (s.used) jobs.push_back(&s);
    const int n = (int)jobs.size();
    if (njobs) *njobs = n;
    // projector descriptors: the TMA-staged jobs first, then the untiled
    std::vector<ProjectJob> tma, plain;
    long long tma_total = 0, plain_total = 0;
    for (int j = 0; j < n; j++) {
        const Slot& s = *jobs[j];
        ProjectJob J;
        memset(&J, 0, sizeof(J));
        ProjectArgs& a = J.a;
        a.G = s.G;
        a.vol = s.x;
        a.geom = s.geom;
        a.ind = nullptr;
        a.ns = s.ns;
        a.nu = s.nu;
        a.nv = s.nv;
        a.du = s.du;
        a.dv = s.dv;
        a.u0 = s.u0;
        a.v0 = s.v0;
        a.out = s.ratio;
        a.y = s.y;
        a.em_small = kEmSmall;
        const long long items = (long long)s.ns * project_batch_items(a);
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
    std::vector<ProjectJob> pj(tma);
    pj.insert(pj.end(), plain.begin(), plain.end());
    // gather descriptors, round by round
    int rounds = 0;
    for (const Slot* s : jobs) rounds = std::max(rounds, s->nblocks);
    const size_t jb = gather_job_bytes();
    std::vector<char> gd;
    E->round_jobs.assign(rounds, 0);
    E->round_totals.assign(3 * (size_t)rounds, 0);
    E->round_offset.assign(rounds, 0);
    for (int r = 0; r < rounds; r++) {
        E->round_offset[r] = gd.size();
        int m = 0;
        for (const Slot* s : jobs) {
            if (r >= s->nblocks) continue;
            gd.resize(gd.size() + jb);
            BackprojectArgs b{};
            b.G = s->G;
            b.sino = s->ratio;
            b.geom = s->geom;
            b.ns = s->ns;
            b.nu = s->nu;
            b.nv = s->nv;
            b.du = s->du;
            b.dv = s->dv;
            b.u0 = s->u0;
            b.v0 = s->v0;
            b.out = s->ws;
            const int view0 = r * s->vb, nb = std::min(s->vb, s->ns - view0);
            if (gather_job_fill(gd.data() + gd.size() - jb, b, view0, nb, s->table) != CT2_OK)
                return set_error(CT2_EINVAL, "geometry outside the gather backprojector's range");
            m++;
        }
        E->round_jobs[r] = m;
        gather_jobs_finalize(gd.data() + E->round_offset[r], m, &E->round_totals[3 * (size_t)r]);
        // keep every round's descriptors 256-byte aligned
        gd.resize((gd.size() + 255) & ~(size_t)255);
    }
    // stream-ordered after the batch's earlier iterations on st, which read
    // the old descriptors
    const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int ncount = 1 + 3 * rounds;
    if (ncount > E->cap_counters) {
        if (E->d_counters) cudaFreeAsync(E->d_counters, st);
        E->d_counters = nullptr;
        E->cap_counters = 0;
        CT2_CUDA(cudaMallocAsync((void**)&E->d_counters, sizeof(unsigned long long) * ncount, st));
        E->cap_counters = ncount;
    }
    if (n > E->cap_proj) {
        if (E->d_proj) cudaFreeAsync(E->d_proj, st);
        E->d_proj = nullptr;
        E->cap_proj = 0;
        CT2_CUDA(cudaMallocAsync((void**)&E->d_proj, sizeof(ProjectJob) * n, st));
        E->cap_proj = n;
    }
    if (gd.size() > E->cap_gather) {
        if (E->d_gather) cudaFreeAsync(E->d_gather, st);
        E->d_gather = nullptr;
        E->cap_gather = 0;
        CT2_CUDA(cudaMallocAsync((void**)&E->d_gather, gd.size(), st));
        E->cap_gather = gd.size();
    }
    if (n)
        CT2_CUDA(cudaMemcpyAsync(E->d_proj, pj.data(), sizeof(ProjectJob) * n,
                                 cudaMemcpyHostToDevice, st));
    if (!gd.empty())
        CT2_CUDA(cudaMemcpyAsync(E->d_gather, gd.data(), gd.size(), cudaMemcpyHostToDevice, st));
    CT2_CUDA(cudaStreamSynchronize(st));  // the host copies are done with pj and gd
    E->nproj = n;
    E->ntma = (int)tma.size();
    E->tma_total = tma_total;
    E->plain_total = plain_total;
    E->committed = true;
    return CT2_OK;
}

int ct2_batch_em_iteration(void* handle, void* stream)
{
    clear_error();
    CT2_REQUIRE(handle != nullptr, "null handle");
    Engine* E = reinterpret_cast<Engine*>(handle);
    CT2_REQUIRE(E->committed, "the batch changed since its last ct2_batch_commit");
    const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (E->nproj == 0) return CT2_OK;
    CT2_CUDA(cudaMemsetAsync(E->d_counters, 0, sizeof(unsigned long long), st));
    int rc = project_batch(E->d_proj, E->ntma, E->tma_total, true, true, E->sms * 4,
                           E->d_counters, st);
    if (rc) return rc;
    rc = project_batch(E->d_proj + E->ntma, E->nproj - E->ntma, E->plain_total, false, true,
                       E->sms * 8, nullptr, st);
    if (rc) return rc;
    for (const Slot& s : E->slots)
        if (s.used)
            CT2_CUDA(cudaMemsetAsync(s.ws, 0, sizeof(float) * (size_t)s.G.n[0] * s.G.n[1] * s.G.n[2],
                                     st));
    for (size_t r = 0; r < E->round_jobs.size(); r++) {
        rc = gather_batch_round(E->d_gather + E->round_offset[r], E->round_jobs[r],
                                &E->round_totals[3 * r], E->sms * 8, E->d_counters + 1 + 3 * r,
                                st);
        if (rc) return rc;
    }
    for (const Slot& s : E->slots) {
        if (!s.used) continue;
        rc = prec_em_tv_update(s.x, CT2_F32, s.ws, s.sens, s.G.n[0], s.G.n[1], s.G.n[2], kEmSmall,
                               s.tv_weight, s.partial, s.partial + 2 * s.parts, st);
        if (rc) return rc;
    }
    return CT2_OK;
}

}  // extern "C"
