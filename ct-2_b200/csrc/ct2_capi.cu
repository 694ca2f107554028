// C ABI: argument validation, the stream-ordered device entry points, and
// the host-pointer entry points that stage through device memory.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "ct2_capi_util.h"
#include "ct2_kernels.h"

namespace ct2 {

static thread_local char g_msg[1024] = "";

int set_error(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
    va_end(ap);
    return code;
}

int clear_error()
{
    g_msg[0] = 0;
    return CT2_OK;
}

std::atomic<unsigned long long> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// Keep freed blocks in the device's stream-ordered pool between calls (the
// default release threshold of 0 hands them back at every synchronisation,
// and the next call maps them again), once per device.
static void keep_pool_memory(int dev)
{
    static std::mutex m;
    static std::map<int, bool> done;
    std::lock_guard<std::mutex> g(m);
    if (done[dev]) return;
    done[dev] = true;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
}

cudaStream_t lib_stream()
{
    static thread_local std::map<int, cudaStream_t> streams;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    auto it = streams.find(dev);
    if (it != streams.end()) return it->second;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    keep_pool_memory(dev);
    streams[dev] = s;
    return s;
}

int check_grid(float dx, float dy, float dz, float x0, float y0, float z0, int nx, int ny, int nz)
{
    CT2_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, "volume dimensions must be >= 0 (got %d,%d,%d)", nx,
                ny, nz);
    CT2_REQUIRE(std::isfinite(dx) && std::isfinite(dy) && std::isfinite(dz) && dx > 0.f &&
                    dy > 0.f && dz > 0.f,
                "voxel spacings must be finite and > 0 (got %g,%g,%g)", dx, dy, dz);
    CT2_REQUIRE(std::isfinite(x0) && std::isfinite(y0) && std::isfinite(z0),
                "volume origin must be finite");
    CT2_REQUIRE((long long)nx * ny < (1ll << 31) && (long long)nx * nz < (1ll << 31) &&
                    (long long)ny * nz < (1ll << 31),
                "volume plane exceeds 2^31 voxels");
    CT2_REQUIRE(nx < (1 << 22) && ny < (1 << 22) && nz < (1 << 22),
                "volume dimension exceeds 2^22");
    return CT2_OK;
}

int check_view(int ns, int nu, int nv, float du, float dv, float u0, float v0)
{
    CT2_REQUIRE(ns >= 0 && nu >= 0 && nv >= 0, "sinogram dimensions must be >= 0 (got %d,%d,%d)",
                ns, nu, nv);
    CT2_REQUIRE(std::isfinite(du) && std::isfinite(dv) && std::isfinite(u0) && std::isfinite(v0),
                "detector spacing and origin must be finite");
    CT2_REQUIRE(ns < 65536, "at most 65535 views per call (got %d)", ns);
    return CT2_OK;
}

Grid make_grid(float dx, float dy, float dz, float x0, float y0, float z0, int nx, int ny, int nz)
{
    Grid G;
    G.d[0] = dx; G.d[1] = dy; G.d[2] = dz;
    G.o[0] = x0; G.o[1] = y0; G.o[2] = z0;
    G.n[0] = nx; G.n[1] = ny; G.n[2] = nz;
    G.s[0] = (long long)ny * nz;
    G.s[1] = nz;
    G.s[2] = 1;
    G.small = ((long long)nx * ny * nz) < (1ll << 32) ? 1 : 0;
    return G;
}

// ---- host staging ----------------------------------------------------

HostCall::HostCall() : st(lib_stream()) {}

HostCall::~HostCall()
{
    for (void* p : bufs) cudaFreeAsync(p, st);
    if (st) cudaStreamSynchronize(st);
}

int HostCall::alloc(void** d, size_t bytes, bool zero)
{
    *d = nullptr;
    if (st == nullptr) return set_error(CT2_ECUDA, "no CUDA device/stream available");
    if (bytes == 0) return CT2_OK;
    CT2_CUDA(cudaMallocAsync(d, bytes, st));
    bufs.push_back(*d);
    if (zero) CT2_CUDA(cudaMemsetAsync(*d, 0, bytes, st));
    return CT2_OK;
}

int HostCall::upload(void** d, const void* h, size_t bytes)
{
    *d = nullptr;
    if (h == nullptr || bytes == 0) return CT2_OK;
    int rc = alloc(d, bytes, false);
    if (rc) return rc;
    CT2_CUDA(cudaMemcpyAsync(*d, h, bytes, cudaMemcpyHostToDevice, st));
    return CT2_OK;
}

int HostCall::download(void* h, const void* d, size_t bytes)
{
    if (bytes == 0) return CT2_OK;
    CT2_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st));
    return CT2_OK;
}

int HostCall::finish()
{
    CT2_CUDA(cudaStreamSynchronize(st));
    CT2_CUDA(cudaGetLastError());
    return CT2_OK;
}

// ---- scratch for the device entry points -----------------------------

Scratch::Scratch(cudaStream_t s) : st(s) {}
Scratch::~Scratch()
{
    for (void* p : bufs) cudaFreeAsync(p, st);
}
int Scratch::get(void** d, size_t bytes, bool zero)
{
    *d = nullptr;
    if (bytes == 0) return CT2_OK;
    int dev = 0;
    CT2_CUDA(cudaGetDevice(&dev));
    keep_pool_memory(dev);
    CT2_CUDA(cudaMallocAsync(d, bytes, st));
    bufs.push_back(*d);
    if (zero) CT2_CUDA(cudaMemsetAsync(*d, 0, bytes, st));
    return CT2_OK;
}

}  // namespace ct2

using namespace ct2;

#define ST(stream) ((cudaStream_t)(stream))

// =====================================================================
// view_proj3D / view_proj3D_tomo: projectors
// =====================================================================

static int dev_view_project(int mode, bool force_z, float* sinomat, const int32_t* indsino,
                            const float* fv, int ns, int nu, int nv, float du, float dv, float u0,
                            float v0, const float* smat, float dx, float dy, float dz, float x0,
                            float y0, float z0, int nx, int ny, int nz, cudaStream_t st)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    rc = check_grid(dx, dy, dz, x0, y0, z0, nx, ny, nz);
    if (rc) return rc;
    const long long nrays = (long long)ns * nu * nv;
    if (nrays == 0) return CT2_OK;
    CT2_REQUIRE(sinomat && fv, "null sinomat/frame_vectors");
    if ((long long)nx * ny * nz == 0) {
        CT2_CUDA(cudaMemsetAsync(sinomat, 0, sizeof(float) * nrays, st));
        return CT2_OK;
    }
    CT2_REQUIRE(smat != nullptr, "null smat");
    ProjectArgs a{};
    a.G = make_grid(dx, dy, dz, x0, y0, z0, nx, ny, nz);
    a.vol = smat;
    a.geom = fv;
    a.ind = indsino;
    a.ns = ns; a.nu = nu; a.nv = nv;
    a.du = du; a.dv = dv; a.u0 = u0; a.v0 = v0;
    a.out = sinomat;
    return project(a, mode, false, force_z, false, st);
}

static int dev_view_backproject(int mode, bool force_z, const float* sinomat,
                                const int32_t* indsino, const float* fv, int ns, int nu, int nv,
                                float du, float dv, float u0, float v0, float* smat, float dx,
                                float dy, float dz, float x0, float y0, float z0, int nx, int ny,
                                int nz, cudaStream_t st)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    rc = check_grid(dx, dy, dz, x0, y0, z0, nx, ny, nz);
    if (rc) return rc;
    const long long nvox = (long long)nx * ny * nz;
    if (nvox == 0) return CT2_OK;
    CT2_REQUIRE(smat != nullptr, "null smat");
    CT2_CUDA(cudaMemsetAsync(smat, 0, sizeof(float) * nvox, st));
    if ((long long)ns * nu * nv == 0) return CT2_OK;
    CT2_REQUIRE(sinomat && fv, "null sinomat/frame_vectors");
    BackprojectArgs a{};
    a.G = make_grid(dx, dy, dz, x0, y0, z0, nx, ny, nz);
    a.sino = sinomat;
    a.ind = indsino;
    a.geom = fv;
    a.ns = ns; a.nu = nu; a.nv = nv;
    a.du = du; a.dv = dv; a.u0 = u0; a.v0 = v0;
    a.out = smat;
    a.out_ones = nullptr;
    return backproject(a, mode, false, force_z, st);
}

// One MLEM step over the view geometry: ratio = y / max(Ax, small) on the
// rays, then A^T ratio and A^T 1 in one brick pass, then the voxel update.
static int dev_view_em(int mode, bool force_z, float small, const float* sinomat,
                       const int32_t* indsino, const float* fv, int ns, int nu, int nv, float du,
                       float dv, float u0, float v0, float* smat, float dx, float dy, float dz,
                       float x0, float y0, float z0, int nx, int ny, int nz, cudaStream_t st)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    rc = check_grid(dx, dy, dz, x0, y0, z0, nx, ny, nz);
    if (rc) return rc;
    const long long nvox = (long long)nx * ny * nz;
    const long long nrays = (long long)ns * nu * nv;
    if (nvox == 0) return CT2_OK;
    CT2_REQUIRE(smat != nullptr, "null smat");
    Scratch S(st);
    float *ratio = nullptr, *ws = nullptr, *ones = nullptr;
    if ((rc = S.get((void**)&ws, sizeof(float) * nvox, true))) return rc;
    if ((rc = S.get((void**)&ones, sizeof(float) * nvox, true))) return rc;
    if (nrays > 0) {
        CT2_REQUIRE(sinomat && fv, "null sinomat/frame_vectors");
        if ((rc = S.get((void**)&ratio, sizeof(float) * nrays, false))) return rc;
        const Grid G = make_grid(dx, dy, dz, x0, y0, z0, nx, ny, nz);
        ProjectArgs p{};
        p.G = G;
        p.vol = smat;
        p.geom = fv;
        p.ind = indsino;
        p.ns = ns; p.nu = nu; p.nv = nv;
        p.du = du; p.dv = dv; p.u0 = u0; p.v0 = v0;
        p.out = ratio;
        p.y = sinomat;
        p.em_small = small;
        if ((rc = project(p, mode, false, force_z, true, st))) return rc;
        BackprojectArgs b{};
        b.G = G;
        b.sino = ratio;
        b.ind = indsino;
        b.geom = fv;
        b.ns = ns; b.nu = nu; b.nv = nv;
        b.du = du; b.dv = dv; b.u0 = u0; b.v0 = v0;
        b.out = ws;
        b.out_ones = ones;
        if ((rc = backproject(b, mode, false, force_z, st))) return rc;
    }
    return em_update(smat, ws, ones, nvox, small, st);
}

#define VIEW_ARGS_DECL                                                                      \
    const int32_t *indsino, const float *frame_vectors, int ns, int nu, int nv, float du, \
        float dv, float u0, float v0
#define VIEW_ARGS indsino, frame_vectors, ns, nu, nv, du, dv, u0, v0
#define GRID_ARGS_DECL \
    float dx, float dy, float dz, float x0, float y0, float z0, int nx, int ny, int nz
#define GRID_ARGS dx, dy, dz, x0, y0, z0, nx, ny, nz

// Host staging for a view-geometry projector: in smat, out sinomat.
// ---- host entry points with copy/compute overlap --------------------
//
// The projector and backprojector host calls split the views into blocks and
// pipeline them over three streams: uploads of block b+1 (indicator,
// sinogram) run on a side stream while block b's kernel runs on the call's
// stream and block b-1's sinogram comes back on a third.  With pinned host
// buffers the copies hide behind the kernels; with pageable ones the driver
// stages them and the overlap shrinks, the results being the same.

namespace {

struct SideStreams {
    cudaStream_t in = nullptr, out = nullptr;
};

SideStreams side_streams()
{
    static thread_local std::map<int, SideStreams> m;
    int dev = 0;
    SideStreams s;
    if (cudaGetDevice(&dev) != cudaSuccess) return s;
    auto it = m.find(dev);
    if (it != m.end()) return it->second;
    if (cudaStreamCreateWithFlags(&s.in, cudaStreamNonBlocking) != cudaSuccess) return SideStreams();
    if (cudaStreamCreateWithFlags(&s.out, cudaStreamNonBlocking) != cudaSuccess) {
        cudaStreamDestroy(s.in);
        return SideStreams();
    }
    m[dev] = s;
    return s;
}

// Events of one pipelined call, destroyed after the call's final sync.
struct Events {
    std::vector<cudaEvent_t> ev;
    ~Events()
    {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
    int make(cudaEvent_t* e)
    {
        CT2_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        ev.push_back(*e);
        return CT2_OK;
    }
};

// Constructed after the call's HostCall: on every return, including an error
// part-way, the side streams are drained before HostCall frees the buffers.
struct SideSync {
    SideStreams s;
    explicit SideSync(SideStreams x) : s(x) {}
    ~SideSync()
    {
        if (s.in) cudaStreamSynchronize(s.in);
        if (s.out) cudaStreamSynchronize(s.out);
    }
};

constexpr int kPipeBlocks = 16;

}  // namespace

static int host_view_project(int mode, bool force_z, float* sinomat, VIEW_ARGS_DECL,
                             const float* smat, GRID_ARGS_DECL)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    if ((rc = check_grid(GRID_ARGS))) return rc;
    const size_t per_view = (size_t)nu * nv, nr = (size_t)ns * per_view;
    const size_t nvox = (size_t)nx * ny * nz;
    if (nr == 0) return CT2_OK;
    CT2_REQUIRE(sinomat && frame_vectors, "null sinomat/frame_vectors");
    HostCall H;
    SideStreams S = side_streams();
    if (S.in == nullptr || nvox == 0 || ns < 2) {  // one block: the plain sequence
        int32_t* d_ind = nullptr;
        float *d_fv = nullptr, *d_vol = nullptr, *d_out = nullptr;
        if ((rc = H.upload((void**)&d_ind, indsino, nr * sizeof(int32_t)))) return rc;
        if ((rc = H.upload((void**)&d_fv, frame_vectors, (size_t)ns * 18 * sizeof(float)))) return rc;
        if ((rc = H.upload((void**)&d_vol, smat, nvox * sizeof(float)))) return rc;
        if ((rc = H.alloc((void**)&d_out, nr * sizeof(float), false))) return rc;
        if ((rc = dev_view_project(mode, force_z, d_out, d_ind, d_fv, ns, nu, nv, du, dv, u0, v0,
                                   d_vol, GRID_ARGS, H.st)))
            return rc;
        if ((rc = H.download(sinomat, d_out, nr * sizeof(float)))) return rc;
        return H.finish();
    }
    CT2_REQUIRE(smat != nullptr, "null smat");
    SideSync drain(S);
    int32_t* d_ind = nullptr;
    float *d_fv = nullptr, *d_vol = nullptr, *d_out = nullptr;
    if (indsino && (rc = H.alloc((void**)&d_ind, nr * sizeof(int32_t), false))) return rc;
    if ((rc = H.upload((void**)&d_fv, frame_vectors, (size_t)ns * 18 * sizeof(float)))) return rc;
    if ((rc = H.upload((void**)&d_vol, smat, nvox * sizeof(float)))) return rc;
    if ((rc = H.alloc((void**)&d_out, nr * sizeof(float), false))) return rc;
    Events E;
    cudaEvent_t ready;
    if ((rc = E.make(&ready))) return rc;
    CT2_CUDA(cudaEventRecord(ready, H.st));  // allocations exist before the side streams use them
    CT2_CUDA(cudaStreamWaitEvent(S.in, ready, 0));
    CT2_CUDA(cudaStreamWaitEvent(S.out, ready, 0));
    const Grid G = make_grid(GRID_ARGS);
    const int vb = (ns + kPipeBlocks - 1) / kPipeBlocks;
    for (int v = 0; v < ns; v += vb) {
        const int nb = (v + vb <= ns) ? vb : ns - v;
        const size_t off = (size_t)v * per_view, cnt = (size_t)nb * per_view;
        if (indsino) {
            cudaEvent_t in;
            if ((rc = E.make(&in))) return rc;
            CT2_CUDA(cudaMemcpyAsync(d_ind + off, indsino + off, cnt * sizeof(int32_t),
                                     cudaMemcpyHostToDevice, S.in));
            CT2_CUDA(cudaEventRecord(in, S.in));
            CT2_CUDA(cudaStreamWaitEvent(H.st, in, 0));
        }
        ProjectArgs a{};
        a.G = G;
        a.vol = d_vol;
        a.geom = d_fv + 18 * (size_t)v;
        a.ind = indsino ? d_ind + off : nullptr;
        a.ns = nb; a.nu = nu; a.nv = nv;
        a.du = du; a.dv = dv; a.u0 = u0; a.v0 = v0;
        a.out = d_out + off;
        if ((rc = project(a, mode, false, force_z, false, H.st))) return rc;
        cudaEvent_t done;
        if ((rc = E.make(&done))) return rc;
        CT2_CUDA(cudaEventRecord(done, H.st));
        CT2_CUDA(cudaStreamWaitEvent(S.out, done, 0));
        CT2_CUDA(cudaMemcpyAsync(sinomat + off, d_out + off, cnt * sizeof(float),
                                 cudaMemcpyDeviceToHost, S.out));
    }
    cudaEvent_t copied;
    if ((rc = E.make(&copied))) return rc;
    CT2_CUDA(cudaEventRecord(copied, S.out));
    CT2_CUDA(cudaStreamWaitEvent(H.st, copied, 0));  // frees and the final sync follow the copies
    return H.finish();
}

static int host_view_backproject(int mode, bool force_z, const float* sinomat, VIEW_ARGS_DECL,
                                 float* smat, GRID_ARGS_DECL)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    if ((rc = check_grid(GRID_ARGS))) return rc;
    const size_t per_view = (size_t)nu * nv, nr = (size_t)ns * per_view;
    const size_t nvox = (size_t)nx * ny * nz;
    if (nr == 0) {  // no rays: the zero-filled volume f2py hands back
        if (nvox) {
            CT2_REQUIRE(smat != nullptr, "null smat");
            memset(smat, 0, nvox * sizeof(float));
        }
        return CT2_OK;
    }
    HostCall H;
    SideStreams S = side_streams();
    if (S.in == nullptr || nvox == 0 || ns < 2) {  // one block: the plain sequence
        int32_t* d_ind = nullptr;
        float *d_fv = nullptr, *d_sino = nullptr, *d_out = nullptr;
        if ((rc = H.upload((void**)&d_ind, indsino, nr * sizeof(int32_t)))) return rc;
        if ((rc = H.upload((void**)&d_fv, frame_vectors, (size_t)ns * 18 * sizeof(float)))) return rc;
        if ((rc = H.upload((void**)&d_sino, sinomat, nr * sizeof(float)))) return rc;
        if ((rc = H.alloc((void**)&d_out, nvox * sizeof(float), false))) return rc;
        if ((rc = dev_view_backproject(mode, force_z, d_sino, d_ind, d_fv, ns, nu, nv, du, dv, u0,
                                       v0, d_out, GRID_ARGS, H.st)))
            return rc;
        if ((rc = H.download(smat, d_out, nvox * sizeof(float)))) return rc;
        return H.finish();
    }
    CT2_REQUIRE(smat != nullptr, "null smat");
    CT2_REQUIRE(sinomat && frame_vectors, "null sinomat/frame_vectors");
    SideSync drain(S);
    int32_t* d_ind = nullptr;
    float *d_fv = nullptr, *d_sino = nullptr, *d_out = nullptr;
    if (indsino && (rc = H.alloc((void**)&d_ind, nr * sizeof(int32_t), false))) return rc;
    if ((rc = H.upload((void**)&d_fv, frame_vectors, (size_t)ns * 18 * sizeof(float)))) return rc;
    if ((rc = H.alloc((void**)&d_sino, nr * sizeof(float), false))) return rc;
    if ((rc = H.alloc((void**)&d_out, nvox * sizeof(float), true))) return rc;  // zero-filled
    Events E;
    cudaEvent_t ready;
    if ((rc = E.make(&ready))) return rc;
    CT2_CUDA(cudaEventRecord(ready, H.st));
    CT2_CUDA(cudaStreamWaitEvent(S.in, ready, 0));
    const Grid G = make_grid(GRID_ARGS);
    const int vb = (ns + kPipeBlocks - 1) / kPipeBlocks;
    for (int v = 0; v < ns; v += vb) {
        const int nb = (v + vb <= ns) ? vb : ns - v;
        const size_t off = (size_t)v * per_view, cnt = (size_t)nb * per_view;
        cudaEvent_t in;
        if ((rc = E.make(&in))) return rc;
        CT2_CUDA(cudaMemcpyAsync(d_sino + off, sinomat + off, cnt * sizeof(float),
                                 cudaMemcpyHostToDevice, S.in));
        if (indsino)
            CT2_CUDA(cudaMemcpyAsync(d_ind + off, indsino + off, cnt * sizeof(int32_t),
                                     cudaMemcpyHostToDevice, S.in));
        CT2_CUDA(cudaEventRecord(in, S.in));
        CT2_CUDA(cudaStreamWaitEvent(H.st, in, 0));
        BackprojectArgs b{};
        b.G = G;
        b.sino = d_sino + off;
        b.ind = indsino ? d_ind + off : nullptr;
        b.geom = d_fv + 18 * (size_t)v;
        b.ns = nb; b.nu = nu; b.nv = nv;
        b.du = du; b.dv = dv; b.u0 = u0; b.v0 = v0;
        b.out = d_out;
        b.out_ones = nullptr;
        if ((rc = backproject(b, mode, false, force_z, H.st))) return rc;
    }
    if ((rc = H.download(smat, d_out, nvox * sizeof(float)))) return rc;
    return H.finish();
}

static int host_view_em(int mode, bool force_z, float small, const float* sinomat,
                        VIEW_ARGS_DECL, float* smat, GRID_ARGS_DECL)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    if ((rc = check_grid(GRID_ARGS))) return rc;
    const size_t nr = (size_t)ns * nu * nv, nvox = (size_t)nx * ny * nz;
    HostCall H;
    int32_t* d_ind = nullptr;
    float *d_fv = nullptr, *d_sino = nullptr, *d_vol = nullptr;
    if ((rc = H.upload((void**)&d_ind, indsino, nr * sizeof(int32_t)))) return rc;
    if ((rc = H.upload((void**)&d_fv, frame_vectors, (size_t)ns * 18 * sizeof(float)))) return rc;
    if ((rc = H.upload((void**)&d_sino, sinomat, nr * sizeof(float)))) return rc;
    if ((rc = H.upload((void**)&d_vol, smat, nvox * sizeof(float)))) return rc;
    if ((rc = dev_view_em(mode, force_z, small, d_sino, d_ind, d_fv, ns, nu, nv, du, dv, u0, v0,
                          d_vol, GRID_ARGS, H.st)))
        return rc;
    if ((rc = H.download(smat, d_vol, nvox * sizeof(float)))) return rc;
    return H.finish();
}

extern "C" {

const char* ct2_last_error(void) { return g_msg; }
const char* ct2_version(void) { return "ct2b200 0.1.0 (sm_100a)"; }

int ct2_set_backprojector(int kind)
{
    clear_error();
    return set_backprojector(kind);
}

int ct2_wait_selftest(int spins)
{
    clear_error();
    CT2_REQUIRE(spins >= 1 && spins <= (1 << 20), "spins must be in [1, 2^20]");
    cudaStream_t st = lib_stream();
    if (st == nullptr) return set_error(CT2_ECUDA, "no CUDA device/stream available");
    int timed_out = 0;
    int rc = wait_selftest(spins, st, &timed_out);
    if (rc) return rc;
    if (timed_out)
        return set_error(CT2_ETIMEOUT, "bounded wait gave up after %d tries (self-test)", spins);
    return set_error(CT2_ECUDA, "bounded-wait self-test: a wait nothing completes succeeded");
}

int ct2_wait_timeouts(int* count, int reset)
{
    clear_error();
    CT2_REQUIRE(count != nullptr, "null count");
    return wait_timeouts(count, reset);
}

int ct2_launch_count(unsigned long long* count, int reset)
{
    clear_error();
    CT2_REQUIRE(count != nullptr, "null count");
    *count = reset ? ct2::g_launches.exchange(0) : ct2::g_launches.load();
    return CT2_OK;
}

// --- view_proj3D ---

int ct2_dev_view_proj3D_sinoproj_linear(float* sinomat, VIEW_ARGS_DECL, const float* smat,
                                        GRID_ARGS_DECL, void* stream)
{
    return dev_view_project(MODE_LINEAR, false, sinomat, VIEW_ARGS, smat, GRID_ARGS, ST(stream));
}
// Host calls of the TMA-staged projector: CT2_ETIMEOUT when one of its
// bounded waits ran out during the call (counted on the device).  The
// outputs are still complete -- a chunk whose copy did not arrive is read
// from global memory, the same sum bit for bit -- but a copy that does not
// complete in time marks a device in trouble.  Calls that overlap on the
// device share the count.
extern "C++" {
template <class F>
inline int timeout_checked(F&& call)
{
    int before = 0, after = 0;
    if (wait_timeouts(&before, 0) != CT2_OK) {
        // no usable device: the call itself reports that (after checking
        // its arguments)
        clear_error();
        return call();
    }
    int rc = call();
    if (rc) return rc;
    if ((rc = wait_timeouts(&after, 0))) return rc;
    if (after != before)
        return set_error(CT2_ETIMEOUT,
                         "%d bounded device wait(s) ran out during the call (outputs complete, "
                         "read from global memory)",
                         after - before);
    return CT2_OK;
}
}  // extern "C++"

int ct2_view_proj3D_sinoproj_linear(float* sinomat, VIEW_ARGS_DECL, const float* smat,
                                    GRID_ARGS_DECL)
{
    return timeout_checked(
        [&] { return host_view_project(MODE_LINEAR, false, sinomat, VIEW_ARGS, smat, GRID_ARGS); });
}
int ct2_dev_view_proj3D_sinoproj_nearest(float* sinomat, VIEW_ARGS_DECL, const float* smat,
                                         GRID_ARGS_DECL, void* stream)
{
    return dev_view_project(MODE_NEAREST_LE, false, sinomat, VIEW_ARGS, smat, GRID_ARGS,
                            ST(stream));
}
int ct2_view_proj3D_sinoproj_nearest(float* sinomat, VIEW_ARGS_DECL, const float* smat,
                                     GRID_ARGS_DECL)
{
    return host_view_project(MODE_NEAREST_LE, false, sinomat, VIEW_ARGS, smat, GRID_ARGS);
}
int ct2_dev_view_proj3D_sinobackproject_linear(const float* sinomat, VIEW_ARGS_DECL, float* smat,
                                               GRID_ARGS_DECL, void* stream)
{
    return dev_view_backproject(MODE_LINEAR, false, sinomat, VIEW_ARGS, smat, GRID_ARGS,
                                ST(stream));
}
int ct2_view_proj3D_sinobackproject_linear(const float* sinomat, VIEW_ARGS_DECL, float* smat,
                                           GRID_ARGS_DECL)
{
    return host_view_backproject(MODE_LINEAR, false, sinomat, VIEW_ARGS, smat, GRID_ARGS);
}
int ct2_dev_view_proj3D_sinobackproject_nearest(const float* sinomat, VIEW_ARGS_DECL, float* smat,
                                                GRID_ARGS_DECL, void* stream)
{
    return dev_view_backproject(MODE_NEAREST_LE, false, sinomat, VIEW_ARGS, smat, GRID_ARGS,
                                ST(stream));
}
int ct2_view_proj3D_sinobackproject_nearest(const float* sinomat, VIEW_ARGS_DECL, float* smat,
                                            GRID_ARGS_DECL)
{
    return host_view_backproject(MODE_NEAREST_LE, false, sinomat, VIEW_ARGS, smat, GRID_ARGS);
}
int ct2_dev_view_proj3D_emratio_linear(float* ratio, const float* y, VIEW_ARGS_DECL,
                                       const float* smat, GRID_ARGS_DECL, void* stream)
{
    clear_error();
    int rc = check_view(ns, nu, nv, du, dv, u0, v0);
    if (rc) return rc;
    if ((rc = check_grid(GRID_ARGS))) return rc;
    const long long nrays = (long long)ns * nu * nv;
    if (nrays == 0) return CT2_OK;
    CT2_REQUIRE(ratio && y && frame_vectors, "null ratio/y/frame_vectors");
    // an empty volume is never read: every ray sum is 0, clamped to 1
    if ((long long)nx * ny * nz > 0) CT2_REQUIRE(smat != nullptr, "null smat");
    ProjectArgs p{};
    p.G = make_grid(GRID_ARGS);
    p.vol = smat;
    p.geom = frame_vectors;
    p.ind = indsino;
    p.ns = ns; p.nu = nu; p.nv = nv;
    p.du = du; p.dv = dv; p.u0 = u0; p.v0 = v0;
    p.out = ratio;
    p.y = y;
    p.em_small = 0.00001f;
    return project(p, MODE_LINEAR, false, false, true, ST(stream));
}

int ct2_dev_view_proj3D_emstep_linear(const float* sinomat, VIEW_ARGS_DECL, float* smat,
                                      GRID_ARGS_DECL, void* stream)
{
    return dev_view_em(MODE_LINEAR, false, 0.00001f, sinomat, VIEW_ARGS, smat, GRID_ARGS,
                       ST(stream));
}
int ct2_view_proj3D_emstep_linear(const float* sinomat, VIEW_ARGS_DECL, float* smat,
                                  GRID_ARGS_DECL)
{
    return timeout_checked([&] {
        return host_view_em(MODE_LINEAR, false, 0.00001f, sinomat, VIEW_ARGS, smat, GRID_ARGS);
    });
}
int ct2_dev_view_proj3D_emstep_nearest(const float* sinomat, VIEW_ARGS_DECL, float* smat,
                                       GRID_ARGS_DECL, void* stream)
{
    return dev_view_em(MODE_NEAREST_LE, false, 0.00000001f, sinomat, VIEW_ARGS, smat, GRID_ARGS,
                       ST(stream));
}
int ct2_view_proj3D_emstep_nearest(const float* sinomat, VIEW_ARGS_DECL, float* smat,
                                   GRID_ARGS_DECL)
{
    return host_view_em(MODE_NEAREST_LE, false, 0.00000001f, sinomat, VIEW_ARGS, smat, GRID_ARGS);
}

// --- view_proj3D_tomo ---

int ct2_dev_view_proj3D_tomo_sinoprojz(float* sinomat, VIEW_ARGS_DECL, const float* smat,
                                       GRID_ARGS_DECL, void* stream)
{
    return dev_view_project(MODE_LINEAR, true, sinomat, VIEW_ARGS, smat, GRID_ARGS, ST(stream));
}
int ct2_view_proj3D_tomo_sinoprojz(float* sinomat, VIEW_ARGS_DECL, const float* smat,
                                   GRID_ARGS_DECL)
{
    return host_view_project(MODE_LINEAR, true, sinomat, VIEW_ARGS, smat, GRID_ARGS);
}
int ct2_dev_view_proj3D_tomo_emstep_linearz(const float* sinomat, VIEW_ARGS_DECL, float* smat,
                                            GRID_ARGS_DECL, void* stream)
{
    return dev_view_em(MODE_LINEAR, true, 0.00001f, sinomat, VIEW_ARGS, smat, GRID_ARGS,
                       ST(stream));
}
int ct2_view_proj3D_tomo_emstep_linearz(const float* sinomat, VIEW_ARGS_DECL, float* smat,
                                        GRID_ARGS_DECL)
{
    return host_view_em(MODE_LINEAR, true, 0.00001f, sinomat, VIEW_ARGS, smat, GRID_ARGS);
}

}  // extern "C"

// =====================================================================
// ray_proj3D
// =====================================================================

static int check_list(int nr)
{
    CT2_REQUIRE(nr >= 0, "nr must be >= 0 (got %d)", nr);
    return CT2_OK;
}

static int dev_list_project(int mode, float* sinomat, const int32_t* indsino, const float* rv,
                            int nr, const float* smat, GRID_ARGS_DECL, cudaStream_t st)
{
    clear_error();
    int rc = check_list(nr);
    if (rc) return rc;
    if ((rc = check_grid(GRID_ARGS))) return rc;
    if (nr == 0) return CT2_OK;
    CT2_REQUIRE(sinomat && rv, "null sinomat/ray_vectors");
    if ((long long)nx * ny * nz == 0) {
        CT2_CUDA(cudaMemsetAsync(sinomat, 0, sizeof(float) * nr, st));
        return CT2_OK;
    }
    CT2_REQUIRE(smat != nullptr, "null smat");
    ProjectArgs a{};
    a.G = make_grid(GRID_ARGS);
    a.vol = smat;
    a.geom = rv;
    a.ind = indsino;
    a.nrays = nr;
    a.out = sinomat;
    return project(a, mode, true, false, false, st);
}

static int dev_list_backproject(int mode, const float* sinomat, const int32_t* indsino,
                                const float* rv, int nr, float* smat, GRID_ARGS_DECL,
                                cudaStream_t st)
{
    clear_error();
    int rc = check_list(nr);
    if (rc) return rc;
    if ((rc = check_grid(GRID_ARGS))) return rc;
    const long long nvox = (long long)nx * ny * nz;
    if (nvox == 0) return CT2_OK;
    CT2_REQUIRE(smat != nullptr, "null smat");
    CT2_CUDA(cudaMemsetAsync(smat, 0, sizeof(float) * nvox, st));
    if (nr == 0) return CT2_OK;
    CT2_REQUIRE(sinomat && rv, "null sinomat/ray_vectors");
    BackprojectArgs a{};
    a.G = make_grid(GRID_ARGS);
    a.sino = sinomat;
    a.ind = indsino;
    a.geom = rv;
    a.nrays = nr;
    a.out = smat;
    return backproject(a, mode, true, false, st);
}

static int dev_list_em(int mode, float small, const float* sinomat, const int32_t* indsino,
                       const float* rv, int nr, float* smat, GRID_ARGS_DECL, cudaStream_t st)
{
    clear_error();
    int rc = check_list(nr);
    if (rc) return rc;
    if ((rc = check_grid(GRID_ARGS))) return rc;
    const long long nvox = (long long)nx * ny * nz;
    if (nvox == 0) return CT2_OK;
    CT2_REQUIRE(smat != nullptr, "null smat");
    Scratch S(st);
    float *ratio = nullptr, *ws = nullptr, *ones = nullptr;
    if ((rc = S.get((void**)&ws, sizeof(float) * nvox, true))) return rc;
    if ((rc = S.get((void**)&ones, sizeof(float) * nvox, true))) return rc;
    if (nr > 0) {
        CT2_REQUIRE(sinomat && rv, "null sinomat/ray_vectors");
        if ((rc = S.get((void**)&ratio, sizeof(float) * nr, false))) return rc;
        const Grid G = make_grid(GRID_ARGS);
        ProjectArgs p{};
        p.G = G;
        p.vol = smat;
        p.geom = rv;
        p.ind = indsino;
        p.nrays = nr;
        p.out = ratio;
        p.y = sinomat;
        p.em_small = small;
        if ((rc = project(p, mode, true, false, true, st))) return rc;
        BackprojectArgs b{};
        b.G = G;
        b.sino = ratio;
        b.ind = indsino;
        b.geom = rv;
        b.nrays = nr;
        b.out = ws;
        b.out_ones = ones;
        if ((rc = backproject(b, mode, true, false, st))) return rc;
    }
    return em_update(smat, ws, ones, nvox, small, st);
}

static int host_list_project(int mode, float* sinomat, const int32_t* indsino, const float* rv,
                             int nr, const float* smat, GRID_ARGS_DECL)
{
    clear_error();
    int rc = check_list(nr);
    if (rc) return rc;
    if ((rc = check_grid(GRID_ARGS))) return rc;
    const size_t nvox = (size_t)nx * ny * nz;
    HostCall H;
    int32_t* d_ind = nullptr;
    float *d_rv = nullptr, *d_vol = nullptr, *d_out = nullptr;
    if ((rc = H.upload((void**)&d_ind, indsino, (size_t)nr * sizeof(int32_t)))) return rc;
    if ((rc = H.upload((void**)&d_rv, rv, (size_t)nr * 6 * sizeof(float)))) return rc;
    if ((rc = H.upload((void**)&d_vol, smat, nvox * sizeof(float)))) return rc;
    if ((rc = H.alloc((void**)&d_out, (size_t)nr * sizeof(float), false))) return rc;
    if ((rc = dev_list_project(mode, d_out, d_ind, d_rv, nr, d_vol, GRID_ARGS, H.st))) return rc;
    if ((rc = H.download(sinomat, d_out, (size_t)nr * sizeof(float)))) return rc;
    return H.finish();
}

extern "C" {

int ct2_dev_ray_proj3D_sinoproj_linear(float* sinomat, const int32_t* indsino,
                                       const float* ray_vectors, int nr, const float* smat,
                                       GRID_ARGS_DECL, void* stream)
{
    return dev_list_project(MODE_LINEAR, sinomat, indsino, ray_vectors, nr, smat, GRID_ARGS,
                            ST(stream));
}
int ct2_ray_proj3D_sinoproj_linear(float* sinomat, const int32_t* indsino,
                                   const float* ray_vectors, int nr, const float* smat,
                                   GRID_ARGS_DECL)
{
    return host_list_project(MODE_LINEAR, sinomat, indsino, ray_vectors, nr, smat, GRID_ARGS);
}
int ct2_dev_ray_proj3D_sinoproj_nearest(float* sinomat, const int32_t* indsino,
                                        const float* ray_vectors, int nr, const float* smat,
                                        GRID_ARGS_DECL, void* stream)
{
    return dev_list_project(MODE_NEAREST_LE, sinomat, indsino, ray_vectors, nr, smat, GRID_ARGS,
                            ST(stream));
}
int ct2_ray_proj3D_sinoproj_nearest(float* sinomat, const int32_t* indsino,
                                    const float* ray_vectors, int nr, const float* smat,
                                    GRID_ARGS_DECL)
{
    return host_list_project(MODE_NEAREST_LE, sinomat, indsino, ray_vectors, nr, smat, GRID_ARGS);
}
int ct2_dev_ray_proj3D_sinobackproject_nearest(const float* sinomat, const int32_t* indsino,
                                               const float* ray_vectors, int nr, float* smat,
                                               GRID_ARGS_DECL, void* stream)
{
    return dev_list_backproject(MODE_NEAREST_LT, sinomat, indsino, ray_vectors, nr, smat,
                                GRID_ARGS, ST(stream));
}
int ct2_ray_proj3D_sinobackproject_nearest(const float* sinomat, const int32_t* indsino,
                                           const float* ray_vectors, int nr, float* smat,
                                           GRID_ARGS_DECL)
{
    clear_error();
    int rc = check_list(nr);
    if (rc) return rc;
    if ((rc = check_grid(GRID_ARGS))) return rc;
    const size_t nvox = (size_t)nx * ny * nz;
    HostCall H;
    int32_t* d_ind = nullptr;
    float *d_rv = nullptr, *d_sino = nullptr, *d_out = nullptr;
    if ((rc = H.upload((void**)&d_ind, indsino, (size_t)nr * sizeof(int32_t)))) return rc;
    if ((rc = H.upload((void**)&d_rv, ray_vectors, (size_t)nr * 6 * sizeof(float)))) return rc;
    if ((rc = H.upload((void**)&d_sino, sinomat, (size_t)nr * sizeof(float)))) return rc;
    if ((rc = H.alloc((void**)&d_out, nvox * sizeof(float), false))) return rc;
    if ((rc = dev_list_backproject(MODE_NEAREST_LT, d_sino, d_ind, d_rv, nr, d_out, GRID_ARGS,
                                   H.st)))
        return rc;
    if ((rc = H.download(smat, d_out, nvox * sizeof(float)))) return rc;
    return H.finish();
}
int ct2_dev_ray_proj3D_emstep_nearest(const float* sinomat, const int32_t* indsino,
                                      const float* ray_vectors, int nr, float* smat,
                                      GRID_ARGS_DECL, void* stream)
{
    return dev_list_em(MODE_NEAREST_LT, 0.00000001f, sinomat, indsino, ray_vectors, nr, smat,
                       GRID_ARGS, ST(stream));
}
int ct2_ray_proj3D_emstep_nearest(const float* sinomat, const int32_t* indsino,
                                  const float* ray_vectors, int nr, float* smat, GRID_ARGS_DECL)
{
    clear_error();
    int rc = check_list(nr);
    if (rc) return rc;
    if ((rc = check_grid(GRID_ARGS))) return rc;
    const size_t nvox = (size_t)nx * ny * nz;
    HostCall H;
    int32_t* d_ind = nullptr;
    float *d_rv = nullptr, *d_sino = nullptr, *d_vol = nullptr;
    if ((rc = H.upload((void**)&d_ind, indsino, (size_t)nr * sizeof(int32_t)))) return rc;
    if ((rc = H.upload((void**)&d_rv, ray_vectors, (size_t)nr * 6 * sizeof(float)))) return rc;
    if ((rc = H.upload((void**)&d_sino, sinomat, (size_t)nr * sizeof(float)))) return rc;
    if ((rc = H.upload((void**)&d_vol, smat, nvox * sizeof(float)))) return rc;
    if ((rc = dev_list_em(MODE_NEAREST_LT, 0.00000001f, d_sino, d_ind, d_rv, nr, d_vol, GRID_ARGS,
                          H.st)))
        return rc;
    if ((rc = H.download(smat, d_vol, nvox * sizeof(float)))) return rc;
    return H.finish();
}

}  // extern "C"
