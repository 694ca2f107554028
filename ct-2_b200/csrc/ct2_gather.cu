// Atomic-free, voxel-driven matched backprojector (linear mode, view geometry).
//
// Reference: view_proj3D.sinobackproject_linear (emil_code/view_proj3D.f:
// 1096-1370) and the A^T 1 accumulation of emstep_linear (:2801-2827), which
// scatter datum * weight along each ray.  Here every voxel gathers the sum of
// y * w over the (ray, slice) samples that reach it, so each voxel is written
// once per view block by the one thread that owns it: no atomics, and the
// summation order is fixed (results are bit-reproducible run to run).
//
// The sample set and weights are the projector's (ct2_project.cu): for a ray
// with driving axis p, slice t, in-plane models fq(t) = fma(bq, t, aq) and
// fr(t) = fma(br, t, ar), the reference's exact valid interval [t0, t1], and
// cells clamp(floor(f), 0, n-2).  A voxel (q = j, r = k) on slice t receives
// y * tvl * W(fq, j) * W(fr, k) with W the weight of that voxel in the linear
// interpolation.  In q this is evaluated exactly as the projector clamps; in
// r (the z axis) as the hat max(0, 1 - |fr - k|), which is the same weight
// wherever the projector's cell is not clamped -- the clamp acts only where
// the fast model sits within ~1e-4 voxel outside the volume while the
// reference arithmetic is still inside, and there the hat drops a weight of
// that size.
//
// Which views: those whose detector v axis has no x or y component
// (frame_vectors[12] == frame_vectors[13] == 0 exactly: the circular cone
// beam family).  There the x and y bin coordinates of a detector column do
// not depend on v, so all x- or y-driven rays of a column share the driving
// axis and the q model bit for bit; a voxel column is reached by the two or
// three detector columns whose fq passes within one voxel of it, and along z
// by the rays whose fr does.  Rays of other views, and z-driven (steep) rays,
// go through the L2-reduction scatter afterwards (k_bpg_residual).
//
// The precision form's backprojector (ct2_dev_prec_backproject) runs the
// same gather over its own ray table: FP64 per-ray setup, the sample
// interval where the FP32 model lies inside the volume (no clamp, so the
// hat is the bilinear weight exactly), FP16 or FP32 data.
//
// Work per view block (as many views as fit the ray-table budget):
//  * k_bpg_table: per ray {ar, br, y * tvl, t0 | (t1 - t0) << 16} in a
//    (view, v, u) layout (u fastest), per detector column {aq, bq, pdiff,
//    axis}, per view the geometry the windows need; rays left to the scatter
//    are listed.
//  * k_bpg: one thread per 4 (x) x 1 (y) x 2 (z) voxels, 32 lanes along y,
//    8 warps along x; per view it finds, from the per-view geometry, the
//    detector columns whose rays can reach its voxels and, per column, the
//    window of v whose fr can; the warp copies the tile of rays its lanes
//    need (columns x rows) into shared memory with coalesced loads, and each
//    lane accumulates its candidates in registers; at the end it
//    adds its sums to the volume (one read and one write per voxel and view
//    block: the volume holds what the caller zero-filled, or the views of
//    earlier blocks and calls -- the host entry points backproject their
//    views in pipelined blocks into one volume).
#include <cuda_fp16.h>

#include <climits>
#include <cstdint>

#include "ct2_capi_util.h"
#include "ct2_common.cuh"
#include "ct2_kernels.h"
#include "ct2_pray.cuh"
#include "ct2_precision.h"
#include "ct2_scatter.cuh"

namespace ct2 {

namespace {

constexpr unsigned kMetaEmpty = 0x0000FFFFu;     // t0 = 65535, len = 0: never valid
constexpr unsigned kMetaResidual = 0xFFFFFFFEu;  // left to the scatter
constexpr float kWinEps = 0.02f;                 // window margin, voxels
constexpr size_t kTableBudget = 512ull << 20;    // bytes of ray table per view block

// Per-view geometry read by the gather (warp-uniform loads).
struct GView {
    float Sx, Sy, Sz;
    float ax, bx, cx, dx;  // x-driven rays: (By - Sy)(u) = ax + bx*u_pos, (Bx - Sx)(u) = cx + dx*u_pos
    float ay, by, cy, dy;  // y-driven rays: (Bx - Sx)(u) = ay + by*u_pos, (By - Sy)(u) = cy + dy*u_pos
    float zq0, euz, ez;    // (Bz - Sz)(u, v) = zq0 + euz*u_pos + ez*v_pos
    int flags;             // bit 0: x-driven columns, bit 1: y-driven columns, bit 2: eligible
};

struct GCol {
    float aq, bq, pdiff;
    int axis;  // 0 x-driven, 1 y-driven, 3 not gathered
};

// What a gather pass reads: the data, indicator, geometry and grid of one
// backprojection, with the data's storage type (ST_F32 or ST_F16).
struct GatherSrc {
    Grid G;
    const void* sino;
    int sino_type;
    const int* ind;
    const float* geom;
    int ns, nu, nv;
    float du, dv, u0, v0;
};

template <typename ST>
__device__ __forceinline__ float ld_datum(const void* p, long long r)
{
    if constexpr (sizeof(ST) == 4)
        return __ldg((const float*)p + r);
    else
        return __half2float(((const __half*)p)[r]);
}

// KIND 0: the reference's REAL*4 ray (ray_setup + exact_interval, cells
// clamped); KIND 1: the precision form's FP64 ray (pray_view, which reads the
// view's frame vector from global memory).  f: the view's frame vector in
// registers.  Returns the ray with its valid slice interval [R.t0, R.t1].
template <int KIND>
__device__ __forceinline__ Ray gather_ray(const GatherSrc& a, const float* f, int view, int u,
                                          int v, int force)
{
    if constexpr (KIND == 0) {
        const float S[3] = {f[0], f[1], f[2]};
        float B[3];
        view_bin(f, u, v, a.du, a.dv, a.u0, a.v0, B);
        Ray R = ray_setup(a.G, S, B, force, MODE_LINEAR);
        if (force < 0) {
            int s0, s1;
            exact_interval(R, R.np, &s0, &s1);
        }
        return R;
    } else {
        return pray_view(a.G, a.geom + 18 * view, u, v, a.du, a.dv, a.u0, a.v0, force);
    }
}

// Driving axis (0 or 1) of the x/y-driven rays of detector column u and the
// column's (Bp - Sp), from the bin at v = 0 (the x and y bin coordinates do
// not depend on v in the views the gather takes).
template <int KIND>
__device__ __forceinline__ int column_axis(const GatherSrc& a, const float* f, int u,
                                           float* pdiff)
{
    if constexpr (KIND == 0) {
        float B[3];
        view_bin(f, u, 0, a.du, a.dv, a.u0, a.v0, B);
        const float ad0 = __fdiv_rn(fabsf(__fsub_rn(B[0], f[0])), a.G.d[0]);
        const float ad1 = __fdiv_rn(fabsf(__fsub_rn(B[1], f[1])), a.G.d[1]);
        const int axis = (ad0 > ad1) ? 0 : 1;
        *pdiff = __fsub_rn(B[axis], f[axis]);
        return axis;
    } else {
        const double uu = (double)a.u0 + ((double)u + 0.5) * (double)a.du;
        const double vv = (double)a.v0 + 0.5 * (double)a.dv;
        double d[2];
        for (int i = 0; i < 2; i++)
            d[i] = ((double)f[6 + i] + (double)f[9 + i] * uu + (double)f[12 + i] * vv) -
                   (double)f[i];
        const int axis = (fabs(d[0]) / (double)a.G.d[0] > fabs(d[1]) / (double)a.G.d[1]) ? 0 : 1;
        *pdiff = (float)d[axis];
        return axis;
    }
}

// Window arithmetic only (the windows carry a margin): fast division.
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

__device__ __forceinline__ float hat(float d) { return fmaxf(0.f, 1.f - fabsf(d)); }

// Weight of cell j in the projector's clamped linear interpolation at f.
__device__ __forceinline__ float qweight(float f, int j, int n)
{
    const float c = fminf(fmaxf(floorf(f), 0.f), (float)(n - 2));
    const float w2 = __fsub_rn(f, c);
    const float fj = (float)j;
    return fj == c ? __fsub_rn(1.0f, w2) : (fj == c + 1.0f ? w2 : 0.f);
}

__device__ __forceinline__ bool valid_at(unsigned m, int t)
{
    return (unsigned)(t - (int)(m & 0xFFFFu)) <= (m >> 16);
}

// Detector index window [lo, hi] (clamped to [0, n-1]): the pixels whose
// centres lie between the continuous positions, the whole row if a position
// is not finite.  The positions come from windows widened by kWinEps voxels,
// more than the window arithmetic's error (~3e-3 voxel), so every pixel whose
// ray reaches the voxels is inside.
__device__ __forceinline__ void index_window(float a, float b, float c, float d, float o,
                                             float inv_step, int n, int* lo, int* hi)
{
    const float mn = fminf(fminf(a, b), fminf(c, d)), mx = fmaxf(fmaxf(a, b), fmaxf(c, d));
    if (!(isfinite(mn) && isfinite(mx))) {
        *lo = 0;
        *hi = n - 1;
        return;
    }
    const float fl = (mn - o) * inv_step - 0.5f, fh = (mx - o) * inv_step - 0.5f;
    *lo = max(0, (int)fmaxf(ceilf(fl), -1.0f));
    *hi = min(n - 1, (int)fminf(floorf(fh), (float)n));
}

// ---------------------------------------------------------------------------
// Table: one thread per ray, a CTA per 32 (u) x 32 (v) tile of one view.
// ---------------------------------------------------------------------------
template <int KIND, typename ST, bool ONES>
__global__ void __launch_bounds__(256) k_bpg_table(GatherSrc a, int view0, float4* rec,
                                                   GCol* cols, GView* views, int* residual,
                                                   int* nresidual)
{
    __shared__ float ys[32][33];
    const int tiles_u = (a.nu + 31) >> 5;
    const int tu = blockIdx.x % tiles_u, tv = blockIdx.x / tiles_u;
    const int lv = blockIdx.y, view = view0 + lv;
    const int ub = tu * 32, vb = tv * 32;
    // the tile's data, read along v (coalesced), held transposed
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int u = ub + k, v = vb + threadIdx.x;
        float y = 0.f;
        if (u < a.nu && v < a.nv) {
            const long long r = ((long long)view * a.nu + u) * a.nv + v;
            const bool on = a.ind == nullptr || a.ind[r] == 1;
            y = on ? (ONES ? 1.0f : ld_datum<ST>(a.sino, r)) : 0.f;
        }
        ys[k][threadIdx.x] = y;
    }
    __syncthreads();
    float f[18];
#pragma unroll
    for (int i = 0; i < 18; i++) f[i] = __ldg(a.geom + 18 * view + i);
    const bool eligible = f[12] == 0.f && f[13] == 0.f;
    const int u = ub + threadIdx.x;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int v = vb + k;
        if (u >= a.nu || v >= a.nv) continue;
        const float y = ys[threadIdx.x][k];
        float c = 0.f;
        unsigned meta = kMetaEmpty;
        float ar = 0.f, br = 0.f;
        if (y != 0.f) {
            const Ray R = gather_ray<KIND>(a, f, view, u, v, -1);
            ar = R.ar;
            br = R.br;
            if (!eligible || R.p == 2) {
                meta = kMetaResidual;
                const int slot = atomicAdd(nresidual, 1);
                residual[slot] = (lv * a.nu + u) * a.nv + v;
            } else if (R.t0 <= R.t1) {
                c = y * R.tvl;
                meta = (unsigned)R.t0 | ((unsigned)(R.t1 - R.t0) << 16);
            }
        }
        rec[((long long)lv * a.nv + v) * a.nu + u] = make_float4(ar, br, c, __uint_as_float(meta));
    }
    // per detector column (first v tile): driving axis of its x/y-driven rays and their q model
    if (tv == 0 && threadIdx.y == 0 && u < a.nu) {
        GCol C;
        C.axis = 3;
        C.aq = C.bq = C.pdiff = 0.f;
        if (eligible) {
            const int axis = column_axis<KIND>(a, f, u, &C.pdiff);
            const Ray R = gather_ray<KIND>(a, f, view, u, 0, axis);
            C.axis = axis;
            C.aq = R.aq;
            C.bq = R.bq;
            atomicOr(&views[lv].flags, 1 << axis);
        }
        cols[(long long)lv * a.nu + u] = C;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
        GView& P = views[lv];
        P.Sx = f[0];
        P.Sy = f[1];
        P.Sz = f[2];
        P.ax = f[7] - f[1];
        P.bx = f[10];
        P.cx = f[6] - f[0];
        P.dx = f[9];
        P.ay = f[6] - f[0];
        P.by = f[9];
        P.cy = f[7] - f[1];
        P.dy = f[10];
        P.zq0 = f[8] - f[2];
        P.euz = f[11];
        P.ez = f[14];
        if (eligible) atomicOr(&P.flags, 4);
    }
}

// ---------------------------------------------------------------------------
// Gather.
// ---------------------------------------------------------------------------
struct GatherArgs {
    Grid G;
    int nu, nv;
    float du, dv, u0, v0;
    int nviews;
    const float4* rec;
    const GCol* cols;
    const GView* views;
    float* out;
};

// Rays staged per warp and view: a tile of detector columns x rows copied
// from the ray table with coalesced loads (all in flight at once), then read
// by the lanes from shared memory.  A tile larger than this (a window wider
// than the configurations ever give) is read from global memory instead.
constexpr int kTileRays = 320;
constexpr int kTileCols = 64;
constexpr int kPlanes = 4;  // x slices per thread
constexpr unsigned kFull = 0xffffffffu;
struct TileSmem {
    float4 ray[kTileRays];
    GCol col[kTileCols];
    int2 win[kTileCols];  // x-driven role: the column's row window
};
constexpr size_t kGatherSmem = 8 * sizeof(TileSmem);

// Row window of column u: rows whose z lies in [zlo, zhi] on the slices at
// distances lA and lB from the source (x- or y-driven per pd's role).
__device__ __forceinline__ void row_window(const GatherArgs& a, const GView& P, float pd, float up,
                                           float lA, float lB, float zlo, float zhi, float iez,
                                           float inv_dv, int* vlo, int* vhi)
{
    const float zq = P.zq0 + P.euz * up;
    const float rA = fdiv(pd, lA), rB = fdiv(pd, lB);  // reciprocal ratios
    index_window(((zlo - P.Sz) * rA - zq) * iez, ((zhi - P.Sz) * rA - zq) * iez,
                 ((zlo - P.Sz) * rB - zq) * iez, ((zhi - P.Sz) * rB - zq) * iez, a.v0, inv_dv,
                 a.nv, vlo, vhi);
}

// Copies the warp's tile [U0, U1] x [V0, V1] of view lv into shared memory
// (uniform arguments).  Returns whether it fits.
__device__ __forceinline__ bool stage_rays(const GatherArgs& a, int lv, int U0, int U1, int V0,
                                           int V1, TileSmem& T, int lane)
{
    const int nu_w = U1 - U0 + 1, nv_w = V1 - V0 + 1;
    if (U1 < U0 || V1 < V0 || nu_w * nv_w > kTileRays) return false;
    const float4* base = a.rec + ((long long)lv * a.nv + V0) * a.nu + U0;
    for (int rv = 0; rv < nv_w; rv++)
        for (int ru = lane; ru < nu_w; ru += 32)
            T.ray[rv * nu_w + ru] = __ldg(base + (long long)rv * a.nu + ru);
    __syncwarp();
    return true;
}

__global__ void __launch_bounds__(256, 3) k_bpg(GatherArgs a)
{
    extern __shared__ float4 gsm[];
    TileSmem& T = reinterpret_cast<TileSmem*>(gsm)[threadIdx.y];
    const Grid& G = a.G;
    const int nx = G.n[0], ny = G.n[1], nz = G.n[2];
    const int tiles_j = (ny + 31) >> 5;
    const int tj = blockIdx.x % tiles_j, ti = blockIdx.x / tiles_j;
    const int lane = threadIdx.x;
    const int j = tj * 32 + lane;
    const int i0 = (ti * 8 + threadIdx.y) * kPlanes;
    const int k = blockIdx.y * 2;
    // lanes outside the volume stay to load their share of the tiles
    const bool live = j < ny && i0 < nx;
    if (!__any_sync(kFull, live)) return;
    const int jw0 = tj * 32, jw1 = min(tj * 32 + 31, ny - 1);  // the warp's y slices
    const float fi0 = (float)i0, fj = (float)j;
    const float fk = (float)k, fk1 = (float)(k + 1);
    const float inv_du = 1.0f / a.du, inv_dv = 1.0f / a.dv;
    // plane positions and windows that do not depend on the view
    const float x0c = G.o[0] + G.d[0] * (fi0 + 0.5f);  // centre of slice i0
    const float x3c = x0c + G.d[0] * (float)(kPlanes - 1);
    const float yP = G.o[1] + G.d[1] * (fj + 0.5f);
    const float yw0 = G.o[1] + G.d[1] * ((float)jw0 + 0.5f);
    const float yw1 = G.o[1] + G.d[1] * ((float)jw1 + 0.5f);
    const float ylo = G.o[1] + G.d[1] * (fj - 0.5f - kWinEps);
    const float yhi = G.o[1] + G.d[1] * (fj + 1.5f + kWinEps);
    const float xlo = G.o[0] + G.d[0] * (fi0 - 0.5f - kWinEps);
    const float xhi = G.o[0] + G.d[0] * (fi0 + (float)kPlanes + 0.5f + kWinEps);
    const float zlo = G.o[2] + G.d[2] * (fk - 0.5f - kWinEps);
    const float zhi = G.o[2] + G.d[2] * (fk + 2.5f + kWinEps);
    float acc[kPlanes][2];  // voxel (i0 + p, j, k + z)
#pragma unroll
    for (int p = 0; p < kPlanes; p++) acc[p][0] = acc[p][1] = 0.f;
    for (int lv = 0; lv < a.nviews; lv++) {
        const GView P = a.views[lv];
        if (!(P.flags & 4)) continue;
        const float4* rv = a.rec + (long long)lv * a.nv * a.nu;
        const GCol* cv = a.cols + (long long)lv * a.nu;
        const float iez = fdiv(1.0f, P.ez);
        if (P.flags & 1) {
            // ---- x-driven rays: slices i0 .. i0+3, voxel row j in y ----
            const float lA = x0c - P.Sx, lB = x3c - P.Sx;
            int ulo = 1, uhi = 0;
            if (live) {
                const float sAl = fdiv(ylo - P.Sy, lA), sAh = fdiv(yhi - P.Sy, lA);
                const float sBl = fdiv(ylo - P.Sy, lB), sBh = fdiv(yhi - P.Sy, lB);
                index_window(fdiv(P.ax - sAl * P.cx, sAl * P.dx - P.bx),
                             fdiv(P.ax - sAh * P.cx, sAh * P.dx - P.bx),
                             fdiv(P.ax - sBl * P.cx, sBl * P.dx - P.bx),
                             fdiv(P.ax - sBh * P.cx, sBh * P.dx - P.bx), a.u0, inv_du, a.nu,
                             &ulo, &uhi);
            }
            const int U0 = __reduce_min_sync(kFull, ulo <= uhi ? ulo : INT_MAX);
            const int U1 = __reduce_max_sync(kFull, ulo <= uhi ? uhi : INT_MIN);
            // every lane shares the slices and z pair, so a column's row
            // window is the same for all: one lane computes it per column
            const int nu_w = U1 - U0 + 1;
            if (U0 <= U1 && nu_w <= kTileCols) {
                int wlo = INT_MAX, whi = INT_MIN;
                for (int c = lane; c < nu_w; c += 32) {
                    const GCol C = cv[U0 + c];
                    int vlo = 1, vhi = 0;
                    if (C.axis == 0)
                        row_window(a, P, C.pdiff, a.u0 + ((float)(U0 + c) + 0.5f) * a.du, lA, lB,
                                   zlo, zhi, iez, inv_dv, &vlo, &vhi);
                    T.col[c] = C;
                    T.win[c] = make_int2(vlo, vhi);
                    if (vlo <= vhi) {
                        wlo = min(wlo, vlo);
                        whi = max(whi, vhi);
                    }
                }
                const int V0 = __reduce_min_sync(kFull, wlo), V1 = __reduce_max_sync(kFull, whi);
                __syncwarp();
                const bool staged = V0 <= V1 && stage_rays(a, lv, U0, U1, V0, V1, T, lane);
                for (int u = ulo; u <= uhi; u++) {
                    const GCol C = T.col[u - U0];
                    const int2 w = T.win[u - U0];
                    if (C.axis != 0 || w.x > w.y) continue;
                    float q[kPlanes];
                    bool any = false;
#pragma unroll
                    for (int p = 0; p < kPlanes; p++) {
                        q[p] = (i0 + p < nx) ? qweight(__fmaf_rn(C.bq, fi0 + (float)p, C.aq), j, ny)
                                             : 0.f;
                        any |= q[p] != 0.f;
                    }
                    if (!any) continue;
                    const float4* tp = T.ray + (u - U0);
                    const float4* gp = rv + u;
                    for (int v = w.x; v <= w.y; v++) {
                        const float4 r = staged ? tp[(v - V0) * nu_w] : __ldg(gp + (long long)v * a.nu);
                        const unsigned m = __float_as_uint(r.w);
                        const int t0 = (int)(m & 0xFFFFu);
                        const unsigned len = m >> 16;
#pragma unroll
                        for (int p = 0; p < kPlanes; p++) {
                            const float c = ((unsigned)(i0 + p - t0) <= len) ? r.z * q[p] : 0.f;
                            const float fr = __fmaf_rn(r.y, fi0 + (float)p, r.x);
                            acc[p][0] = __fmaf_rn(c, hat(fr - fk), acc[p][0]);
                            acc[p][1] = __fmaf_rn(c, hat(fr - fk1), acc[p][1]);
                        }
                    }
                }
                __syncwarp();  // every lane is done with the tile before the next one lands
            } else if (U0 <= U1) {
                // a tile wider than the buffer: columns and rays straight from the table
                for (int u = ulo; u <= uhi; u++) {
                    const GCol C = cv[u];
                    if (C.axis != 0) continue;
                    int vlo, vhi;
                    row_window(a, P, C.pdiff, a.u0 + ((float)u + 0.5f) * a.du, lA, lB, zlo, zhi,
                               iez, inv_dv, &vlo, &vhi);
                    float q[kPlanes];
#pragma unroll
                    for (int p = 0; p < kPlanes; p++)
                        q[p] = (i0 + p < nx) ? qweight(__fmaf_rn(C.bq, fi0 + (float)p, C.aq), j, ny)
                                             : 0.f;
                    for (int v = vlo; v <= vhi; v++) {
                        const float4 r = __ldg(rv + (long long)v * a.nu + u);
                        const unsigned m = __float_as_uint(r.w);
                        const int t0 = (int)(m & 0xFFFFu);
                        const unsigned len = m >> 16;
#pragma unroll
                        for (int p = 0; p < kPlanes; p++) {
                            const float c = ((unsigned)(i0 + p - t0) <= len) ? r.z * q[p] : 0.f;
                            const float fr = __fmaf_rn(r.y, fi0 + (float)p, r.x);
                            acc[p][0] = __fmaf_rn(c, hat(fr - fk), acc[p][0]);
                            acc[p][1] = __fmaf_rn(c, hat(fr - fk1), acc[p][1]);
                        }
                    }
                }
            }
        }
        if (P.flags & 2) {
            // ---- y-driven rays: slice j, voxel columns i0 .. i0+3 in x ----
            const float l = yP - P.Sy;
            int ulo = 1, uhi = 0;
            if (live) {
                const float sl = fdiv(xlo - P.Sx, l), sh = fdiv(xhi - P.Sx, l);
                const float ua = fdiv(P.ay - sl * P.cy, sl * P.dy - P.by);
                const float ub = fdiv(P.ay - sh * P.cy, sh * P.dy - P.by);
                index_window(ua, ub, ua, ub, a.u0, inv_du, a.nu, &ulo, &uhi);
            }
            const int U0 = __reduce_min_sync(kFull, ulo <= uhi ? ulo : INT_MAX);
            const int U1 = __reduce_max_sync(kFull, ulo <= uhi ? uhi : INT_MIN);
            if (U0 <= U1) {
                // the tile's rows: the row position is linear in the column,
                // in 1/(slice distance) and in z, so over the tile (columns
                // U0..U1, the warp's slices, the z window) its extremes lie at
                // the 8 corners; lanes 0-7 take one each, widened by a row for
                // the per-column bins
                float cmin = INFINITY, cmax = -INFINITY;
                if (lane < 8) {
                    const int u = (lane & 1) ? U1 : U0;
                    const float ls = ((lane & 2) ? yw1 : yw0) - P.Sy;
                    const float z = (lane & 4) ? zhi : zlo;
                    const float up = a.u0 + ((float)u + 0.5f) * a.du;
                    const float pd = P.cy + P.dy * up;
                    const float pos = ((z - P.Sz) * fdiv(pd, ls) - (P.zq0 + P.euz * up)) * iez;
                    cmin = cmax = (pos - a.v0) * inv_dv - 0.5f;
                }
                const bool fin = __all_sync(kFull, lane >= 8 || isfinite(cmin));
#pragma unroll
                for (int o = 1; o < 8; o <<= 1) {
                    cmin = fminf(cmin, __shfl_xor_sync(kFull, cmin, o));
                    cmax = fmaxf(cmax, __shfl_xor_sync(kFull, cmax, o));
                }
                cmin = __shfl_sync(kFull, cmin, 0);
                cmax = __shfl_sync(kFull, cmax, 0);
                int V0 = 0, V1 = -1;
                if (fin) {
                    V0 = max(0, (int)fmaxf(floorf(cmin), -1.0f) - 1);
                    V1 = min(a.nv - 1, (int)fminf(ceilf(cmax), (float)a.nv) + 1);
                }
                const int nu_w = U1 - U0 + 1;
                const bool staged = nu_w <= kTileCols && V0 <= V1 &&
                                    stage_rays(a, lv, U0, U1, V0, V1, T, lane);
                for (int u = ulo; u <= uhi; u++) {
                    const GCol C = cv[u];
                    if (C.axis != 1) continue;
                    const float fq = __fmaf_rn(C.bq, fj, C.aq);
                    float q[kPlanes];
                    bool any = false;
#pragma unroll
                    for (int p = 0; p < kPlanes; p++) {
                        q[p] = (i0 + p < nx) ? qweight(fq, i0 + p, nx) : 0.f;
                        any |= q[p] != 0.f;
                    }
                    if (!any) continue;
                    int vlo, vhi;
                    row_window(a, P, C.pdiff, a.u0 + ((float)u + 0.5f) * a.du, l, l, zlo, zhi,
                               iez, inv_dv, &vlo, &vhi);
                    const float4* tp = T.ray + (u - U0);
                    const float4* gp = rv + u;
                    for (int v = vlo; v <= vhi; v++) {
                        const bool in_tile = staged && v >= V0 && v <= V1;
                        const float4 r = in_tile ? tp[(v - V0) * nu_w] : __ldg(gp + (long long)v * a.nu);
                        const unsigned m = __float_as_uint(r.w);
                        const float c = valid_at(m, j) ? r.z : 0.f;
                        const float fr = __fmaf_rn(r.y, fj, r.x);
                        const float h0 = c * hat(fr - fk), h1 = c * hat(fr - fk1);
#pragma unroll
                        for (int p = 0; p < kPlanes; p++) {
                            acc[p][0] = __fmaf_rn(q[p], h0, acc[p][0]);
                            acc[p][1] = __fmaf_rn(q[p], h1, acc[p][1]);
                        }
                    }
                }
                __syncwarp();  // every lane is done with the tile before the next one lands
            }
        }
    }
    if (!live) return;
    // out holds what the caller zero-filled, or earlier view blocks / calls
    const bool has_k1 = k + 1 < nz;
#pragma unroll
    for (int p = 0; p < kPlanes; p++) {
        if (i0 + p >= nx) break;
        float* o = a.out + (long long)(i0 + p) * G.s[0] + (long long)j * G.s[1] +
                   (long long)k * G.s[2];
        o[0] += acc[p][0];
        if (has_k1) o[G.s[2]] += acc[p][1];
    }
}

// Rays the gather leaves out (z-driven rays, views outside its family):
// scattered with L2 reductions, one thread per listed ray, as the scatter
// backprojector of the same form walks them.
template <int KIND, typename ST, bool ONES>
__global__ void __launch_bounds__(256) k_bpg_residual(GatherSrc a, int view0,
                                                      const int* residual, const int* nresidual,
                                                      float* out)
{
    const int n = *nresidual;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int lr = residual[s];
        const int lv = lr / (a.nu * a.nv);
        const int rem = lr - lv * a.nu * a.nv;
        const int u = rem / a.nv, v = rem - u * a.nv;
        const int view = view0 + lv;
        const long long r = ((long long)view * a.nu + u) * a.nv + v;
        const float y = ONES ? 1.0f : ld_datum<ST>(a.sino, r);
        float f[18];
#pragma unroll
        for (int i = 0; i < 18; i++) f[i] = __ldg(a.geom + 18 * view + i);
        const Ray R = gather_ray<KIND>(a, f, view, u, v, -1);
        if (R.t0 > R.t1) continue;
        const Grid& G = a.G;
        const long long sp = sel3l(R.p, G.s[0], G.s[1], G.s[2]);
        const int sq = (int)sel3l(R.q, G.s[0], G.s[1], G.s[2]);
        const int sr = (int)sel3l(R.r, G.s[0], G.s[1], G.s[2]);
        // REAL*4 rays clamp their cells; the precision interval needs no clamp
        linear_scatter_span<KIND == 0, false>(R, out, nullptr, sp, sq, sr, R.t0, R.t1, y * R.tvl,
                                              0.f);
    }
}

int g_bp_kind = 0;  // 0: gather where it applies, 1: always the scatter

}  // namespace

int set_backprojector(int kind)
{
    if (kind != 0 && kind != 1) return set_error(CT2_EINVAL, "backprojector kind must be 0 or 1");
    g_bp_kind = kind;
    return CT2_OK;
}

// Gather backprojection of a (or, with ones, of the indicator's ones) added
// into out.
template <int KIND, typename ST>
static int gather_pass(const GatherSrc& a, bool ones, float* out, cudaStream_t st)
{
    const long long nrays_view = (long long)a.nu * a.nv;
    const size_t per_view = (size_t)nrays_view * (sizeof(float4) + sizeof(int)) +
                            (size_t)a.nu * sizeof(GCol) + sizeof(GView);
    long long vb = (long long)(kTableBudget / per_view);
    if (vb < 1) vb = 1;
    if (vb > a.ns) vb = a.ns;
    if (vb * nrays_view > INT32_MAX) vb = INT32_MAX / nrays_view;
    Scratch S(st);
    float4* rec = nullptr;
    GCol* cols = nullptr;
    GView* views = nullptr;
    int *residual = nullptr, *nres = nullptr;
    int rc;
    if ((rc = S.get((void**)&rec, sizeof(float4) * nrays_view * vb, false))) return rc;
    if ((rc = S.get((void**)&cols, sizeof(GCol) * a.nu * vb, false))) return rc;
    if ((rc = S.get((void**)&views, sizeof(GView) * vb, false))) return rc;
    if ((rc = S.get((void**)&residual, sizeof(int) * nrays_view * vb, false))) return rc;
    if ((rc = S.get((void**)&nres, sizeof(int), false))) return rc;
    CT2_CUDA(cudaFuncSetAttribute(k_bpg, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kGatherSmem));
    const Grid& G = a.G;
    const int tiles_j = (G.n[1] + 31) / 32, tiles_i = (G.n[0] + 8 * kPlanes - 1) / (8 * kPlanes);
    const int kpairs = (G.n[2] + 1) / 2;
    const int tiles_det = ((a.nu + 31) / 32) * ((a.nv + 31) / 32);
    GatherArgs g{};
    g.G = G;
    g.nu = a.nu;
    g.nv = a.nv;
    g.du = a.du;
    g.dv = a.dv;
    g.u0 = a.u0;
    g.v0 = a.v0;
    g.rec = rec;
    g.cols = cols;
    g.views = views;
    g.out = out;
    for (int v0 = 0; v0 < a.ns; v0 += (int)vb) {
        const int nb = (int)min(vb, (long long)(a.ns - v0));
        CT2_CUDA(cudaMemsetAsync(views, 0, sizeof(GView) * nb, st));
        CT2_CUDA(cudaMemsetAsync(nres, 0, sizeof(int), st));
        if (ones)
            k_bpg_table<KIND, ST, true><<<dim3(tiles_det, nb), dim3(32, 8), 0, st>>>(
                a, v0, rec, cols, views, residual, nres);
        else
            k_bpg_table<KIND, ST, false><<<dim3(tiles_det, nb), dim3(32, 8), 0, st>>>(
                a, v0, rec, cols, views, residual, nres);
        CT2_LAUNCHED();
        g.nviews = nb;
        k_bpg<<<dim3(tiles_j * tiles_i, kpairs), dim3(32, 8), kGatherSmem, st>>>(g);
        CT2_LAUNCHED();
        if (ones)
            k_bpg_residual<KIND, ST, true><<<1184, 256, 0, st>>>(a, v0, residual, nres, out);
        else
            k_bpg_residual<KIND, ST, false><<<1184, 256, 0, st>>>(a, v0, residual, nres, out);
        CT2_LAUNCHED();
    }
    return CT2_OK;
}

static bool gather_applies(const Grid& G, int nu, int nv)
{
    if (g_bp_kind != 0) return false;
    if (G.n[0] >= 65534 || G.n[1] >= 65534 || G.n[2] >= 65534) return false;
    if (G.n[0] < 1 || G.n[1] < 1 || G.n[2] < 1) return false;
    return (long long)nu * nv <= (1ll << 30);
}

int backproject_gather(const BackprojectArgs& a, cudaStream_t st)
{
    if (!gather_applies(a.G, a.nu, a.nv)) return 1;
    if (a.ns == 0 || a.nu == 0 || a.nv == 0) return CT2_OK;
    const GatherSrc src{a.G, a.sino, ST_F32, a.ind, a.geom, a.ns, a.nu, a.nv,
                        a.du, a.dv, a.u0, a.v0};
    int rc = gather_pass<0, float>(src, false, a.out, st);
    if (rc) return rc;
    if (a.out_ones != nullptr) rc = gather_pass<0, float>(src, true, a.out_ones, st);
    return rc;
}

int prec_backproject_gather(const PrecBackprojectArgs& a, cudaStream_t st)
{
    if (!gather_applies(a.G, a.nu, a.nv)) return 1;
    if (a.sino_type != ST_F32 && a.sino_type != ST_F16) return 1;
    if (a.ns == 0 || a.nu == 0 || a.nv == 0) return CT2_OK;
    const GatherSrc src{a.G, a.sino, a.sino_type, a.ind, a.geom, a.ns, a.nu, a.nv,
                        a.du, a.dv, a.u0, a.v0};
    const bool f16 = a.sino_type == ST_F16;
    int rc = f16 ? gather_pass<1, __half>(src, false, a.out, st)
                 : gather_pass<1, float>(src, false, a.out, st);
    if (rc) return rc;
    if (a.out_ones != nullptr)
        rc = f16 ? gather_pass<1, __half>(src, true, a.out_ones, st)
                 : gather_pass<1, float>(src, true, a.out_ones, st);
    return rc;
}

}  // namespace ct2
