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
//  * k_bpg_table: per ray {ar, br, y * tvl, t0 | (t1 - t0) << 16} in the
//    sinogram's (view, u, v) order (the rows of a detector column
//    contiguous), per detector column {aq, bq, pdiff, axis}, per view the
//    geometry the windows need; rays left to the scatter are listed.
//  * k_bpg<0>, k_bpg<1>: the x-driven and the y-driven columns.  In these
//    views the rays of one column share their q coordinate on every slice,
//    so a voxel's sum factors as sum over columns of wq * P, with P the
//    column's profile along z on that slice: P(k) = sum over the column's
//    rays of y * tvl * hat(fr - k).  A CTA owns a tile of slices x q cells
//    x z cells in shared memory for the whole block of views; per view it
//    takes the columns that reach the tile, computes their profiles (a warp
//    per column, the lanes along z) and adds wq * P into its cells (a warp
//    per slice and lane cell, columns in order).  At the end it adds its
//    sums to the volume (one read and one write per voxel and view block:
//    the volume holds what the caller zero-filled, or the views of earlier
//    blocks and calls -- the host entry points backproject their views in
//    pipelined blocks into one volume).
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

__device__ __forceinline__ float hat(float d) { return __saturatef(1.0f - fabsf(d)); }

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
// Ray table.
// ---------------------------------------------------------------------------
// Part `part` of `nparts` of view block entry lv (view view0 + lv): rays
// part*blockDim, part*blockDim + nparts*blockDim, ... ; part 0 also writes the
// view's columns and window geometry.  Called by whole CTAs.
template <int KIND, typename ST, bool ONES>
__device__ __forceinline__ void table_part(const GatherSrc& a, int view0, int lv, int part,
                                           int nparts, float4* rec, GCol* cols, GView* views,
                                           int* residual, int* nresidual)
{
    const int view = view0 + lv;
    const int nr = a.nu * a.nv;
    float f[18];
#pragma unroll
    for (int i = 0; i < 18; i++) f[i] = __ldg(a.geom + 18 * view + i);
    const bool eligible = f[12] == 0.f && f[13] == 0.f;
    for (int lr = part * blockDim.x + threadIdx.x; lr < nr; lr += nparts * blockDim.x) {
        const int u = lr / a.nv, v = lr - u * a.nv;
        const long long r = (long long)view * nr + lr;
        const bool on = a.ind == nullptr || a.ind[r] == 1;
        const float y = on ? (ONES ? 1.0f : ld_datum<ST>(a.sino, r)) : 0.f;
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
                residual[slot] = lv * nr + lr;
            } else if (R.t0 <= R.t1) {
                c = y * R.tvl;
                meta = (unsigned)R.t0 | ((unsigned)(R.t1 - R.t0) << 16);
            }
        }
        rec[(long long)lv * nr + lr] = make_float4(ar, br, c, __uint_as_float(meta));
    }
    if (part != 0) return;
    // per detector column: driving axis of its x/y-driven rays and their q
    // model; a column whose rays are all zero or disabled adds nothing and is
    // left out (axis 3), as the scatter skips zero rays
    int axes = 0;
    for (int u = threadIdx.x; u < a.nu; u += blockDim.x) {
        GCol C;
        C.axis = 3;
        C.aq = C.bq = C.pdiff = 0.f;
        bool data = false;
        const long long cr = ((long long)view * a.nu + u) * a.nv;
        for (int v = 0; v < a.nv && !data; v++)
            data = (a.ind == nullptr || a.ind[cr + v] == 1) &&
                   (ONES || ld_datum<ST>(a.sino, cr + v) != 0.f);
        if (eligible && data) {
            const int axis = column_axis<KIND>(a, f, u, &C.pdiff);
            const Ray R = gather_ray<KIND>(a, f, view, u, 0, axis);
            C.axis = axis;
            C.aq = R.aq;
            C.bq = R.bq;
            axes |= 1 << axis;
        }
        cols[(long long)lv * a.nu + u] = C;
    }
    const int any_x = __syncthreads_or(axes & 1), any_y = __syncthreads_or(axes & 2);
    if (threadIdx.x == 0) {
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
        P.flags = (any_x ? 1 : 0) | (any_y ? 2 : 0) | (eligible ? 4 : 0);
    }
}

// Table: one thread per ray, in the sinogram's own (view, u, v) order; a
// CTA row (blockIdx.y) per view of the block.
template <int KIND, typename ST, bool ONES>
__global__ void __launch_bounds__(256) k_bpg_table(GatherSrc a, int view0, float4* rec,
                                                   GCol* cols, GView* views, int* residual,
                                                   int* nresidual)
{
    table_part<KIND, ST, ONES>(a, view0, blockIdx.y, blockIdx.x, gridDim.x, rec, cols, views,
                               residual, nresidual);
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

// One CTA owns a tile of kS slices (along the driving axis p of the pass's
// role) x kQ cells along the column axis q x kK cells along z, and keeps its
// sums in shared memory over all views of the block.  Per view and batch of
// detector columns:
//  1. every column's clamped q cell cq and weight wq on each slice (the
//     projector's interpolation in q);
//  2. the phase count: the smallest ph >= 3 such that columns ph, 2 ph, ...
//     apart never feed a common cell on any slice (every pair is checked);
//  3. per phase, a warp per column of the phase: lane l computes, for the
//     tile's kS slices and its kKL z cells k, the column's profile
//     P(s, k) = sum over its rays of datum * hat(fr(s) - k), walking the rows
//     whose fr can reach its cells (a window from the column's linear z
//     model, widened by kWinEps) once for all kS slices, and adds
//     (1 - wq) * P to cell cq and wq * P to cell cq + 1.  No two columns of
//     a phase touch a common cell, and phases run in order.
// Every voxel is summed in a fixed order: no atomics, and the result is the
// same bit for bit on every run.
constexpr int kS = 4;           // slices per tile
constexpr int kQ = 16;          // q cells per tile
constexpr int kKL = 2;          // z cells per lane
constexpr int kK = 32 * kKL;    // z cells per tile
constexpr int kNB = 32;         // columns per batch
constexpr int kWarps = 4;       // warps per CTA
constexpr int kNoCell = INT_MIN;
struct ProfSmem {
    float acc[kS][kQ + 2][kKL][32];  // cells -1 .. kQ: the outer two are never written out
    int cq[kNB][kS];                 // tile cell (cq - Q0), or kNoCell
    float wq[kNB][kS];
};
constexpr size_t kGatherSmem = sizeof(ProfSmem);

// The profile of one column on the tile's kS slices for this lane's kKL z
// cells ka, ka + 1: P(s, k) = sum over rows vlo..vhi of
// y * tvl * hat(fr(s) - k).  CHECK: test every sample against its ray's
// valid interval; otherwise (a tile far inside the volume) every sample is
// valid, and the pair of z cells is accumulated with packed f32x2 FMAs
// (bit-identical to the scalar ones).
template <bool CHECK>
__device__ __forceinline__ void column_profile(const float4* __restrict__ rc, int vlo, int vhi,
                                               int S0, float kfa, float (&P)[kS][kKL])
{
    static_assert(kKL == 2, "the z cells of a lane are accumulated as one f32x2 pair");
    const float kfb = kfa + 1.0f;
    if constexpr (CHECK) {
#pragma unroll
        for (int s = 0; s < kS; s++) P[s][0] = P[s][1] = 0.f;
        for (int v = vlo; v <= vhi; v++) {
            const float4 r = __ldg(rc + v);
            const unsigned m = __float_as_uint(r.w);
            const int t0 = (int)(m & 0xFFFFu);
            const unsigned len = m >> 16;
#pragma unroll
            for (int s = 0; s < kS; s++) {
                const float cs = ((unsigned)(S0 + s - t0) <= len) ? r.z : 0.f;
                const float fr = __fmaf_rn(r.y, (float)(S0 + s), r.x);
                P[s][0] = __fmaf_rn(cs, hat(fr - kfa), P[s][0]);
                P[s][1] = __fmaf_rn(cs, hat(fr - kfb), P[s][1]);
            }
        }
    } else {
        uint64_t P2[kS];
#pragma unroll
        for (int s = 0; s < kS; s++) P2[s] = f2_pack(0.f, 0.f);
        for (int v = vlo; v <= vhi; v++) {
            const float4 r = __ldg(rc + v);
            const uint64_t c2 = f2_pack(r.z, r.z);
#pragma unroll
            for (int s = 0; s < kS; s++) {
                const float fr = __fmaf_rn(r.y, (float)(S0 + s), r.x);
                P2[s] = f2_fma(c2, f2_pack(hat(fr - kfa), hat(fr - kfb)), P2[s]);
            }
        }
#pragma unroll
        for (int s = 0; s < kS; s++) f2_unpack(P2[s], P[s][0], P[s][1]);
    }
}

// ROLE 0: the x-driven columns (slices along x, q = y); ROLE 1: the
// y-driven ones (slices along y, q = x).
// Tile (bx, bz) of the role's grid of tiles: the whole view block's sums
// for its cells, added to a.out.  Called by whole CTAs.
template <int ROLE>
__device__ __forceinline__ void gather_tile(const GatherArgs& a, int bx, int bz, ProfSmem& sm)
{
    constexpr int QA = 1 - ROLE;
    const Grid& G = a.G;
    const int np = G.n[ROLE], nq = G.n[QA], nz = G.n[2];
    const int tiles_s = (np + kS - 1) / kS;
    const int ts = bx % tiles_s, tq = bx / tiles_s;
    const int S0 = ts * kS, Q0 = tq * kQ, K0 = bz * kK;
    const int S1 = min(S0 + kS, np) - 1, Q1 = min(Q0 + kQ, nq) - 1;
    const int w = threadIdx.y, lane = threadIdx.x, tid = w * 32 + lane;
    float* acc_flat = &sm.acc[0][0][0][0];
    for (int e = tid; e < kS * (kQ + 2) * kKL * 32; e += 32 * kWarps) acc_flat[e] = 0.f;
    // view-independent positions: first and last slice centres, the q range
    // whose rays reach the tile's cells (fq in (Q0 - 1, Q1 + 1)), this lane's
    // z cells and the fr range that reaches them
    const float pA = G.o[ROLE] + G.d[ROLE] * ((float)S0 + 0.5f);
    const float pB = G.o[ROLE] + G.d[ROLE] * ((float)S1 + 0.5f);
    const float qlo = G.o[QA] + G.d[QA] * ((float)Q0 - 0.5f - kWinEps);
    const float qhi = G.o[QA] + G.d[QA] * ((float)Q1 + 1.5f + kWinEps);
    const int ka = K0 + kKL * lane;
    const float frlo = (float)ka - 1.0f - kWinEps;
    const float frhi = (float)(ka + kKL - 1) + 1.0f + kWinEps;
    const float inv_du = 1.0f / a.du, inv_dz = 1.0f / G.d[2];
    const float kfa = (float)ka;
    // A tile whose cells lie at least two cells inside the volume in q and
    // z: every sample that reaches one of its cells has its fast q and r
    // coordinates at least a cell inside the volume, far inside the GUARD
    // band, so it lies in its ray's valid interval and needs no test.
    const bool interior = Q0 >= 2 && Q1 <= nq - 3 && K0 >= 2 && min(K0 + kK, nz) - 1 <= nz - 3;
    bool any = false;
    for (int lv = 0; lv < a.nviews; lv++) {
        const GView V = a.views[lv];
        if ((V.flags & (1 << ROLE)) == 0) continue;
        any = true;
        const float Sp = ROLE == 0 ? V.Sx : V.Sy, Sq = ROLE == 0 ? V.Sy : V.Sx;
        const float aR = ROLE == 0 ? V.ax : V.ay, bR = ROLE == 0 ? V.bx : V.by;
        const float cR = ROLE == 0 ? V.cx : V.cy, dR = ROLE == 0 ? V.dx : V.dy;
        // columns whose centre rays cross the tile: a ray of column u has
        // slope (Bq - Sq) / (Bp - Sp) = (aR + bR up) / (cR + dR up) in the
        // (p, q) plane; the tile's extreme slopes lie at its corners
        int ulo, uhi;
        {
            const float lA = pA - Sp, lB = pB - Sp;
            const float s0 = fdiv(qlo - Sq, lA), s1 = fdiv(qhi - Sq, lA);
            const float s2 = fdiv(qlo - Sq, lB), s3 = fdiv(qhi - Sq, lB);
            index_window(fdiv(aR - s0 * cR, s0 * dR - bR), fdiv(aR - s1 * cR, s1 * dR - bR),
                         fdiv(aR - s2 * cR, s2 * dR - bR), fdiv(aR - s3 * cR, s3 * dR - bR),
                         a.u0, inv_du, a.nu, &ulo, &uhi);
        }
        const float4* rview = a.rec + (long long)lv * a.nu * a.nv;
        const GCol* cview = a.cols + (long long)lv * a.nu;
        const float zv = (V.Sz - G.o[2]) * inv_dz - 0.5f;  // fr of the source height
        const float zrow = V.ez * a.dv * inv_dz;           // d(Bz)/dv in voxels
        for (int ub = ulo; ub <= uhi; ub += kNB) {
            const int nb = min(kNB, uhi - ub + 1);
            // ---- 1. cells and weights of the batch's columns
            for (int e = tid; e < nb * kS; e += 32 * kWarps) {
                const int c = e / kS, s = e - c * kS;
                const GCol C = cview[ub + c];
                int cq = kNoCell;
                float wqv = 0.f;
                if (C.axis == ROLE && S0 + s < np) {
                    const float fq = __fmaf_rn(C.bq, (float)(S0 + s), C.aq);
                    const float cf = fminf(fmaxf(floorf(fq), 0.f), (float)(nq - 2));
                    wqv = __fsub_rn(fq, cf);
                    const int q0 = (int)cf - Q0;
                    if (q0 >= -1 && q0 < kQ) cq = q0;  // feeds a cell of the tile
                }
                sm.cq[c][s] = cq;
                sm.wq[c][s] = wqv;
            }
            __syncthreads();
            // ---- 2. phase count
            int ph = 3;
            for (;; ph++) {
                bool ok = true;
                for (int e = tid; e < nb * kS; e += 32 * kWarps) {
                    const int c = e / kS, s = e - c * kS;
                    const int q = sm.cq[c][s];
                    if (q == kNoCell) continue;
                    for (int c2 = c + ph; c2 < nb; c2 += ph) {
                        const int q2 = sm.cq[c2][s];
                        if (q2 != kNoCell && abs(q2 - q) < 2) ok = false;
                    }
                }
                if (__syncthreads_and(ok) || ph >= nb) break;
            }
            // ---- 3. profiles and their cells, phase by phase
            for (int phase = 0; phase < ph; phase++) {
                for (int c = phase + ph * w; c < nb; c += ph * kWarps) {
                    bool live = false;
#pragma unroll
                    for (int s = 0; s < kS; s++) live |= sm.cq[c][s] != kNoCell;
                    if (!live) continue;
                    const int u = ub + c;
                    const GCol C = cview[u];
                    // the column's z model on slice p: fr(v) = zv + lam (z0 + zrow v)
                    // with lam = (p - Sp) / (Bp - Sp); extremes over the tile's
                    // slices at its first and last
                    const float up = a.u0 + ((float)u + 0.5f) * a.du;
                    const float z0 = (V.zq0 + V.euz * up + V.ez * (a.v0 + 0.5f * a.dv)) * inv_dz;
                    const float inv_pd = fdiv(1.0f, C.pdiff);
                    const float lamA = (pA - Sp) * inv_pd, lamB = (pB - Sp) * inv_pd;
                    const float aA = zv + lamA * z0, bA = lamA * zrow;
                    const float aB = zv + lamB * z0, bB = lamB * zrow;
                    const float r0 = fdiv(frlo - aA, bA), r1 = fdiv(frhi - aA, bA);
                    const float r2 = fdiv(frlo - aB, bB), r3 = fdiv(frhi - aB, bB);
                    const float mn = fminf(fminf(r0, r1), fminf(r2, r3));
                    const float mx = fmaxf(fmaxf(r0, r1), fmaxf(r2, r3));
                    int vlo = 0, vhi = a.nv - 1;
                    if (isfinite(mn) && isfinite(mx)) {
                        vlo = max(0, (int)fmaxf(ceilf(mn), -1.0f));
                        vhi = min(a.nv - 1, (int)fminf(floorf(mx), (float)a.nv));
                    }
                    if (ka >= nz) vhi = vlo - 1;
                    float P[kS][kKL];
                    const float4* rc = rview + (long long)u * a.nv;
                    if (interior)
                        column_profile<false>(rc, vlo, vhi, S0, kfa, P);
                    else
                        column_profile<true>(rc, vlo, vhi, S0, kfa, P);
#pragma unroll
                    for (int s = 0; s < kS; s++) {
                        const int q = sm.cq[c][s];
                        if (q == kNoCell) continue;
                        const float wv = sm.wq[c][s], wl = __fsub_rn(1.0f, wv);
#pragma unroll
                        for (int kk = 0; kk < kKL; kk++) {
                            float& t0c = sm.acc[s][q + 1][kk][lane];
                            t0c = __fmaf_rn(wl, P[s][kk], t0c);
                            float& t1c = sm.acc[s][q + 2][kk][lane];
                            t1c = __fmaf_rn(wv, P[s][kk], t1c);
                        }
                    }
                }
                __syncthreads();
            }
        }
    }
    if (!any) return;
    // out holds what the caller zero-filled, or earlier view blocks / calls
    const long long sp = G.s[ROLE], sq = G.s[QA], sz = G.s[2];
    for (int e = tid; e < kS * kQ * kKL * 32; e += 32 * kWarps) {
        const int l = e & 31, kk = (e >> 5) % kKL;
        const int q = (e / (32 * kKL)) % kQ, s = e / (32 * kKL * kQ);
        const int p = S0 + s, qq = Q0 + q, k = K0 + kKL * l + kk;
        if (p >= np || qq >= nq || k >= nz) continue;
        a.out[p * sp + qq * sq + k * sz] += sm.acc[s][q + 1][kk][l];
    }
}

template <int ROLE>
__global__ void __launch_bounds__(32 * kWarps, 8) k_bpg(const __grid_constant__ GatherArgs a)
{
    extern __shared__ float4 gsm[];
    gather_tile<ROLE>(a, blockIdx.x, blockIdx.y, *reinterpret_cast<ProfSmem*>(gsm));
}

// Rays the gather leaves out (z-driven rays, views outside its family):
// scattered with L2 reductions, one thread per listed ray, as the scatter
// backprojector of the same form walks them.
template <int KIND, typename ST, bool ONES>
__device__ __forceinline__ void residual_ray(const GatherSrc& a, int view0, int lr, float* out)
{
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
    if (R.t0 > R.t1) return;
    const Grid& G = a.G;
    const long long sp = sel3l(R.p, G.s[0], G.s[1], G.s[2]);
    const int sq = (int)sel3l(R.q, G.s[0], G.s[1], G.s[2]);
    const int sr = (int)sel3l(R.r, G.s[0], G.s[1], G.s[2]);
    // REAL*4 rays clamp their cells; the precision interval needs no clamp
    linear_scatter_span<KIND == 0, false>(R, out, nullptr, sp, sq, sr, R.t0, R.t1, y * R.tvl,
                                          0.f);
}

template <int KIND, typename ST, bool ONES>
__global__ void __launch_bounds__(256) k_bpg_residual(GatherSrc a, int view0,
                                                      const int* residual, const int* nresidual,
                                                      float* out)
{
    const int n = *nresidual;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        residual_ray<KIND, ST, ONES>(a, view0, residual[s], out);
}

// ---------------------------------------------------------------------------
// Several backprojections in one launch per kernel (the served stream's
// batched iteration).  A job is one view block of one backprojection of
// FP32 data (no indicator) into its own volume; every kernel takes work items
// across all jobs in turn, and each item runs exactly the code of the
// single-job kernels.
// ---------------------------------------------------------------------------
struct GatherJob {
    GatherSrc src;
    GatherArgs g;
    int view0;
    float4* rec;
    GCol* cols;
    GView* views;
    int* residual;
    int* nres;
    long long item0[3];  // first table item, first x-driven tile, first y-driven tile
    int tparts;          // table parts per view
    int tiles[2];        // tiles per z layer, x- and y-driven role
    int ztiles;
};

__device__ __forceinline__ int find_job(const GatherJob* jobs, int njobs, int k, long long it)
{
    int j = 0;
    while (j + 1 < njobs && jobs[j + 1].item0[k] <= it) j++;
    return j;
}

__global__ void k_bpg_reset_batch(const GatherJob* jobs, int njobs, unsigned long long* counters)
{
    for (int j = threadIdx.x; j < njobs; j += blockDim.x) *jobs[j].nres = 0;
    if (threadIdx.x < 3) counters[threadIdx.x] = 0;
}

// Next work item of a batched launch, taken from the launch's counter by
// thread 0 and read by the CTA after a barrier (every thread is then also
// done with the previous item).
__device__ __forceinline__ long long next_item(unsigned long long* counter)
{
    __shared__ long long s_item;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) s_item = (long long)atomicAdd(counter, 1ull);
    __syncthreads();
    return s_item;
}

constexpr int kTableGroup = 4;  // table parts (256 rays each) per batched work item

__global__ void __launch_bounds__(256) k_bpg_table_batch(const GatherJob* jobs, int njobs,
                                                         long long total,
                                                         unsigned long long* counter)
{
    for (long long it = next_item(counter); it < total; it = next_item(counter)) {
        const GatherJob& J = jobs[find_job(jobs, njobs, 0, it)];
        const long long li = it - J.item0[0];
        const int items = (J.tparts + kTableGroup - 1) / kTableGroup;  // per view
        const int lv = (int)(li / items), grp = (int)(li - (long long)lv * items);
        for (int part = grp * kTableGroup; part < min(J.tparts, (grp + 1) * kTableGroup); part++)
            table_part<0, float, false>(J.src, J.view0, lv, part, J.tparts, J.rec, J.cols,
                                        J.views, J.residual, J.nres);
    }
}

template <int ROLE>
__global__ void __launch_bounds__(32 * kWarps, 8) k_bpg_batch(const GatherJob* jobs, int njobs,
                                                              long long total,
                                                              unsigned long long* counter)
{
    extern __shared__ float4 gsm[];
    ProfSmem& sm = *reinterpret_cast<ProfSmem*>(gsm);
    __shared__ GatherArgs g;  // the item's job, read once per item
    for (long long it = next_item(counter); it < total; it = next_item(counter)) {
        const int j = find_job(jobs, njobs, 1 + ROLE, it);
        const long long li = it - jobs[j].item0[1 + ROLE];
        const int per = jobs[j].tiles[ROLE];
        const int bz = (int)(li / per), bx = (int)(li - (long long)bz * per);
        if (threadIdx.x == 0 && threadIdx.y == 0) g = jobs[j].g;
        __syncthreads();
        gather_tile<ROLE>(g, bx, bz, sm);
    }
}

__global__ void __launch_bounds__(256) k_bpg_residual_batch(const GatherJob* jobs, int njobs)
{
    for (int j = 0; j < njobs; j++) {
        const int n = *jobs[j].nres;
        for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
            residual_ray<0, float, false>(jobs[j].src, jobs[j].view0, jobs[j].residual[s],
                                          jobs[j].g.out);
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
// Views per block: as many as the table budget holds (at least one).
static long long block_views(int ns, int nu, int nv)
{
    const long long nrays_view = (long long)nu * nv;
    const size_t per_view = (size_t)nrays_view * (sizeof(float4) + sizeof(int)) +
                            (size_t)nu * sizeof(GCol) + sizeof(GView);
    long long vb = (long long)(kTableBudget / per_view);
    if (vb < 1) vb = 1;
    if (vb > ns) vb = ns;
    if (vb * nrays_view > INT32_MAX) vb = INT32_MAX / nrays_view;
    return vb;
}

template <int KIND, typename ST>
static int gather_pass(const GatherSrc& a, bool ones, float* out, cudaStream_t st)
{
    const long long nrays_view = (long long)a.nu * a.nv;
    const long long vb = block_views(a.ns, a.nu, a.nv);
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
    CT2_CUDA(cudaFuncSetAttribute(k_bpg<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kGatherSmem));
    CT2_CUDA(cudaFuncSetAttribute(k_bpg<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kGatherSmem));
    const Grid& G = a.G;
    const int ztiles = (G.n[2] + kK - 1) / kK;
    const int tiles_x = ((G.n[0] + kS - 1) / kS) * ((G.n[1] + kQ - 1) / kQ);  // x-driven role
    const int tiles_y = ((G.n[1] + kS - 1) / kS) * ((G.n[0] + kQ - 1) / kQ);  // y-driven role
    const int table_blocks = (int)min((nrays_view + 255) / 256, 2048ll);
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
        CT2_CUDA(cudaMemsetAsync(nres, 0, sizeof(int), st));
        if (ones)
            k_bpg_table<KIND, ST, true><<<dim3(table_blocks, nb), 256, 0, st>>>(
                a, v0, rec, cols, views, residual, nres);
        else
            k_bpg_table<KIND, ST, false><<<dim3(table_blocks, nb), 256, 0, st>>>(
                a, v0, rec, cols, views, residual, nres);
        CT2_LAUNCHED();
        g.nviews = nb;
        k_bpg<0><<<dim3(tiles_x, ztiles), dim3(32, kWarps), kGatherSmem, st>>>(g);
        CT2_LAUNCHED();
        k_bpg<1><<<dim3(tiles_y, ztiles), dim3(32, kWarps), kGatherSmem, st>>>(g);
        CT2_LAUNCHED();
        if (ones)
            k_bpg_residual<KIND, ST, true><<<1184, 256, 0, st>>>(a, v0, residual, nres, out);
        else
            k_bpg_residual<KIND, ST, false><<<1184, 256, 0, st>>>(a, v0, residual, nres, out);
        CT2_LAUNCHED();
    }
    return CT2_OK;
}

static bool gather_fits(const Grid& G, int nu, int nv)
{
    if (G.n[0] >= 65534 || G.n[1] >= 65534 || G.n[2] >= 65534) return false;
    if (G.n[0] < 2 || G.n[1] < 2 || G.n[2] < 2) return false;
    return (long long)nu * nv <= (1ll << 30);
}

static bool gather_applies(const Grid& G, int nu, int nv)
{
    return g_bp_kind == 0 && gather_fits(G, nu, nv);
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

// ---- batched backprojections (the served stream's iteration)

size_t gather_job_bytes() { return sizeof(GatherJob); }

bool gather_batch_applies(const BackprojectArgs& a)
{
    return gather_applies(a.G, a.nu, a.nv) && a.ind == nullptr;
}

int gather_block_views(int ns, int nu, int nv) { return (int)block_views(ns, nu, nv); }

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t gather_scratch_bytes(int nu, int nv, int vb)
{
    const size_t nr = (size_t)nu * nv * vb;
    return align256(nr * sizeof(float4)) + align256((size_t)nu * vb * sizeof(GCol)) +
           align256((size_t)vb * sizeof(GView)) + align256(nr * sizeof(int)) + 256;
}

int gather_job_fill(void* desc, const BackprojectArgs& a, int view0, int nb, void* scratch)
{
    if (!gather_fits(a.G, a.nu, a.nv) || a.ind != nullptr || nb < 1 || view0 < 0 ||
        view0 + nb > a.ns)
        return 1;
    GatherJob& J = *reinterpret_cast<GatherJob*>(desc);
    J = GatherJob{};
    J.src = GatherSrc{a.G, a.sino, ST_F32, nullptr, a.geom, a.ns, a.nu, a.nv,
                      a.du, a.dv, a.u0, a.v0};
    char* p = reinterpret_cast<char*>(scratch);
    const size_t nr = (size_t)a.nu * a.nv * nb;
    J.rec = reinterpret_cast<float4*>(p);
    p += align256(nr * sizeof(float4));
    J.cols = reinterpret_cast<GCol*>(p);
    p += align256((size_t)a.nu * nb * sizeof(GCol));
    J.views = reinterpret_cast<GView*>(p);
    p += align256((size_t)nb * sizeof(GView));
    J.residual = reinterpret_cast<int*>(p);
    p += align256(nr * sizeof(int));
    J.nres = reinterpret_cast<int*>(p);
    J.view0 = view0;
    J.g = GatherArgs{};
    J.g.G = a.G;
    J.g.nu = a.nu;
    J.g.nv = a.nv;
    J.g.du = a.du;
    J.g.dv = a.dv;
    J.g.u0 = a.u0;
    J.g.v0 = a.v0;
    J.g.nviews = nb;
    J.g.rec = J.rec;
    J.g.cols = J.cols;
    J.g.views = J.views;
    J.g.out = a.out;
    J.tparts = (a.nu * a.nv + 255) / 256;
    J.tiles[0] = ((a.G.n[0] + kS - 1) / kS) * ((a.G.n[1] + kQ - 1) / kQ);
    J.tiles[1] = ((a.G.n[1] + kS - 1) / kS) * ((a.G.n[0] + kQ - 1) / kQ);
    J.ztiles = (a.G.n[2] + kK - 1) / kK;
    return CT2_OK;
}

void gather_jobs_finalize(void* descs, int njobs, long long totals[3])
{
    GatherJob* J = reinterpret_cast<GatherJob*>(descs);
    totals[0] = totals[1] = totals[2] = 0;
    for (int j = 0; j < njobs; j++) {
        J[j].item0[0] = totals[0];
        J[j].item0[1] = totals[1];
        J[j].item0[2] = totals[2];
        totals[0] += (long long)J[j].g.nviews * ((J[j].tparts + kTableGroup - 1) / kTableGroup);
        totals[1] += (long long)J[j].tiles[0] * J[j].ztiles;
        totals[2] += (long long)J[j].tiles[1] * J[j].ztiles;
    }
}

int gather_batch_round(const void* d_descs, int njobs, const long long totals[3], int grid,
                       unsigned long long* counters, cudaStream_t st)
{
    if (njobs <= 0) return CT2_OK;
    const GatherJob* J = reinterpret_cast<const GatherJob*>(d_descs);
    CT2_CUDA(cudaFuncSetAttribute(k_bpg_batch<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kGatherSmem));
    CT2_CUDA(cudaFuncSetAttribute(k_bpg_batch<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kGatherSmem));
    k_bpg_reset_batch<<<1, 64, 0, st>>>(J, njobs, counters);
    CT2_LAUNCHED();
    k_bpg_table_batch<<<grid, 256, 0, st>>>(J, njobs, totals[0], counters);
    CT2_LAUNCHED();
    k_bpg_batch<0><<<grid, dim3(32, kWarps), kGatherSmem, st>>>(J, njobs, totals[1],
                                                                 counters + 1);
    CT2_LAUNCHED();
    k_bpg_batch<1><<<grid, dim3(32, kWarps), kGatherSmem, st>>>(J, njobs, totals[2],
                                                                 counters + 2);
    CT2_LAUNCHED();
    k_bpg_residual_batch<<<grid, 256, 0, st>>>(J, njobs);
    CT2_LAUNCHED();
    return CT2_OK;
}

}  // namespace ct2
