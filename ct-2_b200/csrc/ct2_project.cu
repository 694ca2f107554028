// Forward projectors: thread-per-ray Joseph line integrals.
//
// Reference: view_proj3D.sinoproj_linear / sinoproj_nearest
// (emil_code/view_proj3D.f:703-910 / :915-1092), view_proj3D_tomo.sinoprojz
// (emil_code/view_proj3D_tomo.f:4-148), ray_proj3D.sinoproj_linear /
// sinoproj_nearest (emil_code/ray_proj3D.f:514-671 / :677-804).
//
// Mapping: one thread per detector pixel; a CTA covers 32 pixels along v by
// 8 along u of one view, so a warp's 32 rays are consecutive in v.  The
// sinogram (ns, nu, nv) is C-ordered with v fastest, so stores coalesce, and
// for the circular cone-beam geometry v runs along z, the fastest axis of the
// C-ordered volume, so each bilinear tap of a warp touches one or two 128-byte
// lines.  The EM variant writes the ratio y / max(Ax, small) instead of Ax.
#include <cuda.h>  // CUtensorMap and its enums (encoded through the runtime's driver entry point)

#include <climits>

#include "ct2_common.cuh"
#include "ct2_kernels.h"

namespace ct2 {

template <bool CLAMP>
__device__ __forceinline__ float linear_span(const Ray& R, const float* __restrict__ vol,
                                             long long sp, int sq, int sr, int t0, int t1)
{
    float acc = 0.f;
    if (t0 > t1) return acc;
    const float* plane = vol + (long long)t0 * sp;
    float tf = (float)t0;
#pragma unroll 2
    for (int t = t0; t <= t1; t++, tf += 1.0f, plane += sp) {
        int iq, ir;
        float wq2, wr2;
        sample_in<CLAMP>(R, tf, iq, ir, wq2, wr2);
        const float* b = plane + (iq * sq + ir * sr);
        const float v00 = __ldg(b), v10 = __ldg(b + sq);
        const float v01 = __ldg(b + sr), v11 = __ldg(b + sq + sr);
        const float vi1 = __fmaf_rn(wq2, v10 - v00, v00);
        const float vi2 = __fmaf_rn(wq2, v11 - v01, v01);
        acc += __fmaf_rn(wr2, vi2 - vi1, vi1);
    }
    return acc;
}

// The unclamped interior run [t0, t1] of a ray whose in-plane axis r has
// stride 1 (the x- and y-driven rays of a z-fastest volume): the same
// samples, cells and weights as linear_span<false>, with the coordinate,
// floor and weight arithmetic of q and r packed into f32x2 instructions and
// the tap addresses formed from 32-bit offsets (the caller guarantees that
// every offset in the volume fits in 32 bits).  floor(x) = bits(x + 1.5*2^23
// rounded down) - 0x4B400000; the constant is folded into the base offset.
__device__ __forceinline__ float linear_span_r1(const Ray& R, const float* __restrict__ vol,
                                                uint32_t sp, uint32_t sq, int t0, int t1)
{
    float acc = 0.f;
    if (t0 > t1) return acc;
    const uint64_t A = f2_pack(R.aq, R.ar), B = f2_pack(R.bq, R.br);
    const uint64_t M = f2_pack(12582912.0f, 12582912.0f), ONE = f2_pack(1.0f, 1.0f);
    uint64_t T = f2_pack((float)t0, (float)t0);
    // offset(t) = t*sp + iq*sq + ir, with iq = bq - 0x4B400000, ir = br - 0x4B400000
    uint32_t base = (uint32_t)t0 * sp - 0x4B400000u * (sq + 1u);
    const float* __restrict__ volq = vol + sq;
#pragma unroll 4
    for (int t = t0; t <= t1; t++) {
        const uint64_t f = f2_fma(B, T, A);
        const uint64_t tt = f2_add_rd(f, M);
        const uint64_t w = f2_sub(f, f2_sub(tt, M));
        float tq, tr, wq2, wr2;
        f2_unpack(tt, tq, tr);
        f2_unpack(w, wq2, wr2);
        const uint32_t off = __float_as_uint(tq) * sq + __float_as_uint(tr) + base;
        const float* b0 = vol + off;
        const float* b1 = volq + off;
        const float v00 = __ldg(b0), v01 = __ldg(b0 + 1);
        const float v10 = __ldg(b1), v11 = __ldg(b1 + 1);
        const uint64_t lo = f2_pack(v00, v01);
        const uint64_t vi = f2_fma(f2_pack(wq2, wq2), f2_sub(f2_pack(v10, v11), lo), lo);
        float vi1, vi2;
        f2_unpack(vi, vi1, vi2);
        acc += __fmaf_rn(wr2, vi2 - vi1, vi1);
        T = f2_add(T, ONE);
        base += sp;
    }
    return acc;
}

// Line integral of one ray: the exact interval's clamped ends and its
// interior run, or (nearest mode) the reference arithmetic per sample.
template <int MODE>
__device__ __forceinline__ float ray_sum(const Grid& G, Ray& R, const float* __restrict__ vol)
{
    const long long sp = sel3l(R.p, G.s[0], G.s[1], G.s[2]);
    const int sq = (int)sel3l(R.q, G.s[0], G.s[1], G.s[2]);
    const int sr = (int)sel3l(R.r, G.s[0], G.s[1], G.s[2]);
    if (MODE == MODE_LINEAR) {
        int s0, s1;
        exact_interval(R, R.np, &s0, &s1);
        if (R.t0 > R.t1) return 0.f;
        float acc;
        if (s0 > s1) {
            acc = linear_span<true>(R, vol, sp, sq, sr, R.t0, R.t1);
        } else {
            // the clamped ends first, so that only the interior run's state is
            // live in its loop
            acc = linear_span<true>(R, vol, sp, sq, sr, R.t0, s0 - 1);
            acc += linear_span<true>(R, vol, sp, sq, sr, s1 + 1, R.t1);
            if (sr == 1 && G.small)
                acc += linear_span_r1(R, vol, (uint32_t)sp, (uint32_t)sq, s0, s1);
            else
                acc += linear_span<false>(R, vol, sp, sq, sr, s0, s1);
        }
        return acc * R.tvl;
    }
    float acc = 0.f;
    if (R.t0 > R.t1) return 0.f;
    const float* plane = vol + (long long)R.t0 * sp;
    for (int t = R.t0; t <= R.t1; t++, plane += sp) {
        int iq, ir;
        if (sample_nearest(R, t, MODE, iq, ir)) acc += __ldg(plane + iq * sq + ir * sr);
    }
    return acc * R.tvl;
}

// Writes ray r's line integral s, or for EM y / max(s, small) with the
// reference's clamp.
template <bool EMRATIO>
__device__ __forceinline__ void store_ray(const ProjectArgs& a, long long r, float s)
{
    if (EMRATIO) {
        const float raysum = (s < a.em_small) ? 1.0f : s;
        a.out[r] = __fdiv_rn(a.y[r], raysum);
    } else {
        a.out[r] = s;
    }
}

// Detector pixel (ju, kv) of view `view` (view geometry, in range).
template <int MODE, int FORCE, bool EMRATIO>
__device__ __forceinline__ void project_view_pixel(const ProjectArgs& a, int view, int ju, int kv)
{
    const long long r = ((long long)view * a.nu + ju) * a.nv + kv;
    const float* fv = a.geom + 18 * view;
    float S[3], B[3];
    S[0] = __ldg(fv); S[1] = __ldg(fv + 1); S[2] = __ldg(fv + 2);
    float f[18];
#pragma unroll
    for (int i = 0; i < 18; i++) f[i] = __ldg(fv + i);
    view_bin(f, ju, kv, a.du, a.dv, a.u0, a.v0, B);
    if (a.ind != nullptr && a.ind[r] != 1) {
        a.out[r] = 0.f;  // f2py zero-fills intent(out); disabled rays stay 0
        return;
    }
    Ray R = ray_setup(a.G, S, B, FORCE, MODE);
    store_ray<EMRATIO>(a, r, ray_sum<MODE>(a.G, R, a.vol));
}

// out[r] = A x (or, for EM, y / max(A x, small) with the reference's clamp).
template <int MODE, bool LIST, int FORCE, bool EMRATIO>
__global__ void __launch_bounds__(256) k_project(ProjectArgs a)
{
    if (LIST) {
        const long long r =
            (long long)blockIdx.x * blockDim.x * blockDim.y + threadIdx.y * blockDim.x + threadIdx.x;
        if (r >= a.nrays) return;
        const float* v = a.geom + 6 * r;
        float S[3], B[3];
        S[0] = v[0]; S[1] = v[1]; S[2] = v[2];
        B[0] = v[3]; B[1] = v[4]; B[2] = v[5];
        if (a.ind != nullptr && a.ind[r] != 1) {
            a.out[r] = 0.f;
            return;
        }
        Ray R = ray_setup(a.G, S, B, FORCE, MODE);
        store_ray<EMRATIO>(a, r, ray_sum<MODE>(a.G, R, a.vol));
    } else {
        const int tiles_v = (a.nv + 31) >> 5;
        const int tu = blockIdx.x / tiles_v, tv = blockIdx.x - tu * tiles_v;
        const int kv = tv * 32 + threadIdx.x, ju = tu * 8 + threadIdx.y;
        if (kv >= a.nv || ju >= a.nu) return;
        project_view_pixel<MODE, FORCE, EMRATIO>(a, blockIdx.y, ju, kv);
    }
}

// Several jobs' projections (or EM ratios) in one persistent launch: a work
// item is a 32 (v) x 8 (u) pixel tile of one view of one job, the CTAs take
// items in turn; every pixel is computed exactly as k_project computes it.
template <bool EMRATIO>
__global__ void __launch_bounds__(256) k_project_batch(const ProjectJob* __restrict__ jobs,
                                                       int njobs, long long total)
{
    for (long long it = blockIdx.x; it < total; it += gridDim.x) {
        int j = 0;
        while (j + 1 < njobs && jobs[j + 1].item0 <= it) j++;
        const ProjectArgs a = jobs[j].a;
        const long long li = it - jobs[j].item0;
        const int tiles_v = (a.nv + 31) >> 5, tiles = tiles_v * ((a.nu + 7) >> 3);
        const int view = (int)(li / tiles), tile = (int)(li - (long long)view * tiles);
        const int tu = tile / tiles_v, tv = tile - tu * tiles_v;
        const int kv = tv * 32 + threadIdx.x, ju = tu * 8 + threadIdx.y;
        if (kv < a.nv && ju < a.nu)
            project_view_pixel<MODE_LINEAR, -1, EMRATIO>(a, view, ju, kv);
    }
}

int project_batch_items(const ProjectArgs& a)
{
    return ((a.nv + 31) >> 5) * ((a.nu + 7) >> 3);  // per view
}


// ---------------------------------------------------------------------
// TMA-staged projector (view geometry, linear mode, x- or y-driven tiles)
//
// A CTA's 8 x 32 rays cross the volume together.  Their interior runs are cut
// into chunks of TK slices; for each chunk one thread computes the box of
// cells the tile can touch -- the slice position is linear-fractional over
// the detector tile and linear in t, so its extremes lie at the tile's four
// corner rays and the chunk's two ends -- and loads it into shared memory
// with one TMA tile copy (cp.async.bulk.tensor, no multicast) completing on
// an mbarrier, two chunks ahead (double buffer).  Each ray then reads its
// bilinear taps from shared memory, after checking that its own first and
// last cells of the chunk lie in the box (its cells move monotonically with
// t, so every cell between does too); a ray or chunk outside the box reads
// global memory as the untiled kernel does.  The sample set, cells and
// weights are those of k_project.  A form with two rays per thread (the same
// 32 x 8 tile on 128 threads, the q arithmetic shared) gave bit-identical
// sums but took 19.9 ms against 13.0 ms on 256^3 x 360 views x 384^2 (B200):
// the boxes bound a CTA's rays, so halving the threads per tile halved the
// resident warps (16 per SM) with the shared memory per SM unchanged.  A
// staged span taking two slices at a time (coordinates paired per axis
// across the two slices, both interpolations as pair operations, fewer
// instructions per sample) was also bit-identical and took 13.17 ms.
// ---------------------------------------------------------------------
constexpr int TK = 8, TQ = 20, TR = 40;  // box: slices x q rows x r columns (r innermost)
constexpr int TSTAGE = TK * TQ * TR;
constexpr unsigned TSTAGE_BYTES = TSTAGE * 4u;
constexpr int kMbarSpins = 1 << 22;     // bounded wait (each try_wait also suspends briefly)

static __device__ int g_tma_timeouts = 0;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase with the given parity, at most `spins` tries.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int spins)
{
    for (int i = 0; i < spins; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// The projector's wait: gives up after kMbarSpins tries, counts the timeout
// (ct2_wait_timeouts) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    if (mbar_wait_bounded(bar, parity, kMbarSpins)) return true;
    atomicAdd(&g_tma_timeouts, 1);
    return false;
}
__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// Interior samples [lo, hi] of one ray from a staged box whose origin is
// (tc, qlo, rlo): PX = 0 (x-driven; box stored [TK][TQ][TR]) or 1 (y-driven;
// box stored [TQ][TK][TR]).
template <int PX>
__device__ __forceinline__ float staged_span(const Ray& R, const float* __restrict__ box, int qlo,
                                             int rlo, int tc, int lo, int hi)
{
    constexpr uint32_t S_T = PX == 0 ? TQ * TR : TR;
    constexpr uint32_t S_Q = PX == 0 ? TR : TK * TR;
    const uint64_t A = f2_pack(R.aq, R.ar), B = f2_pack(R.bq, R.br);
    const uint64_t M = f2_pack(12582912.0f, 12582912.0f), ONE = f2_pack(1.0f, 1.0f);
    uint64_t T = f2_pack((float)lo, (float)lo);
    uint32_t base = (uint32_t)(lo - tc) * S_T - ((uint32_t)qlo + 0x4B400000u) * S_Q -
                    ((uint32_t)rlo + 0x4B400000u);
    float acc = 0.f;
#pragma unroll 4
    for (int t = lo; t <= hi; t++) {
        const uint64_t f = f2_fma(B, T, A);
        const uint64_t tt = f2_add_rd(f, M);
        float tq, tr, wq2, wr2;
        f2_unpack(tt, tq, tr);
        f2_unpack(f2_sub(f, f2_sub(tt, M)), wq2, wr2);
        const float* b = box + (__float_as_uint(tq) * S_Q + __float_as_uint(tr) + base);
        const uint64_t lo2 = f2_pack(b[0], b[1]);
        const uint64_t vi = f2_fma(f2_pack(wq2, wq2), f2_sub(f2_pack(b[S_Q], b[S_Q + 1]), lo2), lo2);
        float vi1, vi2;
        f2_unpack(vi, vi1, vi2);
        acc += __fmaf_rn(wr2, vi2 - vi1, vi1);
        T = f2_add(T, ONE);
        base += S_T;
    }
    return acc;
}

// Box of chunk c (first slice tc, last te) from the corner models; stages it
// (or marks it unusable) and arrives on the stage's mbarrier.
__device__ __forceinline__ void issue_chunk(const float (*corner)[4], int px, int tc, int te,
                                            int (*box)[3], int st, uint64_t* bar, float* stage,
                                            const CUtensorMap* mapx, const CUtensorMap* mapy)
{
    float qmin = INFINITY, qmax = -INFINITY, rmin = INFINITY, rmax = -INFINITY;
    for (int k = 0; k < 4; k++) {
        for (int e = 0; e < 2; e++) {
            const float t = (float)(e ? te : tc);
            const float fq = __fmaf_rn(corner[k][1], t, corner[k][0]);
            const float fr = __fmaf_rn(corner[k][3], t, corner[k][2]);
            qmin = fminf(qmin, fq);
            qmax = fmaxf(qmax, fq);
            rmin = fminf(rmin, fr);
            rmax = fmaxf(rmax, fr);
        }
    }
    bool ok = isfinite(qmin) && isfinite(qmax) && isfinite(rmin) && isfinite(rmax) &&
              fabsf(qmin) < 1e6f && fabsf(qmax) < 1e6f && fabsf(rmin) < 1e6f && fabsf(rmax) < 1e6f;
    int qlo = 0, rlo = 0;
    if (ok) {
        qlo = (int)floorf(qmin - 0.05f);
        const int qhi = (int)floorf(qmax + 0.05f) + 1;
        rlo = ((int)floorf(rmin - 0.05f)) & ~3;  // TMA: innermost coordinate a multiple of 16 bytes
        const int rhi = (int)floorf(rmax + 0.05f) + 1;
        ok = (qhi - qlo + 1 <= TQ) && (rhi - rlo + 1 <= TR);
    }
    box[st][0] = qlo;
    box[st][1] = rlo;
    box[st][2] = ok ? 1 : 0;
    if (ok) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(bar, TSTAGE_BYTES);
        if (px == 0)
            tma_load_3d(stage, mapx, bar, rlo, qlo, tc);  // (z, y, x): box TR x TQ x TK
        else
            tma_load_3d(stage, mapy, bar, rlo, tc, qlo);  // (z, y, x): box TR x TK x TQ
    } else {
        mbar_arrive(bar);
    }
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// A tensor map read from global memory, which the host rewrote (a copy into a
// descriptor array whose addresses get reused): orders the copy's writes
// before this thread's later copies through the map, so none of them uses a
// map cached from an earlier content of the same address.  System scope: the
// writer is a host copy.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(
                     reinterpret_cast<uint64_t>(map))
                 : "memory");
}

// Tile `tile` (32 v x 8 u pixels) of view `view`, with the volume's tensor
// maps at mx (x-driven boxes) and my (y-driven boxes).  Called by whole CTAs;
// reinit: the CTA ran an earlier tile, whose mbarriers are invalidated
// before they are set up again (every copy of that tile has completed).
template <bool EMRATIO>
__device__ __forceinline__ void project_tma_tile(const ProjectArgs& a, const CUtensorMap* mx,
                                                 const CUtensorMap* my, int tile, int view,
                                                 bool reinit)
{
    extern __shared__ __align__(128) float tsm[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ int s_box[2][3];
    __shared__ int s_tlo, s_thi, s_pmin, s_pmax, s_abort;
    __shared__ float s_corner[4][4];
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int tiles_v = (a.nv + 31) >> 5;
    const int tu = tile / tiles_v, tv = tile - tu * tiles_v;
    const int kv = tv * 32 + threadIdx.x, ju = tu * 8 + threadIdx.y;
    const bool in_det = (kv < a.nv) && (ju < a.nu);
    const long long r = in_det ? ((long long)view * a.nu + ju) * a.nv + kv : 0;
    const bool on = in_det && (a.ind == nullptr || a.ind[r] == 1);
    if (tid == 0) {
        s_tlo = INT_MAX;
        s_thi = INT_MIN;
        s_pmin = 3;
        s_pmax = -1;
        s_abort = 0;
        if (reinit) {
            mbar_inval(&mbar[0]);
            mbar_inval(&mbar[1]);
        }
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    float f[18];
#pragma unroll
    for (int i = 0; i < 18; i++) f[i] = __ldg(a.geom + 18 * view + i);
    Ray R;
    int s0 = 1, s1 = 0;
    float acc = 0.f;
    long long sp = 0;
    int sq = 0, sr = 0;
    if (on) {
        const float S[3] = {f[0], f[1], f[2]};
        float B[3];
        view_bin(f, ju, kv, a.du, a.dv, a.u0, a.v0, B);
        R = ray_setup(a.G, S, B, -1, MODE_LINEAR);
        exact_interval(R, R.np, &s0, &s1);
        sp = sel3l(R.p, a.G.s[0], a.G.s[1], a.G.s[2]);
        sq = (int)sel3l(R.q, a.G.s[0], a.G.s[1], a.G.s[2]);
        sr = (int)sel3l(R.r, a.G.s[0], a.G.s[1], a.G.s[2]);
        if (R.t0 <= R.t1) {
            if (s0 > s1) {
                acc = linear_span<true>(R, a.vol, sp, sq, sr, R.t0, R.t1);
            } else {
                acc = linear_span<true>(R, a.vol, sp, sq, sr, R.t0, s0 - 1);
                acc += linear_span<true>(R, a.vol, sp, sq, sr, s1 + 1, R.t1);
                atomicMin(&s_tlo, s0);
                atomicMax(&s_thi, s1);
                atomicMin(&s_pmin, R.p);
                atomicMax(&s_pmax, R.p);
            }
        } else {
            s0 = 1;
            s1 = 0;
        }
    }
    __syncthreads();
    const int px = s_pmin;
    const bool staged = (s_pmin == s_pmax) && (px <= 1) && a.G.small;
    if (staged && tid < 4) {
        // corner rays of the tile (clipped to the detector), forced to the tile's axis
        const int cj = (tid & 1) ? min(tu * 8 + 7, a.nu - 1) : tu * 8;
        const int ck = (tid & 2) ? min(tv * 32 + 31, a.nv - 1) : tv * 32;
        const float S[3] = {f[0], f[1], f[2]};
        float B[3];
        view_bin(f, cj, ck, a.du, a.dv, a.u0, a.v0, B);
        const Ray C = ray_setup(a.G, S, B, px, MODE_LINEAR);
        s_corner[tid][0] = C.aq;
        s_corner[tid][1] = C.bq;
        s_corner[tid][2] = C.ar;
        s_corner[tid][3] = C.br;
    }
    __syncthreads();
    if (staged) {
        const int tlo = s_tlo, thi = s_thi;
        const int nchunks = (thi >= tlo) ? (thi - tlo) / TK + 1 : 0;
        // last chunk issued into each stage (thread 0's bookkeeping, -1: none)
        int last_issued[2] = {-1, -1};
        if (tid == 0) {
            for (int c = 0; c < 2 && c < nchunks; c++) {
                issue_chunk(s_corner, px, tlo + c * TK, min(tlo + c * TK + TK - 1, thi), s_box, c,
                            &mbar[c], tsm + c * TSTAGE, mx, my);
                last_issued[c] = c;
            }
        }
        // A wait that runs out: that thread reads the chunk from global memory
        // (the same sum bit for bit) and raises s_abort; after the next block
        // barrier no thread waits on or reads a stage again, thread 0 issues
        // no further copy, and before the CTA ends thread 0 waits (bounded)
        // for the copies still in flight, so none lands in reassigned memory.
        bool aborted = false;
        for (int c = 0; c < nchunks; c++) {
            const int st = c & 1;
            bool stage_ready = false;
            if (!aborted) {
                stage_ready = mbar_wait(&mbar[st], (uint32_t)((c >> 1) & 1));
                if (!stage_ready) {
                    s_abort = 1;
                    aborted = true;
                }
            }
            const int tc = tlo + c * TK;
            const int lo = max(tc, s0), hi = min(tc + TK - 1, s1);
            if (lo <= hi) {
                const int qlo = s_box[st][0], rlo = s_box[st][1];
                bool in_box = stage_ready && s_box[st][2] != 0 && sr == 1;
                if (in_box) {
                    // the ray's own cells at the chunk ends (monotone in t)
                    int qa = (int)floorf(__fmaf_rn(R.bq, (float)lo, R.aq));
                    int qb = (int)floorf(__fmaf_rn(R.bq, (float)hi, R.aq));
                    int ra = (int)floorf(__fmaf_rn(R.br, (float)lo, R.ar));
                    int rb = (int)floorf(__fmaf_rn(R.br, (float)hi, R.ar));
                    in_box = min(qa, qb) >= qlo && max(qa, qb) + 1 <= qlo + TQ - 1 &&
                             min(ra, rb) >= rlo && max(ra, rb) + 1 <= rlo + TR - 1;
                }
                if (in_box)
                    acc += (px == 0) ? staged_span<0>(R, tsm + st * TSTAGE, qlo, rlo, tc, lo, hi)
                                     : staged_span<1>(R, tsm + st * TSTAGE, qlo, rlo, tc, lo, hi);
                else if (sr == 1)
                    acc += linear_span_r1(R, a.vol, (uint32_t)sp, (uint32_t)sq, lo, hi);
                else
                    acc += linear_span<false>(R, a.vol, sp, sq, sr, lo, hi);
            }
            __syncthreads();
            if (s_abort) aborted = true;
            if (tid == 0 && !aborted && c + 2 < nchunks) {
                const int c2 = c + 2;
                issue_chunk(s_corner, px, tlo + c2 * TK, min(tlo + c2 * TK + TK - 1, thi), s_box,
                            st, &mbar[st], tsm + st * TSTAGE, mx, my);
                last_issued[st] = c2;
            }
        }
        if (tid == 0 && aborted) {
            for (int sidx = 0; sidx < 2; sidx++)
                if (last_issued[sidx] >= 0)
                    mbar_wait(&mbar[sidx], (uint32_t)((last_issued[sidx] >> 1) & 1));
        }
    } else if (s0 <= s1) {
        if (sr == 1 && a.G.small)
            acc += linear_span_r1(R, a.vol, (uint32_t)sp, (uint32_t)sq, s0, s1);
        else
            acc += linear_span<false>(R, a.vol, sp, sq, sr, s0, s1);
    }
    if (!in_det) return;
    if (!on) {
        a.out[r] = 0.f;
        return;
    }
    const float s = acc * R.tvl;
    if (EMRATIO) {
        const float raysum = (s < a.em_small) ? 1.0f : s;
        a.out[r] = __fdiv_rn(a.y[r], raysum);
    } else {
        a.out[r] = s;
    }
}

template <bool EMRATIO>
__global__ void __launch_bounds__(256) k_project_tma(ProjectArgs a,
                                                     const __grid_constant__ CUtensorMap mapx,
                                                     const __grid_constant__ CUtensorMap mapy)
{
    project_tma_tile<EMRATIO>(a, &mapx, &mapy, blockIdx.x, blockIdx.y, false);
}

// Next work item of a batched launch: thread 0 takes it from the launch's
// counter, the CTA reads it after a barrier (so every thread is also done
// with the previous item).
__device__ __forceinline__ long long next_item(unsigned long long* counter)
{
    __shared__ long long s_item;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) s_item = (long long)atomicAdd(counter, 1ull);
    __syncthreads();
    return s_item;
}

// The TMA-staged projector (or EM ratio) over several jobs: items are (job,
// view, tile) as in k_project_batch, each CTA takes items from the counter
// until none are left; a job's tensor maps live in its descriptor.
template <bool EMRATIO>
__global__ void __launch_bounds__(256, 4) k_project_tma_batch(const ProjectJob* __restrict__ jobs,
                                                           int njobs, long long total,
                                                           unsigned long long* counter)
{
    bool reinit = false;
    int fenced = -1;  // the job whose maps thread 0 last fenced
    for (long long it = next_item(counter); it < total; it = next_item(counter)) {
        int j = 0;
        while (j + 1 < njobs && jobs[j + 1].item0 <= it) j++;
        const ProjectJob& J = jobs[j];
        // thread 0 issues every copy of the item
        if (threadIdx.x == 0 && threadIdx.y == 0 && j != fenced) {
            tensormap_acquire(&J.mapx);
            tensormap_acquire(&J.mapy);
            fenced = j;
        }
        const long long li = it - J.item0;
        const int tiles = ((J.a.nv + 31) >> 5) * ((J.a.nu + 7) >> 3);
        const int view = (int)(li / tiles), tile = (int)(li - (long long)view * tiles);
        project_tma_tile<EMRATIO>(J.a, &J.mapx, &J.mapy, tile, view, reinit);
        reinit = true;
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled()
{
    static const EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        EncodeTiledFn f = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            f = (EncodeTiledFn)p;
        cudaGetLastError();
        return f;
    }();
    return fn;
}

// Launches the TMA-staged projector if the volume admits tensor maps
// (16-byte aligned base and row pitch, offsets within 32 bits); returns 1 if
// it did not apply (the caller then launches k_project).
int encode_volume_maps(const ProjectArgs& a, CUtensorMap* mapx, CUtensorMap* mapy)
{
    const int nx = a.G.n[0], ny = a.G.n[1], nz = a.G.n[2];
    if (!a.G.small || nx < 2 || ny < 2 || nz < 4 || (nz % 4) != 0 ||
        (reinterpret_cast<uintptr_t>(a.vol) & 15) != 0 || a.G.s[2] != 1 ||
        a.G.s[1] != nz || a.G.s[0] != (long long)ny * nz)
        return 1;
    EncodeTiledFn enc = encode_tiled();
    if (enc == nullptr) return 1;
    // The encode resolves the base address in the calling thread's current
    // context.  A thread whose first CUDA call this is (autograd's worker, a
    // fresh host thread: cudaGetDevice binds nothing) has none, the encode
    // fails and the volume would take the untiled projector, whose sums are
    // grouped differently; binding the device's primary context first gives
    // every thread the same path and the same bits.
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaSetDevice(dev) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
    const cuuint64_t strides[2] = {(cuuint64_t)nz * 4, (cuuint64_t)ny * nz * 4};
    const cuuint32_t boxx[3] = {TR, TQ, TK}, boxy[3] = {TR, TK, TQ}, es[3] = {1, 1, 1};
    void* g = const_cast<float*>(a.vol);
    if (enc(mapx, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, g, dims, strides, boxx, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return 1;
    if (enc(mapy, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, g, dims, strides, boxy, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return 1;
    return CT2_OK;
}

template <bool EMRATIO>
static int launch_project_tma(const ProjectArgs& a, cudaStream_t st)
{
    CUtensorMap mapx, mapy;
    if (encode_volume_maps(a, &mapx, &mapy) != CT2_OK) return 1;
    CT2_CUDA(cudaFuncSetAttribute(k_project_tma<EMRATIO>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * TSTAGE_BYTES));
    const int tiles = ((a.nv + 31) / 32) * ((a.nu + 7) / 8);
    k_project_tma<EMRATIO><<<dim3(tiles, a.ns), dim3(32, 8), 2 * TSTAGE_BYTES, st>>>(a, mapx, mapy);
    CT2_LAUNCHED();
    return CT2_OK;
}

template <int MODE, bool LIST, int FORCE, bool EMRATIO>
static int launch_project(const ProjectArgs& a, cudaStream_t st)
{
    if (LIST) {
        if (a.nrays == 0) return CT2_OK;
        const long long blocks = (a.nrays + 255) / 256;
        k_project<MODE, LIST, FORCE, EMRATIO><<<dim3((unsigned)blocks), dim3(32, 8), 0, st>>>(a);
    } else {
        if (a.ns == 0 || a.nu == 0 || a.nv == 0) return CT2_OK;
        const int tiles = ((a.nv + 31) / 32) * ((a.nu + 7) / 8);
        k_project<MODE, LIST, FORCE, EMRATIO><<<dim3(tiles, a.ns), dim3(32, 8), 0, st>>>(a);
    }
    CT2_LAUNCHED();
    return CT2_OK;
}

// Self-test of the bounded wait: one thread waits, at most `spins` tries, on
// an mbarrier that expects one arrival nothing makes and that no copy
// targets; the wait runs out and *status is set to 1 (the projector's
// timeout count is left alone).
__global__ void k_wait_selftest(int spins, int* status)
{
    __shared__ __align__(8) uint64_t bar;
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const bool ok = mbar_wait_bounded(&bar, 0u, spins);
    *status = ok ? 0 : 1;
}

int wait_selftest(int spins, cudaStream_t st, int* timed_out)
{
    int* d = nullptr;
    CT2_CUDA(cudaMallocAsync((void**)&d, sizeof(int), st));
    k_wait_selftest<<<1, 1, 0, st>>>(spins, d);
    note_launch();
    cudaError_t e = cudaGetLastError();
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    CT2_CUDA(e);
    *timed_out = h;
    return CT2_OK;
}

int wait_timeouts(int* count, int reset)
{
    CT2_CUDA(cudaMemcpyFromSymbol(count, g_tma_timeouts, sizeof(int)));
    if (reset) {
        const int zero = 0;
        CT2_CUDA(cudaMemcpyToSymbol(g_tma_timeouts, &zero, sizeof(int)));
    }
    return CT2_OK;
}

int project(const ProjectArgs& a, int mode, bool list, bool force_z, bool em_ratio,
            cudaStream_t st)
{
    // Instantiate only the combinations the reference has (plus the EM ratio
    // forms of every projector the EM steps use).
    if (!list) {
        if (force_z) {
            if (mode != MODE_LINEAR) return set_error(CT2_EINVAL, "z-driven projector is linear only");
            return em_ratio ? launch_project<MODE_LINEAR, false, 2, true>(a, st)
                            : launch_project<MODE_LINEAR, false, 2, false>(a, st);
        }
        if (mode == MODE_LINEAR) {
            if (a.ns > 0 && a.nu > 0 && a.nv > 0) {
                const int rc = em_ratio ? launch_project_tma<true>(a, st)
                                        : launch_project_tma<false>(a, st);
                if (rc != 1) return rc;
            }
            return em_ratio ? launch_project<MODE_LINEAR, false, -1, true>(a, st)
                            : launch_project<MODE_LINEAR, false, -1, false>(a, st);
        }
        if (mode == MODE_NEAREST_LE)
            return em_ratio ? launch_project<MODE_NEAREST_LE, false, -1, true>(a, st)
                            : launch_project<MODE_NEAREST_LE, false, -1, false>(a, st);
        return set_error(CT2_EINVAL, "unsupported projector mode");
    }
    if (mode == MODE_LINEAR)
        return em_ratio ? launch_project<MODE_LINEAR, true, -1, true>(a, st)
                        : launch_project<MODE_LINEAR, true, -1, false>(a, st);
    if (mode == MODE_NEAREST_LE)
        return em_ratio ? launch_project<MODE_NEAREST_LE, true, -1, true>(a, st)
                        : launch_project<MODE_NEAREST_LE, true, -1, false>(a, st);
    if (mode == MODE_NEAREST_LT)
        return em_ratio ? launch_project<MODE_NEAREST_LT, true, -1, true>(a, st)
                        : launch_project<MODE_NEAREST_LT, true, -1, false>(a, st);
    return set_error(CT2_EINVAL, "unsupported projector mode");
}

template <bool EMRATIO>
static int launch_project_batch(const ProjectJob* jobs, int njobs, long long total, bool tma,
                                int grid, unsigned long long* counter, cudaStream_t st)
{
    if (tma) {
        CT2_CUDA(cudaFuncSetAttribute(k_project_tma_batch<EMRATIO>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      2 * TSTAGE_BYTES));
        k_project_tma_batch<EMRATIO><<<grid, dim3(32, 8), 2 * TSTAGE_BYTES, st>>>(
            jobs, njobs, total, counter);
    } else {
        k_project_batch<EMRATIO><<<grid, dim3(32, 8), 0, st>>>(jobs, njobs, total);
    }
    CT2_LAUNCHED();
    return CT2_OK;
}

int project_batch(const ProjectJob* jobs, int njobs, long long total, bool tma, bool em_ratio,
                  int grid, unsigned long long* counter, cudaStream_t st)
{
    if (njobs <= 0 || total <= 0) return CT2_OK;
    return em_ratio ? launch_project_batch<true>(jobs, njobs, total, tma, grid, counter, st)
                    : launch_project_batch<false>(jobs, njobs, total, tma, grid, counter, st);
}

}  // namespace ct2
