// Matched backprojectors: the exact transposes of the projectors in
// ct2_project.cu, plus the MLEM voxel update.
//
// Reference: view_proj3D.sinobackproject_linear / sinobackproject_nearest
// (emil_code/view_proj3D.f:1096-1370 / :1374-1595), the wsmat/onemat
// accumulation of emstep_linear / emstep_nearest (:2801-2827, :3045-3071),
// ray_proj3D.sinobackproject_nearest (emil_code/ray_proj3D.f:809-980).
//
// The Fortran builds each ray's (weight, voxel) list and scatters
// datum * weight into the volume.  Here a thread walks rays with the
// projector's own ray_setup / sample functions -- so every (ray, voxel)
// weight is bit-identical to the forward one and the pair is an exact
// transpose up to summation order -- and adds the taps into the volume with
// L2 reductions (red.global.add.f32).  The volume (64 MB at 256^3) stays
// largely resident in the 126 MB L2 during the pass.  In linear mode a
// thread walks two detector-adjacent rays of one column together (k_bp_pair:
// shared q arithmetic, taps on the same cell added before the reduction);
// measured on B200 at 256^3 x 360 views x 384^2, backprojecting the
// phantom's projection: 17.0 ms against 18.3 ms for one ray per lane with
// the pair merge done by shuffles, and 24.9 ms for four
// rays per thread (fewer reductions, but each warp instruction's lanes then
// spread over about twice as many cache lines, and the L1 reduction path,
// already 84 % busy, is charged per line).  16-byte vector reductions
// (red.global.add.v4.f32, zero-padded around each tap pair) were measured
// 1.7x slower: the reduction path is also charged per element.  A
// shared-memory variant that owned volume bricks per CTA and accumulated
// there was measured 9x slower (226 ms vs 24 ms): its per-(ray, brick) setup
// and block-wide barriers cost more than the L2 atomics it avoided.
#include <cstdint>

#include "ct2_common.cuh"
#include "ct2_kernels.h"
#include "ct2_scatter.cuh"

namespace ct2 {

static int num_sms()
{
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

// Per-lane scatter of one linear ray whose exact interval [R.t0, R.t1] and
// unclamped part [s0, s1] are known.
template <bool TWO>
__device__ __forceinline__ void scatter_linear_interval(const BackprojectArgs& a, const Ray& R,
                                                        float y, int s0, int s1)
{
    const Grid& G = a.G;
    const long long sp = sel3l(R.p, G.s[0], G.s[1], G.s[2]);
    const int sq = (int)sel3l(R.q, G.s[0], G.s[1], G.s[2]);
    const int sr = (int)sel3l(R.r, G.s[0], G.s[1], G.s[2]);
    const float c = y * R.tvl, c1 = R.tvl;
    if (R.t0 > R.t1) return;
    if (s0 > s1) {
        linear_scatter_span<true, TWO>(R, a.out, a.out_ones, sp, sq, sr, R.t0, R.t1, c, c1);
    } else {
        linear_scatter_span<true, TWO>(R, a.out, a.out_ones, sp, sq, sr, R.t0, s0 - 1, c, c1);
        linear_scatter_span<false, TWO>(R, a.out, a.out_ones, sp, sq, sr, s0, s1, c, c1);
        linear_scatter_span<true, TWO>(R, a.out, a.out_ones, sp, sq, sr, s1 + 1, R.t1, c, c1);
    }
}

// Scatter datum y of one ray into the volume(s): the exact transpose of
// ray_sum in ct2_project.cu (same interval, same cells, same weights).
template <int MODE, bool TWO>
__device__ __forceinline__ void scatter_ray(const BackprojectArgs& a, Ray R, float y)
{
    const Grid& G = a.G;
    const long long sp = sel3l(R.p, G.s[0], G.s[1], G.s[2]);
    const int sq = (int)sel3l(R.q, G.s[0], G.s[1], G.s[2]);
    const int sr = (int)sel3l(R.r, G.s[0], G.s[1], G.s[2]);
    const float c = y * R.tvl, c1 = R.tvl;
    if constexpr (MODE == MODE_LINEAR) {
        int s0, s1;
        exact_interval(R, R.np, &s0, &s1);
        if (R.t0 > R.t1) return;
        if (s0 > s1) {
            linear_scatter_span<true, TWO>(R, a.out, a.out_ones, sp, sq, sr, R.t0, R.t1, c, c1);
        } else {
            linear_scatter_span<true, TWO>(R, a.out, a.out_ones, sp, sq, sr, R.t0, s0 - 1, c, c1);
            linear_scatter_span<false, TWO>(R, a.out, a.out_ones, sp, sq, sr, s0, s1, c, c1);
            linear_scatter_span<true, TWO>(R, a.out, a.out_ones, sp, sq, sr, s1 + 1, R.t1, c, c1);
        }
    } else {
        for (int t = R.t0; t <= R.t1; t++) {
            int iq, ir;
            if (!sample_nearest(R, t, MODE, iq, ir)) continue;
            const long long idx = (long long)t * sp + iq * sq + ir * sr;
            atomicAdd(a.out + idx, c);
            if (TWO) atomicAdd(a.out_ones + idx, c1);
        }
    }
}

// View geometry, nearest modes: one thread per ray (the projector's
// mapping: a warp is 32 consecutive detector pixels along v of one view).
template <int MODE, int FORCE, bool TWO>
__global__ void __launch_bounds__(256) k_bp_ray(BackprojectArgs a)
{
    static_assert(MODE != MODE_LINEAR, "linear mode runs k_bp_pair");
    const int tiles_v = (a.nv + 31) >> 5;
    const int tu = blockIdx.x / tiles_v, tv = blockIdx.x - tu * tiles_v;
    const int kv = tv * 32 + threadIdx.x, ju = tu * 8 + threadIdx.y;
    const int view = blockIdx.y;
    if (ju >= a.nu || kv >= a.nv) return;
    const long long r = ((long long)view * a.nu + ju) * a.nv + kv;
    if (a.ind != nullptr && a.ind[r] != 1) return;
    const float y = a.sino[r];
    if (!TWO && y == 0.f) return;
    float f[18];
#pragma unroll
    for (int i = 0; i < 18; i++) f[i] = __ldg(a.geom + 18 * view + i);
    const float S[3] = {f[0], f[1], f[2]};
    float B[3];
    view_bin(f, ju, kv, a.du, a.dv, a.u0, a.v0, B);
    scatter_ray<MODE, TWO>(a, ray_setup(a.G, S, B, FORCE, MODE), y);
}

template <int MODE, int FORCE, bool TWO>
static int launch_ray(const BackprojectArgs& a, cudaStream_t st)
{
    if (a.ns == 0 || a.nu == 0 || a.nv == 0) return CT2_OK;
    const int tiles = ((a.nv + 31) / 32) * ((a.nu + 7) / 8);
    k_bp_ray<MODE, FORCE, TWO><<<dim3(tiles, a.ns), dim3(32, 8), 0, st>>>(a);
    CT2_LAUNCHED();
    return CT2_OK;
}

// View geometry, linear mode, two rays per thread: detector pixels kv and
// kv+1 of one column (a warp covers 64 consecutive pixels along v).  When the
// two rays share the driving axis and the q model -- every column of the
// circular cone beam -- pair_scatter_column walks them together; otherwise
// each ray goes through the single-ray scatter.  No instruction below
// exchanges data between lanes, so lanes may leave early.  Three CTAs per SM
// (80 registers, a few bytes spilled): on a variant of this walk, two CTAs
// at 96 registers and no spills measured 6 % slower.
template <int FORCE, bool TWO>
__global__ void __launch_bounds__(256, 3) k_bp_pair(BackprojectArgs a)
{
    const int tiles_v = (a.nv + 63) >> 6;
    const int tu = blockIdx.x / tiles_v, tv = blockIdx.x - tu * tiles_v;
    const int kv0 = tv * 64 + 2 * threadIdx.x, ju = tu * 8 + threadIdx.y;
    const int view = blockIdx.y;
    if (ju >= a.nu || kv0 >= a.nv) return;
    const bool has1 = kv0 + 1 < a.nv;
    const long long r0 = ((long long)view * a.nu + ju) * a.nv + kv0;
    const bool on0 = a.ind == nullptr || a.ind[r0] == 1;
    const bool on1 = has1 && (a.ind == nullptr || a.ind[r0 + 1] == 1);
    const float y0 = on0 ? a.sino[r0] : 0.f;
    const float y1 = on1 ? a.sino[r0 + 1] : 0.f;
    const bool want0 = on0 && (TWO || y0 != 0.f), want1 = on1 && (TWO || y1 != 0.f);
    if (!want0 && !want1) return;
    float f[18];
#pragma unroll
    for (int i = 0; i < 18; i++) f[i] = __ldg(a.geom + 18 * view + i);
    const float S[3] = {f[0], f[1], f[2]};
    float B0[3], B1[3];
    view_bin(f, ju, kv0, a.du, a.dv, a.u0, a.v0, B0);
    view_bin(f, ju, kv0 + 1, a.du, a.dv, a.u0, a.v0, B1);
    Ray Ra = ray_setup(a.G, S, B0, FORCE, MODE_LINEAR);
    Ray Rb = ray_setup(a.G, S, B1, FORCE, MODE_LINEAR);
    int sa0 = 0, sa1 = -1, sb0 = 0, sb1 = -1;
    if (want0) exact_interval(Ra, Ra.np, &sa0, &sa1);
    if (want1) exact_interval(Rb, Rb.np, &sb0, &sb1);
    const bool same = (Ra.p == Rb.p) && (__float_as_int(Ra.aq) == __float_as_int(Rb.aq)) &&
                      (__float_as_int(Ra.bq) == __float_as_int(Rb.bq));
    if (!same) {
        if (want0) scatter_linear_interval<TWO>(a, Ra, y0, sa0, sa1);
        if (want1) scatter_linear_interval<TWO>(a, Rb, y1, sb0, sb1);
        return;
    }
    if (!want0) {
        Ra.t0 = Ra.np;
        Ra.t1 = -1;
    }
    if (!want1) {
        Rb.t0 = Rb.np;
        Rb.t1 = -1;
    }
    const Grid& G = a.G;
    const long long sp = sel3l(Ra.p, G.s[0], G.s[1], G.s[2]);
    const int sq = (int)sel3l(Ra.q, G.s[0], G.s[1], G.s[2]);
    const int sr = (int)sel3l(Ra.r, G.s[0], G.s[1], G.s[2]);
    const float c0 = y0 * Ra.tvl, c1 = y1 * Rb.tvl;
    if (sr == 1 && G.small)
        pair_scatter_column<TWO, true>(Ra, Rb, a.out, a.out_ones, sp, sq, sr, c0, c1, Ra.tvl,
                                       Rb.tvl);
    else
        pair_scatter_column<TWO, false>(Ra, Rb, a.out, a.out_ones, sp, sq, sr, c0, c1, Ra.tvl,
                                        Rb.tvl);
}

template <int FORCE, bool TWO>
static int launch_pair(const BackprojectArgs& a, cudaStream_t st)
{
    if (a.ns == 0 || a.nu == 0 || a.nv == 0) return CT2_OK;
    const int tiles = ((a.nv + 63) / 64) * ((a.nu + 7) / 8);
    k_bp_pair<FORCE, TWO><<<dim3(tiles, a.ns), dim3(32, 8), 0, st>>>(a);
    CT2_LAUNCHED();
    return CT2_OK;
}

// Ray-list geometry: one thread per ray.
template <int MODE, bool TWO>
__global__ void __launch_bounds__(256) k_bp_list(BackprojectArgs a)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nrays) return;
    if (a.ind != nullptr && a.ind[r] != 1) return;
    const float y = a.sino[r];
    if (!TWO && y == 0.f) return;
    const float* v = a.geom + 6 * r;
    const float S[3] = {v[0], v[1], v[2]};
    const float B[3] = {v[3], v[4], v[5]};
    scatter_ray<MODE, TWO>(a, ray_setup(a.G, S, B, -1, MODE), y);
}

template <int MODE, bool TWO>
static int launch_list(const BackprojectArgs& a, cudaStream_t st)
{
    if (a.nrays == 0) return CT2_OK;
    k_bp_list<MODE, TWO><<<(unsigned)((a.nrays + 255) / 256), 256, 0, st>>>(a);
    CT2_LAUNCHED();
    return CT2_OK;
}

int backproject(const BackprojectArgs& a, int mode, bool list, bool force_z, cudaStream_t st)
{
    const bool two = a.out_ones != nullptr;
    if (list) {
        if (mode == MODE_LINEAR)
            return two ? launch_list<MODE_LINEAR, true>(a, st) : launch_list<MODE_LINEAR, false>(a, st);
        if (mode == MODE_NEAREST_LE)
            return two ? launch_list<MODE_NEAREST_LE, true>(a, st)
                       : launch_list<MODE_NEAREST_LE, false>(a, st);
        if (mode == MODE_NEAREST_LT)
            return two ? launch_list<MODE_NEAREST_LT, true>(a, st)
                       : launch_list<MODE_NEAREST_LT, false>(a, st);
        return set_error(CT2_EINVAL, "unsupported backprojector mode");
    }
    if (force_z) {
        if (mode != MODE_LINEAR) return set_error(CT2_EINVAL, "z-driven backprojector is linear only");
        return two ? launch_pair<2, true>(a, st) : launch_pair<2, false>(a, st);
    }
    if (mode == MODE_LINEAR) {
        const int rc = backproject_gather(a, st);
        if (rc != 1) return rc;
        return two ? launch_pair<-1, true>(a, st) : launch_pair<-1, false>(a, st);
    }
    if (mode == MODE_NEAREST_LE)
        return two ? launch_ray<MODE_NEAREST_LE, -1, true>(a, st)
                   : launch_ray<MODE_NEAREST_LE, -1, false>(a, st);
    return set_error(CT2_EINVAL, "unsupported backprojector mode");
}

__global__ void k_em_update(float* __restrict__ x, const float* __restrict__ ws,
                            const float* __restrict__ ones, long long n, float small)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float o = ones[i];
        if (o < small) o = 1.0f;
        x[i] = __fdiv_rn(__fmul_rn(x[i], ws[i]), o);
    }
}

int em_update(float* x, const float* ws, const float* ones, long long n, float small,
              cudaStream_t st)
{
    if (n == 0) return CT2_OK;
    long long blocks = (n + 255) / 256;
    const long long cap = (long long)num_sms() * 16;
    if (blocks > cap) blocks = cap;
    k_em_update<<<(unsigned)blocks, 256, 0, st>>>(x, ws, ones, n, small);
    CT2_LAUNCHED();
    return CT2_OK;
}

}  // namespace ct2
