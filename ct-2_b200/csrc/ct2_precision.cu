// Precision form of the Joseph projector pair and the EM+TV step.
//
// Storage: volumes in BF16, sinograms (data, projections, EM ratios) in FP16;
// FP16 volumes (three more mantissa bits than BF16, for iterations that make
// many small in-place updates such as ART) and FP32 storage (which isolates
// the arithmetic from the storage rounding) run through the same kernels.  Arithmetic: per-ray geometry in FP64 -- source and detector bin,
// direction, driving axis, slopes, travelled length and the sample model --
// so nothing cancels in FP32 at large source-detector distances; bilinear
// taps and lerps in FP32; every ray sum accumulated in FP32 with Kahan
// compensation; the EM+TV norms (||x_EM - x||, ||g||) in FP64 in a fixed order.
//
// The algorithm is the reference's linear Joseph projector and its matched
// backprojector (emil_code/view_proj3D.f:703-910, :1096-1370; z-driven form
// emil_code/view_proj3D_tomo.f:4-148) and the MLEM update of emstep_linear
// (:2801-2827), computed at this precision instead of the Fortran's REAL*4
// setup; its oracle is the FP64 restatement of the same algorithm.
//
// Sample set.  Slice t is taken iff its FP32 model coordinates
// fq = fma(bq, t, aq), fr = fma(br, t, ar) satisfy 0 <= fq < nq-1 and
// 0 <= fr < nr-1 (the interior-cell test of the linear mode).  Each is
// monotone in t, so the set is one interval, found once per ray; the
// projector and the backprojector evaluate the same model, so they take the
// same samples with the same weights and are exact transposes up to the
// order of the FP32 additions.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>

#include "ct2_common.cuh"
#include "ct2_pray.cuh"
#include "ct2_precision.h"
#include "ct2_scatter.cuh"
#include "ct2_tv.cuh"

namespace ct2 {

static int prec_num_sms()
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

template <typename T>
__device__ __forceinline__ float ld_f(const T* p);
template <>
__device__ __forceinline__ float ld_f<float>(const float* p)
{
    return __ldg(p);
}
template <>
__device__ __forceinline__ float ld_f<__nv_bfloat16>(const __nv_bfloat16* p)
{
    return __bfloat162float(__ldg(p));
}
template <>
__device__ __forceinline__ float ld_f<__half>(const __half* p)
{
    return __half2float(__ldg(p));
}

template <typename T>
__device__ __forceinline__ T st_f(float v);
template <>
__device__ __forceinline__ float st_f<float>(float v)
{
    return v;
}
template <>
__device__ __forceinline__ __nv_bfloat16 st_f<__nv_bfloat16>(float v)
{
    return __float2bfloat16_rn(v);
}
template <>
__device__ __forceinline__ __half st_f<__half>(float v)
{
    return __float2half_rn(v);
}

// Kahan-compensated FP32 sum of the bilinear samples over [R.t0, R.t1].
template <typename VT>
__device__ __forceinline__ float kahan_span(const Ray& R, const VT* __restrict__ vol, long long sp,
                                            int sq, int sr)
{
    float acc = 0.f, comp = 0.f;
    const VT* plane = vol + (long long)R.t0 * sp;
    float tf = (float)R.t0;
#pragma unroll 2
    for (int t = R.t0; t <= R.t1; t++, tf += 1.0f, plane += sp) {
        int iq, ir;
        float wq2, wr2;
        sample_in<false>(R, tf, iq, ir, wq2, wr2);
        const VT* b = plane + (iq * sq + ir * sr);
        const float v00 = ld_f(b), v10 = ld_f(b + sq);
        const float v01 = ld_f(b + sr), v11 = ld_f(b + sq + sr);
        const float vi1 = __fmaf_rn(wq2, v10 - v00, v00);
        const float vi2 = __fmaf_rn(wq2, v11 - v01, v01);
        const float v = __fmaf_rn(wr2, vi2 - vi1, vi1);
        const float yk = __fsub_rn(v, comp);
        const float tk = __fadd_rn(acc, yk);
        comp = __fsub_rn(__fsub_rn(tk, acc), yk);
        acc = tk;
    }
    return acc;
}

// One bilinear sample of slice t for kahan_span_r1 (r stride 1, 32-bit
// offsets): coordinates, floor and weights of q and r in f32x2 instructions.
// Every t of the ray's interval is interior (0 <= fq < nq-1, 0 <= fr < nr-1
// for this same fma), so the floor needs no clamp.
template <typename VT>
__device__ __forceinline__ float sample_r1(const VT* __restrict__ vol, const VT* __restrict__ volq,
                                           uint64_t A, uint64_t B, uint64_t T, uint32_t sq,
                                           uint32_t base)
{
    const uint64_t M = f2_pack(12582912.0f, 12582912.0f);
    const uint64_t f = f2_fma(B, T, A);
    const uint64_t tt = f2_add_rd(f, M);
    float tq, tr, wq2, wr2;
    f2_unpack(tt, tq, tr);
    f2_unpack(f2_sub(f, f2_sub(tt, M)), wq2, wr2);
    const uint32_t off = __float_as_uint(tq) * sq + __float_as_uint(tr) + base;
    const float v00 = ld_f(vol + off), v01 = ld_f(vol + off + 1);
    const float v10 = ld_f(volq + off), v11 = ld_f(volq + off + 1);
    const uint64_t lo = f2_pack(v00, v01);
    float vi1, vi2;
    f2_unpack(f2_fma(f2_pack(wq2, wq2), f2_sub(f2_pack(v10, v11), lo), lo), vi1, vi2);
    return __fmaf_rn(wr2, vi2 - vi1, vi1);
}

// kahan_span for a ray whose r axis has stride 1 in a volume with 32-bit
// offsets: packed sample arithmetic, and the compensation applied to blocks
// of four samples (each block summed in FP32, the block sums Kahan-added),
// which keeps the compensated error bound along the ray at a third of the
// per-sample cost.
template <typename VT>
__device__ __forceinline__ float kahan_span_r1(const Ray& R, const VT* __restrict__ vol,
                                               uint32_t sp, uint32_t sq)
{
    const uint64_t A = f2_pack(R.aq, R.ar), B = f2_pack(R.bq, R.br);
    const uint64_t ONE = f2_pack(1.0f, 1.0f);
    const VT* __restrict__ volq = vol + sq;
    uint64_t T = f2_pack((float)R.t0, (float)R.t0);
    uint32_t base = (uint32_t)R.t0 * sp - 0x4B400000u * (sq + 1u);
    float acc = 0.f, comp = 0.f;
    int t = R.t0;
    for (; t + 3 <= R.t1; t += 4) {
        const float s0 = sample_r1(vol, volq, A, B, T, sq, base);
        T = f2_add(T, ONE);
        const float s1 = sample_r1(vol, volq, A, B, T, sq, base + sp);
        T = f2_add(T, ONE);
        const float s2 = sample_r1(vol, volq, A, B, T, sq, base + 2 * sp);
        T = f2_add(T, ONE);
        const float s3 = sample_r1(vol, volq, A, B, T, sq, base + 3 * sp);
        T = f2_add(T, ONE);
        base += 4 * sp;
        const float blk = (s0 + s1) + (s2 + s3);
        const float yk = __fsub_rn(blk, comp);
        const float tk = __fadd_rn(acc, yk);
        comp = __fsub_rn(__fsub_rn(tk, acc), yk);
        acc = tk;
    }
    for (; t <= R.t1; t++) {
        const float v = sample_r1(vol, volq, A, B, T, sq, base);
        T = f2_add(T, ONE);
        base += sp;
        const float yk = __fsub_rn(v, comp);
        const float tk = __fadd_rn(acc, yk);
        comp = __fsub_rn(__fsub_rn(tk, acc), yk);
        acc = tk;
    }
    return acc;
}

// The two taps of a z-pair word as FP32.
template <typename VT>
__device__ __forceinline__ void pair_to_f(uint32_t w, float& lo, float& hi)
{
    if constexpr (std::is_same<VT, __half>::value) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w));
        lo = f.x;
        hi = f.y;
    } else {
        lo = __uint_as_float(w << 16);
        hi = __uint_as_float(w & 0xFFFF0000u);
    }
}

// kahan_span_r1 reading the z-pair words: two aligned 4-byte loads per sample.
template <typename VT>
__device__ __forceinline__ float sample_pairs(const uint32_t* __restrict__ pv,
                                              const uint32_t* __restrict__ pq, uint64_t A,
                                              uint64_t B, uint64_t T, uint32_t sq, uint32_t base)
{
    const uint64_t M = f2_pack(12582912.0f, 12582912.0f);
    const uint64_t f = f2_fma(B, T, A);
    const uint64_t tt = f2_add_rd(f, M);
    float tq, tr, wq2, wr2;
    f2_unpack(tt, tq, tr);
    f2_unpack(f2_sub(f, f2_sub(tt, M)), wq2, wr2);
    const uint32_t off = __float_as_uint(tq) * sq + __float_as_uint(tr) + base;
    float v00, v01, v10, v11;
    pair_to_f<VT>(__ldg(pv + off), v00, v01);
    pair_to_f<VT>(__ldg(pq + off), v10, v11);
    const uint64_t lo = f2_pack(v00, v01);
    float vi1, vi2;
    f2_unpack(f2_fma(f2_pack(wq2, wq2), f2_sub(f2_pack(v10, v11), lo), lo), vi1, vi2);
    return __fmaf_rn(wr2, vi2 - vi1, vi1);
}

template <typename VT>
__device__ __forceinline__ float kahan_span_pairs(const Ray& R, const uint32_t* __restrict__ pairs,
                                                  uint32_t sp, uint32_t sq)
{
    const uint64_t A = f2_pack(R.aq, R.ar), B = f2_pack(R.bq, R.br);
    const uint64_t ONE = f2_pack(1.0f, 1.0f);
    const uint32_t* __restrict__ pq = pairs + sq;
    uint64_t T = f2_pack((float)R.t0, (float)R.t0);
    uint32_t base = (uint32_t)R.t0 * sp - 0x4B400000u * (sq + 1u);
    float acc = 0.f, comp = 0.f;
    int t = R.t0;
    for (; t + 3 <= R.t1; t += 4) {
        const float s0 = sample_pairs<VT>(pairs, pq, A, B, T, sq, base);
        T = f2_add(T, ONE);
        const float s1 = sample_pairs<VT>(pairs, pq, A, B, T, sq, base + sp);
        T = f2_add(T, ONE);
        const float s2 = sample_pairs<VT>(pairs, pq, A, B, T, sq, base + 2 * sp);
        T = f2_add(T, ONE);
        const float s3 = sample_pairs<VT>(pairs, pq, A, B, T, sq, base + 3 * sp);
        T = f2_add(T, ONE);
        base += 4 * sp;
        const float blk = (s0 + s1) + (s2 + s3);
        const float yk = __fsub_rn(blk, comp);
        const float tk = __fadd_rn(acc, yk);
        comp = __fsub_rn(__fsub_rn(tk, acc), yk);
        acc = tk;
    }
    for (; t <= R.t1; t++) {
        const float v = sample_pairs<VT>(pairs, pq, A, B, T, sq, base);
        T = f2_add(T, ONE);
        base += sp;
        const float yk = __fsub_rn(v, comp);
        const float tk = __fadd_rn(acc, yk);
        comp = __fsub_rn(__fsub_rn(tk, acc), yk);
        acc = tk;
    }
    return acc;
}

template <typename VT>
__global__ void k_make_pairs(const VT* __restrict__ v, uint32_t* __restrict__ pairs, long long n,
                             int nz)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const uint32_t lo = *reinterpret_cast<const uint16_t*>(v + i);
        const bool last = (i % nz) == nz - 1;
        const uint32_t hi = last ? 0u : *reinterpret_cast<const uint16_t*>(v + i + 1);
        pairs[i] = lo | (hi << 16);
    }
}

int prec_make_pairs(const void* vol, int vol_type, uint32_t* pairs, long long n, int nz,
                    cudaStream_t st)
{
    if (n == 0) return CT2_OK;
    long long blocks = (n + 255) / 256;
    const long long cap = (long long)prec_num_sms() * 16;
    if (blocks > cap) blocks = cap;
    if (vol_type == ST_BF16)
        k_make_pairs<__nv_bfloat16><<<(unsigned)blocks, 256, 0, st>>>(
            (const __nv_bfloat16*)vol, pairs, n, nz);
    else if (vol_type == ST_F16)
        k_make_pairs<__half><<<(unsigned)blocks, 256, 0, st>>>((const __half*)vol, pairs, n, nz);
    else
        return set_error(CT2_EINVAL, "z-pair words are for 16-bit volumes");
    CT2_LAUNCHED();
    return CT2_OK;
}

// A x, or y / (Ax < small ? 1 : Ax) (the reference's EM clamp), one thread per
// ray, CTA = 32 v x 8 u of one view (the reference-parity projector's mapping).
template <typename VT, typename ST, bool EMRATIO, int FORCE>
__global__ void __launch_bounds__(256) k_pproject(PrecProjectArgs a)
{
    const int tiles_v = (a.nv + 31) >> 5;
    const int tu = blockIdx.x / tiles_v, tv = blockIdx.x - tu * tiles_v;
    const int kv = tv * 32 + threadIdx.x, ju = tu * 8 + threadIdx.y;
    const int view = blockIdx.y;
    if (kv >= a.nv || ju >= a.nu) return;
    const long long r = ((long long)view * a.nu + ju) * a.nv + kv;
    ST* out = (ST*)a.out;
    if (a.ind != nullptr && a.ind[r] != 1) {
        out[r] = st_f<ST>(0.f);
        return;
    }
    const Ray R = pray_view(a.G, a.geom + 18 * view, ju, kv, a.du, a.dv, a.u0, a.v0, FORCE);
    const long long sp = sel3l(R.p, a.G.s[0], a.G.s[1], a.G.s[2]);
    const int sq = (int)sel3l(R.q, a.G.s[0], a.G.s[1], a.G.s[2]);
    const int sr = (int)sel3l(R.r, a.G.s[0], a.G.s[1], a.G.s[2]);
    float s = 0.f;
    if (R.t0 <= R.t1) {
        const bool r1 = (sr == 1) && a.G.small;
        if (sizeof(VT) == 2 && r1 && a.pairs != nullptr)
            s = kahan_span_pairs<VT>(R, a.pairs, (uint32_t)sp, (uint32_t)sq) * R.tvl;
        else if (r1)
            s = kahan_span_r1<VT>(R, (const VT*)a.vol, (uint32_t)sp, (uint32_t)sq) * R.tvl;
        else
            s = kahan_span<VT>(R, (const VT*)a.vol, sp, sq, sr) * R.tvl;
    }
    if (EMRATIO) {
        const float yv = ld_f<ST>((const ST*)a.y + r);
        const float raysum = (s < a.em_small) ? 1.0f : s;
        out[r] = st_f<ST>(__fdiv_rn(yv, raysum));
    } else {
        out[r] = st_f<ST>(s);
    }
}

template <typename VT, typename ST, bool EMRATIO, int FORCE>
static int launch_pproject(const PrecProjectArgs& a, cudaStream_t st)
{
    if (a.ns == 0 || a.nu == 0 || a.nv == 0) return CT2_OK;
    const int tiles = ((a.nv + 31) / 32) * ((a.nu + 7) / 8);
    k_pproject<VT, ST, EMRATIO, FORCE><<<dim3(tiles, a.ns), dim3(32, 8), 0, st>>>(a);
    CT2_LAUNCHED();
    return CT2_OK;
}

template <typename VT, typename ST>
static int pproject_types(const PrecProjectArgs& a, bool force_z, cudaStream_t st)
{
    const bool em = a.y != nullptr;
    if (force_z)
        return em ? launch_pproject<VT, ST, true, 2>(a, st) : launch_pproject<VT, ST, false, 2>(a, st);
    return em ? launch_pproject<VT, ST, true, -1>(a, st) : launch_pproject<VT, ST, false, -1>(a, st);
}

int prec_project(const PrecProjectArgs& a, bool force_z, cudaStream_t st)
{
    if (a.vol_type == ST_BF16 && a.sino_type == ST_F16)
        return pproject_types<__nv_bfloat16, __half>(a, force_z, st);
    if (a.vol_type == ST_F16 && a.sino_type == ST_F16)
        return pproject_types<__half, __half>(a, force_z, st);
    if (a.vol_type == ST_F32 && a.sino_type == ST_F32)
        return pproject_types<float, float>(a, force_z, st);
    return set_error(CT2_EINVAL,
                     "precision form: (volume, sinogram) types must be (bf16, f16), (f16, f16) or (f32, f32)");
}

// Matched backprojector: the projector's rays, samples and weights, taps sent
// to the FP32 accumulators as L2 reductions.  Two rays per thread (detector
// pixels kv and kv+1 of one column; a warp covers 64 pixels along v): rays
// that share the driving axis and the q model walk together through
// pair_scatter_column, others one by one.  No instruction exchanges data
// between lanes.
template <typename ST, int FORCE, bool TWO>
__global__ void __launch_bounds__(256, 3) k_pbackproject(PrecBackprojectArgs a)
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
    const float y0 = on0 ? ld_f<ST>((const ST*)a.sino + r0) : 0.f;
    const float y1 = on1 ? ld_f<ST>((const ST*)a.sino + r0 + 1) : 0.f;
    const bool want0 = on0 && (TWO || y0 != 0.f), want1 = on1 && (TWO || y1 != 0.f);
    if (!want0 && !want1) return;
    Ray Ra = pray_view(a.G, a.geom + 18 * view, ju, kv0, a.du, a.dv, a.u0, a.v0, FORCE);
    Ray Rb = pray_view(a.G, a.geom + 18 * view, ju, kv0 + 1, a.du, a.dv, a.u0, a.v0, FORCE);
    const long long sp = sel3l(Ra.p, a.G.s[0], a.G.s[1], a.G.s[2]);
    const int sq = (int)sel3l(Ra.q, a.G.s[0], a.G.s[1], a.G.s[2]);
    const int sr = (int)sel3l(Ra.r, a.G.s[0], a.G.s[1], a.G.s[2]);
    const bool same = (Ra.p == Rb.p) && (__float_as_int(Ra.aq) == __float_as_int(Rb.aq)) &&
                      (__float_as_int(Ra.bq) == __float_as_int(Rb.bq));
    if (!same) {
        if (want0)
            linear_scatter_span<false, TWO>(Ra, a.out, a.out_ones, sp, sq, sr, Ra.t0, Ra.t1,
                                            y0 * Ra.tvl, Ra.tvl);
        if (want1) {
            const long long spb = sel3l(Rb.p, a.G.s[0], a.G.s[1], a.G.s[2]);
            const int sqb = (int)sel3l(Rb.q, a.G.s[0], a.G.s[1], a.G.s[2]);
            const int srb = (int)sel3l(Rb.r, a.G.s[0], a.G.s[1], a.G.s[2]);
            linear_scatter_span<false, TWO>(Rb, a.out, a.out_ones, spb, sqb, srb, Rb.t0, Rb.t1,
                                            y1 * Rb.tvl, Rb.tvl);
        }
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
    const float c0 = y0 * Ra.tvl, c1 = y1 * Rb.tvl;
    if (sr == 1 && a.G.small)
        pair_scatter_column<TWO, true>(Ra, Rb, a.out, a.out_ones, sp, sq, sr, c0, c1, Ra.tvl,
                                       Rb.tvl);
    else
        pair_scatter_column<TWO, false>(Ra, Rb, a.out, a.out_ones, sp, sq, sr, c0, c1, Ra.tvl,
                                        Rb.tvl);
}

template <typename ST, int FORCE, bool TWO>
static int launch_pbackproject(const PrecBackprojectArgs& a, cudaStream_t st)
{
    if (a.ns == 0 || a.nu == 0 || a.nv == 0) return CT2_OK;
    const int tiles = ((a.nv + 63) / 64) * ((a.nu + 7) / 8);
    k_pbackproject<ST, FORCE, TWO><<<dim3(tiles, a.ns), dim3(32, 8), 0, st>>>(a);
    CT2_LAUNCHED();
    return CT2_OK;
}

template <typename ST>
static int pbackproject_type(const PrecBackprojectArgs& a, bool force_z, cudaStream_t st)
{
    const bool two = a.out_ones != nullptr;
    if (force_z)
        return two ? launch_pbackproject<ST, 2, true>(a, st) : launch_pbackproject<ST, 2, false>(a, st);
    return two ? launch_pbackproject<ST, -1, true>(a, st) : launch_pbackproject<ST, -1, false>(a, st);
}

int prec_backproject(const PrecBackprojectArgs& a, bool force_z, cudaStream_t st)
{
    if (!force_z) {
        const int rc = prec_backproject_gather(a, st);
        if (rc != 1) return rc;
    }
    if (a.sino_type == ST_F16) return pbackproject_type<__half>(a, force_z, st);
    if (a.sino_type == ST_F32) return pbackproject_type<float>(a, force_z, st);
    return set_error(CT2_EINVAL, "precision form: sinogram type must be f16 or f32");
}

// ---------------------------------------------------------------------
// ART over one colour of one view
// ---------------------------------------------------------------------

template <typename VT>
__device__ __forceinline__ float ld_plain(const VT* p)
{
    if constexpr (sizeof(VT) == 4)
        return *(const float*)p;
    else if constexpr (std::is_same<VT, __half>::value)
        return __half2float(*p);
    else
        return __bfloat162float(*p);
}

// kArtLanes lanes per ray of the colour (cu0, cv0) of one view: lane l takes
// the ray's slices t0 + l, t0 + l + kArtLanes, ...; each lane keeps a Kahan
// sum of its samples and of their squared weights, the lanes add their
// partial sums, and every lane then applies
//     x += reg_fac * (y - raysum) * w / sum(w^2)
// on its own slices' taps (view_proj3D_tomo.f:154-347), each corrected tap
// rounded to nearest in the storage type.  Stochastic rounding of the
// corrections (Gupta et al., ICML 2015) was measured and dropped: on the
// full tomosynthesis slab BF16 storage ends 5.8e-2 from the FP64 oracle
// with it against 6.0e-2 without, on the small slab 1.7e-2 against 1.2e-2 --
// the drift is the random walk of ~500 roundings per voxel, which
// stochastic rounding does not shorten (it removes bias, at a larger
// variance per rounding).  No other ray of the
// colour touches those taps, and a ray's lanes update different slices, so
// plain read-modify-writes are race-free.  Splitting a ray shortens each
// lane's dependent chain and fills the GPU with more warps (one colour of
// one view is only ~90 k rays); the rays of a warp are consecutive rays of
// the colour along u (x on the slab detector), and with the volume stored
// z-major (x fastest) their taps at a slice lie a few voxels apart in one
// row.  Measured on the tomosynthesis slab (15 ART+TV iterations): 1 lane
// per ray 235 ms, 2 lanes 174 ms, 4 lanes 182 ms, 8 lanes 302 ms -- more
// lanes per ray spread a warp's loads over more z planes.
constexpr int kArtLanes = 2;

template <typename VT, typename ST>
__global__ void __launch_bounds__(128) k_part_colour(PrecArtArgs a, int view, int cu0, int cv0)
{
    constexpr int RAYS = 128 / kArtLanes;  // rays per block
    const int lr = threadIdx.x & (kArtLanes - 1);
    const int i = blockIdx.x * RAYS + (int)(threadIdx.x / kArtLanes);
    const int ju = cu0 + i * a.cu, kv = cv0 + (int)blockIdx.y * a.cv;
    // every exit below is taken by all lanes of the ray together
    if (kv >= a.nv || ju >= a.nu) return;
    const long long r = ((long long)view * a.nu + ju) * a.nv + kv;
    if (a.ind != nullptr && a.ind[r] != 1) return;
    const Ray R = pray_view(a.G, a.geom + 18 * view, ju, kv, a.du, a.dv, a.u0, a.v0, 2);
    if (R.t0 > R.t1) return;
    // this ray's lanes in the warp
    const unsigned group = ((1u << kArtLanes) - 1u) << (threadIdx.x & 31 & ~(kArtLanes - 1));
    const long long sp = sel3l(R.p, a.G.s[0], a.G.s[1], a.G.s[2]);
    const long long sq = sel3l(R.q, a.G.s[0], a.G.s[1], a.G.s[2]);
    const long long sr = sel3l(R.r, a.G.s[0], a.G.s[1], a.G.s[2]);
    VT* x = (VT*)a.x;
    float acc = 0.f, comp = 0.f, w2 = 0.f;
#pragma unroll 4
    for (int t = R.t0 + lr; t <= R.t1; t += kArtLanes) {
        int iq, ir;
        float wq2, wr2;
        sample_in<false>(R, (float)t, iq, ir, wq2, wr2);
        const VT* b = x + (t * sp + iq * sq + ir * sr);
        const float v00 = ld_plain(b), v10 = ld_plain(b + sq);
        const float v01 = ld_plain(b + sr), v11 = ld_plain(b + sq + sr);
        const float vi1 = __fmaf_rn(wq2, v10 - v00, v00);
        const float vi2 = __fmaf_rn(wq2, v11 - v01, v01);
        const float v = __fmaf_rn(wr2, vi2 - vi1, vi1);
        const float yk = __fsub_rn(v, comp);
        const float tk = __fadd_rn(acc, yk);
        comp = __fsub_rn(__fsub_rn(tk, acc), yk);
        acc = tk;
        const float wq1 = 1.0f - wq2, wr1 = 1.0f - wr2;
        const float e = wq1 * wr1, f = wq2 * wr1, g = wq1 * wr2, h = wq2 * wr2;
        w2 += e * e + f * f + g * g + h * h;
    }
    // the lanes' compensated partial sums; the butterfly gives every lane
    // the same bits
    float part = __fsub_rn(acc, comp);
#pragma unroll
    for (int o = 1; o < kArtLanes; o <<= 1) {
        part += __shfl_xor_sync(group, part, o);
        w2 += __shfl_xor_sync(group, w2, o);
    }
    const float s = part * R.tvl;
    const float ww = w2 * (R.tvl * R.tvl);
    if (!(ww > 0.f)) return;
    const float yv = ld_f<ST>((const ST*)a.y + r);
    const float coef = a.reg_fac * (yv - s) / ww * R.tvl;
    // two samples per step, both loaded before either is stored: their taps
    // lie on different slices of the driving axis, so they never overlap,
    // and the loads of the second need not wait for the stores of the first
    // (a generic batch of K samples held in small arrays compiled to slower
    // code: 126 ms against 110 ms for the slab's 15 iterations)
    for (int t = R.t0 + lr; t <= R.t1; t += 2 * kArtLanes) {
        const int u = t + kArtLanes;
        const bool two = u <= R.t1;
        int iq, ir, iq2 = 0, ir2 = 0;
        float wq2, wr2, wq22 = 0.f, wr22 = 0.f;
        sample_in<false>(R, (float)t, iq, ir, wq2, wr2);
        if (two) sample_in<false>(R, (float)u, iq2, ir2, wq22, wr22);
        VT* b = x + (t * sp + iq * sq + ir * sr);
        VT* c = two ? x + (u * sp + iq2 * sq + ir2 * sr) : b;
        const float b00 = ld_plain(b), b10 = ld_plain(b + sq), b01 = ld_plain(b + sr),
                    b11 = ld_plain(b + sq + sr);
        float c00 = 0.f, c10 = 0.f, c01 = 0.f, c11 = 0.f;
        if (two) {
            c00 = ld_plain(c);
            c10 = ld_plain(c + sq);
            c01 = ld_plain(c + sr);
            c11 = ld_plain(c + sq + sr);
        }
        const float wq1 = 1.0f - wq2, wr1 = 1.0f - wr2;
        b[0] = st_f<VT>(b00 + coef * (wq1 * wr1));
        b[sq] = st_f<VT>(b10 + coef * (wq2 * wr1));
        b[sr] = st_f<VT>(b01 + coef * (wq1 * wr2));
        b[sq + sr] = st_f<VT>(b11 + coef * (wq2 * wr2));
        if (two) {
            const float wq12 = 1.0f - wq22, wr12 = 1.0f - wr22;
            c[0] = st_f<VT>(c00 + coef * (wq12 * wr12));
            c[sq] = st_f<VT>(c10 + coef * (wq22 * wr12));
            c[sr] = st_f<VT>(c01 + coef * (wq12 * wr22));
            c[sq + sr] = st_f<VT>(c11 + coef * (wq22 * wr22));
        }
    }
}

template <typename VT, typename ST>
static int art_sweep_typed(const PrecArtArgs& a, cudaStream_t st)
{
    for (int view = 0; view < a.ns; view++) {
        for (int cu0 = 0; cu0 < a.cu && cu0 < a.nu; cu0++) {
            const int nu_c = (a.nu - cu0 + a.cu - 1) / a.cu;
            for (int cv0 = 0; cv0 < a.cv && cv0 < a.nv; cv0++) {
                const int nv_c = (a.nv - cv0 + a.cv - 1) / a.cv;
                constexpr int rays = 128 / kArtLanes;
                k_part_colour<VT, ST><<<dim3((nu_c + rays - 1) / rays, nv_c), 128, 0, st>>>(
                    a, view, cu0, cv0);
                CT2_LAUNCHED();
            }
        }
    }
    return CT2_OK;
}

int prec_art_sweep(const PrecArtArgs& a, cudaStream_t st)
{
    if (a.ns == 0 || a.nu == 0 || a.nv == 0) return CT2_OK;
    if (a.vol_type == ST_BF16 && a.sino_type == ST_F16)
        return art_sweep_typed<__nv_bfloat16, __half>(a, st);
    if (a.vol_type == ST_F16 && a.sino_type == ST_F16) return art_sweep_typed<__half, __half>(a, st);
    if (a.vol_type == ST_F32 && a.sino_type == ST_F32) return art_sweep_typed<float, float>(a, st);
    return set_error(CT2_EINVAL,
                     "precision form: (volume, sinogram) types must be (bf16, f16), (f16, f16) or (f32, f32)");
}

// ---------------------------------------------------------------------
// EM+TV step
// ---------------------------------------------------------------------

int prec_parts(long long n)
{
    long long blocks = (n + 255) / 256;
    const long long cap = (long long)prec_num_sms() * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (int)blocks;
}

// ws <- xe = x * ws / (sens < small ? 1 : sens); partial sum of (xe - x)^2.
template <typename VT>
__global__ void __launch_bounds__(256) k_pem(const VT* __restrict__ x, float* __restrict__ ws,
                                             const float* __restrict__ sens, long long n,
                                             float small, double* __restrict__ partial)
{
    __shared__ double sh[8];
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float xo = ld_f(x + i);
        float o = sens[i];
        if (o < small) o = 1.0f;
        const float xe = __fdiv_rn(__fmul_rn(xo, ws[i]), o);
        ws[i] = xe;
        const double d = (double)xe - (double)xo;
        acc += d * d;
    }
    const double t = block_sum_double(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// partial sum of g(xe)^2, g the unnormalised TV gradient (lam = 0).
__global__ void __launch_bounds__(256) k_ptv_norm(const float* __restrict__ xe, int nx, int ny,
                                                  int nz, double* __restrict__ partial)
{
    __shared__ double sh[8];
    const long long n = (long long)nx * ny * nz;
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int iz = (int)(i % nz);
        const long long rest = i / nz;
        const int iy = (int)(rest % ny), ix = (int)(rest / ny);
        const double g = (double)tv_grad_at(xe, ix, iy, iz, nx, ny, nz, 0.0f);
        acc += g * g;
    }
    const double t = block_sum_double(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// scale = w * ||xe - x|| / ||g|| (||g|| < 1e-5 -> 1, totalvar.f:576-586), FP64.
__global__ void k_ptv_scale(const double* __restrict__ partial, int parts, float w,
                            double* __restrict__ scale)
{
    __shared__ double sh[8];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < parts; i += blockDim.x) {
        a += partial[i];
        b += partial[parts + i];
    }
    const double sa = block_sum_double(a, sh);
    const double sb = block_sum_double(b, sh);
    if (threadIdx.x == 0) {
        double gn = sqrt(sb);
        if (gn < 0.00001) gn = 1.0;
        *scale = (double)w * sqrt(sa) / gn;
    }
}

// x <- max(0, xe - scale * g(xe)), rounded to the storage type.
template <typename VT>
__global__ void __launch_bounds__(256) k_ptv_apply(VT* __restrict__ x, const float* __restrict__ xe,
                                                   int nx, int ny, int nz,
                                                   const double* __restrict__ scale)
{
    const long long n = (long long)nx * ny * nz;
    const float s = (float)*scale;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int iz = (int)(i % nz);
        const long long rest = i / nz;
        const int iy = (int)(rest % ny), ix = (int)(rest / ny);
        const float g = tv_grad_at(xe, ix, iy, iz, nx, ny, nz, 0.0f);
        x[i] = st_f<VT>(fmaxf(__fmaf_rn(-s, g, __ldg(xe + i)), 0.0f));
    }
}

// ws <- x (as FP32); partial sum of (x - prev)^2.
template <typename VT>
__global__ void __launch_bounds__(256) k_pdelta(const VT* __restrict__ x, const VT* __restrict__ prev,
                                                float* __restrict__ ws, long long n,
                                                double* __restrict__ partial)
{
    __shared__ double sh[8];
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float xv = ld_f(x + i);
        ws[i] = xv;
        const double d = (double)xv - (double)ld_f(prev + i);
        acc += d * d;
    }
    const double t = block_sum_double(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// The TV step shared by EM+TV and ART+TV: partial[0:parts] already holds the
// squared-step partials and ws the FP32 volume xe.
template <typename VT>
static int tv_tail(VT* x, float* ws, int nx, int ny, int nz, float w, int parts, double* partial,
                   double* scale, cudaStream_t st)
{
    k_ptv_norm<<<parts, 256, 0, st>>>(ws, nx, ny, nz, partial + parts);
    CT2_LAUNCHED();
    k_ptv_scale<<<1, 256, 0, st>>>(partial, parts, w, scale);
    CT2_LAUNCHED();
    k_ptv_apply<VT><<<parts, 256, 0, st>>>(x, ws, nx, ny, nz, scale);
    CT2_LAUNCHED();
    return CT2_OK;
}

template <typename VT>
static int em_tv_typed(VT* x, float* ws, const float* sens, int nx, int ny, int nz, float small,
                       float w, double* partial, double* scale, cudaStream_t st)
{
    const long long n = (long long)nx * ny * nz;
    if (n == 0) return CT2_OK;
    const int parts = prec_parts(n);
    k_pem<VT><<<parts, 256, 0, st>>>(x, ws, sens, n, small, partial);
    CT2_LAUNCHED();
    return tv_tail<VT>(x, ws, nx, ny, nz, w, parts, partial, scale, st);
}

template <typename VT>
static int art_tv_typed(VT* x, const VT* prev, float* ws, int nx, int ny, int nz, float w,
                        double* partial, double* scale, cudaStream_t st)
{
    const long long n = (long long)nx * ny * nz;
    if (n == 0) return CT2_OK;
    const int parts = prec_parts(n);
    k_pdelta<VT><<<parts, 256, 0, st>>>(x, prev, ws, n, partial);
    CT2_LAUNCHED();
    return tv_tail<VT>(x, ws, nx, ny, nz, w, parts, partial, scale, st);
}

int prec_art_tv_update(void* x, int vol_type, const void* prev, float* ws, int nx, int ny, int nz,
                       float tv_weight, double* partial, double* scale, cudaStream_t st)
{
    if (vol_type == ST_BF16)
        return art_tv_typed<__nv_bfloat16>((__nv_bfloat16*)x, (const __nv_bfloat16*)prev, ws, nx,
                                           ny, nz, tv_weight, partial, scale, st);
    if (vol_type == ST_F16)
        return art_tv_typed<__half>((__half*)x, (const __half*)prev, ws, nx, ny, nz, tv_weight,
                                    partial, scale, st);
    if (vol_type == ST_F32)
        return art_tv_typed<float>((float*)x, (const float*)prev, ws, nx, ny, nz, tv_weight,
                                   partial, scale, st);
    return set_error(CT2_EINVAL, "precision form: volume type must be bf16, f16 or f32");
}

int prec_em_tv_update(void* x, int vol_type, float* ws, const float* sens, int nx, int ny, int nz,
                      float small, float tv_weight, double* partial, double* scale,
                      cudaStream_t st)
{
    if (vol_type == ST_BF16)
        return em_tv_typed<__nv_bfloat16>((__nv_bfloat16*)x, ws, sens, nx, ny, nz, small,
                                          tv_weight, partial, scale, st);
    if (vol_type == ST_F16)
        return em_tv_typed<__half>((__half*)x, ws, sens, nx, ny, nz, small, tv_weight, partial,
                                   scale, st);
    if (vol_type == ST_F32)
        return em_tv_typed<float>((float*)x, ws, sens, nx, ny, nz, small, tv_weight, partial,
                                  scale, st);
    return set_error(CT2_EINVAL, "precision form: volume type must be bf16, f16 or f32");
}

}  // namespace ct2
