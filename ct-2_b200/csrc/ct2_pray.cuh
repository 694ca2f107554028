// FP64 per-ray setup of the precision form, shared by its projector,
// backprojectors and ART (ct2_precision.cu) and the gather backprojector
// (ct2_gather.cu): source, detector bin, direction, driving axis, slopes,
// travelled length and the FP32 sample model in FP64, and the ray's sample
// interval -- the slices where the model's own FP32 coordinates lie in
// [0, n-1) on both in-plane axes, so every cell is interior without a clamp.
//
// Reference: the per-ray arithmetic of emil_code/view_proj3D.f:784-900,
// evaluated in FP64 rather than REAL*4.
#pragma once

#include "ct2_common.cuh"

namespace ct2 {

// {t in [tmin, tmax] : 0 <= fma(b, t, a) < hi}, one interval (possibly empty)
// because the FP32 fma with fixed a, b is monotone in t.
__device__ __forceinline__ void model_interval_co(float a, float b, float hi, int tmin, int tmax,
                                                  int* t0, int* t1)
{
    *t0 = tmax + 1;
    *t1 = tmax;
    if (!isfinite(a) || !isfinite(b) || tmin > tmax) return;
    if (b == 0.f) {
        if (a >= 0.f && a < hi) {
            *t0 = tmin;
            *t1 = tmax;
        }
        return;
    }
    const double ta = -(double)a / (double)b, tb = ((double)hi - (double)a) / (double)b;
    double tl = fmin(ta, tb), th = fmax(ta, tb);
    tl = floor(tl) - 1.0;
    th = ceil(th) + 1.0;
    if (tl < (double)tmin) tl = (double)tmin;
    if (th > (double)tmax) th = (double)tmax;
    if (tl > th) return;
    int l = (int)tl, h = (int)th;
    while (l <= h) {
        const float f = __fmaf_rn(b, (float)l, a);
        if (f >= 0.f && f < hi) break;
        l++;
    }
    while (h >= l) {
        const float f = __fmaf_rn(b, (float)h, a);
        if (f >= 0.f && f < hi) break;
        h--;
    }
    *t0 = l;
    *t1 = h;
}

__device__ __forceinline__ double sel3d(int i, double a, double b, double c)
{
    return i == 0 ? a : (i == 1 ? b : c);
}

// FP64 ray setup from source S to detector bin B; fills the fields of Ray the
// sample and scatter helpers read (axis permutation, sizes, travelled length,
// model coefficients) and the ray's sample interval [t0, t1].
__device__ __forceinline__ Ray pray_setup(const Grid& G, const double S[3], const double B[3],
                                          int force_axis)
{
    Ray R;
    const double d0 = B[0] - S[0], d1 = B[1] - S[1], d2 = B[2] - S[2];
    const double a0 = fabs(d0) / (double)G.d[0], a1 = fabs(d1) / (double)G.d[1],
                 a2 = fabs(d2) / (double)G.d[2];
    int axis;
    if (force_axis >= 0)
        axis = force_axis;
    else if (a0 > a1 && a0 > a2)
        axis = 0;
    else if (a1 > a2)
        axis = 1;
    else
        axis = 2;
    int p, q, r;
    axis_perm(axis, p, q, r);
    R.p = p;
    R.q = q;
    R.r = r;
    R.np = sel3i(p, G.n[0], G.n[1], G.n[2]);
    R.nq = sel3i(q, G.n[0], G.n[1], G.n[2]);
    R.nr = sel3i(r, G.n[0], G.n[1], G.n[2]);
    const double pd = sel3d(p, d0, d1, d2), qd = sel3d(q, d0, d1, d2), rd = sel3d(r, d0, d1, d2);
    const double op = sel3(p, G.o[0], G.o[1], G.o[2]), dp = sel3(p, G.d[0], G.d[1], G.d[2]);
    const double oq = sel3(q, G.o[0], G.o[1], G.o[2]), dq = sel3(q, G.d[0], G.d[1], G.d[2]);
    const double orr = sel3(r, G.o[0], G.o[1], G.o[2]), dr = sel3(r, G.d[0], G.d[1], G.d[2]);
    const double sp = sel3d(p, S[0], S[1], S[2]), sq = sel3d(q, S[0], S[1], S[2]),
                 sr = sel3d(r, S[0], S[1], S[2]);
    const double qs = qd / pd, rs = rd / pd;
    R.qs = (float)qs;
    R.rs = (float)rs;
    R.tvl = (float)(dp * sqrt(1.0 + qs * qs + rs * rs));
    // slice t centre p_t = op + dp*(t + 0.5); cell coordinate (q(p_t) - oq)/dq - 0.5
    const double dsp = op + 0.5 * dp - sp;
    R.aq = (float)((sq + qs * dsp - oq) / dq - 0.5);
    R.bq = (float)(qs * dp / dq);
    R.ar = (float)((sr + rs * dsp - orr) / dr - 0.5);
    R.br = (float)(rs * dp / dr);
    R.sp = (float)sp;
    R.sq = (float)sq;
    R.sr = (float)sr;
    R.op = (float)op;
    R.dp = (float)dp;
    R.oq = (float)oq;
    R.dq = (float)dq;
    R.orr = (float)orr;
    R.dr = (float)dr;
    int q0, q1, r0, r1;
    model_interval_co(R.aq, R.bq, (float)(R.nq - 1), 0, R.np - 1, &q0, &q1);
    model_interval_co(R.ar, R.br, (float)(R.nr - 1), 0, R.np - 1, &r0, &r1);
    R.t0 = max(q0, r0);
    R.t1 = min(q1, r1);
    return R;
}

// Ray of detector pixel (ju, kv) of one view, bin u0 + (j - 0.5)*du with
// 1-based j (view_proj3D.f:784-796), all in FP64.
__device__ __forceinline__ Ray pray_view(const Grid& G, const float* __restrict__ fv, int ju,
                                         int kv, float du, float dv, float u0, float v0, int force)
{
    double f[15];
#pragma unroll
    for (int i = 0; i < 15; i++) f[i] = (double)__ldg(fv + i);
    const double u = (double)u0 + ((double)ju + 0.5) * (double)du;
    const double v = (double)v0 + ((double)kv + 0.5) * (double)dv;
    const double S[3] = {f[0], f[1], f[2]};
    double B[3];
#pragma unroll
    for (int i = 0; i < 3; i++) B[i] = f[6 + i] + f[9 + i] * u + f[12 + i] * v;
    return pray_setup(G, S, B, force);
}

}  // namespace ct2
