// Sequential Kaczmarz (ART) steps in the reference's ray order.
//
// Reference: view_proj3D.artstep_linear / artstep_nearest
// (emil_code/view_proj3D.f:1950-2271 / :2275-2503), view_proj3D_tomo.artstepz /
// artstepz2vol (emil_code/view_proj3D_tomo.f:154-347 / :352-612),
// ray_proj3D.artstep_linear / artstep_nearest (emil_code/ray_proj3D.f:987-1268 /
// :1272-1450).
//
// The Fortran updates the volume after every ray, so ray r+1 reads what ray r
// wrote: the order view -> u -> v is part of the result.  This kernel keeps
// that order exactly: one warp walks the rays one after another; within a ray
// the 32 lanes split the driving-axis slices (the samples of one ray lie in
// distinct slices, so their taps never collide), reduce the ray sum and the
// squared weight norm with shuffles, then apply
//     x += reg_fac * (y - raysum) * w / sum(w^2)
// to their own slices' taps.  __syncwarp() orders one ray's writes before
// the next ray's reads.  Loads go through L1, not the non-coherent
// read-only path: every kernel here that touches the volume runs as one CTA,
// so all its loads and stores pass through one SM's L1 and see each other
// (the reference-order sweep of config 0 with 16 warps: 187 ms through L1,
// 217 ms with L2-only loads; with 32 warps, 169 ms).  The view geometry runs the same per-ray code on many warps at
// once, on rays that provably touch disjoint voxels (k_art_wave below); the
// ray-list geometry runs strictly in order (k_art_ordered).
#include "ct2_common.cuh"
#include "ct2_kernels.h"

namespace ct2 {

struct VolRef {
    Grid G;
    float* x;
};

// Ray sum (sum of val, without the tvl factor) and squared-weight sum (without
// tvl^2) of this lane's slices of one ray through one volume.
template <int MODE>
__device__ __forceinline__ void lane_sums(const VolRef& V, const Ray& R, int lane, float& s,
                                          float& w2)
{
    const long long sp = sel3l(R.p, V.G.s[0], V.G.s[1], V.G.s[2]);
    const long long sq = sel3l(R.q, V.G.s[0], V.G.s[1], V.G.s[2]);
    const long long sr = sel3l(R.r, V.G.s[0], V.G.s[1], V.G.s[2]);
    for (int t = R.t0 + lane; t <= R.t1; t += 32) {
        const float tf = (float)t;
        if (MODE == MODE_LINEAR) {
            int iq, ir;
            float wq2, wr2;
            sample_in<true>(R, tf, iq, ir, wq2, wr2);
            const float wq1 = 1.0f - wq2, wr1 = 1.0f - wr2;
            const float* b = V.x + t * sp + iq * sq + ir * sr;
            const float v00 = b[0], v10 = b[sq], v01 = b[sr], v11 = b[sq + sr];
            const float vi1 = wq1 * v00 + wq2 * v10;
            const float vi2 = wq1 * v01 + wq2 * v11;
            s += wr1 * vi1 + wr2 * vi2;
            const float a = wq1 * wr1, bb = wq2 * wr1, c = wq1 * wr2, d = wq2 * wr2;
            w2 += a * a + bb * bb + c * c + d * d;
        } else {
            int iq, ir;
            if (!sample_nearest(R, t, MODE, iq, ir)) continue;
            s += V.x[t * sp + iq * sq + ir * sr];
            w2 += 1.0f;
        }
    }
}

template <int MODE>
__device__ __forceinline__ void lane_update(const VolRef& V, const Ray& R, int lane, float coef)
{
    const long long sp = sel3l(R.p, V.G.s[0], V.G.s[1], V.G.s[2]);
    const long long sq = sel3l(R.q, V.G.s[0], V.G.s[1], V.G.s[2]);
    const long long sr = sel3l(R.r, V.G.s[0], V.G.s[1], V.G.s[2]);
    if (MODE == MODE_LINEAR) {
        // two samples per step, all eight taps loaded before any is stored:
        // the taps of one sample are four distinct voxels and two samples lie
        // on different slices, so nothing overlaps, and the loads need not
        // wait for the stores (through one pointer the compiler cannot tell)
        for (int t = R.t0 + lane; t <= R.t1; t += 64) {
            const int u = t + 32;
            const bool two = u <= R.t1;
            int iq, ir, iq2 = 0, ir2 = 0;
            float wq2, wr2, wq22 = 0.f, wr22 = 0.f;
            sample_in<true>(R, (float)t, iq, ir, wq2, wr2);
            if (two) sample_in<true>(R, (float)u, iq2, ir2, wq22, wr22);
            float* b = V.x + t * sp + iq * sq + ir * sr;
            float* c = two ? V.x + u * sp + iq2 * sq + ir2 * sr : b;
            const float b00 = b[0], b10 = b[sq], b01 = b[sr], b11 = b[sq + sr];
            float c00 = 0.f, c10 = 0.f, c01 = 0.f, c11 = 0.f;
            if (two) {
                c00 = c[0];
                c10 = c[sq];
                c01 = c[sr];
                c11 = c[sq + sr];
            }
            const float wq1 = 1.0f - wq2, wr1 = 1.0f - wr2;
            b[0] = b00 + coef * (wq1 * wr1);
            b[sq] = b10 + coef * (wq2 * wr1);
            b[sr] = b01 + coef * (wq1 * wr2);
            b[sq + sr] = b11 + coef * (wq2 * wr2);
            if (two) {
                const float wq12 = 1.0f - wq22, wr12 = 1.0f - wr22;
                c[0] = c00 + coef * (wq12 * wr12);
                c[sq] = c10 + coef * (wq22 * wr12);
                c[sr] = c01 + coef * (wq12 * wr22);
                c[sq + sr] = c11 + coef * (wq22 * wr22);
            }
        }
        return;
    }
    for (int t = R.t0 + lane; t <= R.t1; t += 32) {
        {
            int iq, ir;
            if (!sample_nearest(R, t, MODE, iq, ir)) continue;
            V.x[t * sp + iq * sq + ir * sr] += coef;
        }
    }
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int MODE, bool LIST, int FORCE, bool TWOVOL>
__global__ void __launch_bounds__(32) k_art_ordered(ArtArgs a)
{
    const int lane = threadIdx.x;
    const long long nrays = LIST ? a.nrays : (long long)a.ns * a.nu * a.nv;
    VolRef V{a.G, a.x};
    VolRef VA{a.GA, a.xa};
    for (long long r = 0; r < nrays; r++) {
        if (a.ind != nullptr && a.ind[r] != 1) continue;
        float S[3], B[3];
        if (LIST) {
            const float* v = a.geom + 6 * r;
            S[0] = v[0]; S[1] = v[1]; S[2] = v[2];
            B[0] = v[3]; B[1] = v[4]; B[2] = v[5];
        } else {
            const long long per_view = (long long)a.nu * a.nv;
            const int view = (int)(r / per_view);
            const long long rem = r - (long long)view * per_view;
            const int ju = (int)(rem / a.nv), kv = (int)(rem - (long long)ju * a.nv);
            float f[18];
#pragma unroll
            for (int i = 0; i < 18; i++) f[i] = __ldg(a.geom + 18 * view + i);
            S[0] = f[0]; S[1] = f[1]; S[2] = f[2];
            view_bin(f, ju, kv, a.du, a.dv, a.u0, a.v0, B);
        }
        const float y = __ldg(a.y + r);
        Ray R = ray_setup(V.G, S, B, FORCE, MODE);
        if (MODE == MODE_LINEAR) {
            int s0, s1;
            exact_interval(R, R.np, &s0, &s1);
        }
        float s = 0.f, w2 = 0.f;
        lane_sums<MODE>(V, R, lane, s, w2);
        s = warp_sum(s) * R.tvl;
        w2 = warp_sum(w2) * (R.tvl * R.tvl);
        Ray RA;
        if (TWOVOL) {
            RA = ray_setup(VA.G, S, B, FORCE, MODE);
            if (MODE == MODE_LINEAR) {
                int s0, s1;
                exact_interval(RA, RA.np, &s0, &s1);
            }
            float sa = 0.f, w2a = 0.f;
            lane_sums<MODE>(VA, RA, lane, sa, w2a);
            s += warp_sum(sa) * RA.tvl;
            w2 += warp_sum(w2a) * (RA.tvl * RA.tvl);
        }
        if (w2 > 0.f) {  // a ray with no samples leaves the volume unchanged
            const float coef = a.reg_fac * (y - s) / w2;
            lane_update<MODE>(V, R, lane, coef * R.tvl);
            if (TWOVOL) lane_update<MODE>(VA, RA, lane, coef * RA.tvl);
        }
        __syncwarp();
        __threadfence_block();
    }
}

// ---- view geometry: the same order, rays that cannot touch run together --
//
// All rays of a view leave one source S.  The rays of detector row k lie in
// the plane through S and the row's line (direction eu); every row plane
// contains the line L through S along eu.  Each tap of a ray lies within
// about one voxel (index units; 1 + the guard band where an edge cell is
// clamped) of the ray's line inside the volume, so two rays cannot share a
// voxel if every point of one is at least kSep voxels (Chebyshev, index
// units) from every point of the other inside the volume.  A point P of row
// plane k' is at Euclidean distance dist(P, L) * sin(phi) from row plane k,
// phi their dihedral angle, and |(P - Q).n| for the plane's unit normal n
// is at most the Chebyshev index distance times sum_i |n_i| d_i.
// k_art_rows finds per view the smallest row gap cv with min over the volume
// of dist(P, L) times sin of the smallest dihedral angle between rows cv
// apart at least kSep times the largest sum_i |n_i| d_i over the row planes;
// rays whose rows differ by cv or more then never touch.
//
// The reference order is view -> u (column j) -> v (row k).  Rays (j, k)
// with the same step s = k + cv*j differ by a multiple of cv rows, so they
// are disjoint and run together; a ray that the reference applies before an
// overlapping one (same column and lower row, or a lower column within cv
// rows) has a smaller step.  Running the steps in order with a block-wide
// barrier between them therefore gives each ray exactly the volume it sees
// in the sequential sweep, and the ray's own arithmetic (lane partial sums,
// shuffle reduction) is that of k_art_ordered: the result is the same, bit
// for bit.  cv = nv (no safe gap found, e.g. a source inside the volume's
// reach) degenerates to one ray per step.
constexpr double kSep = 2.5;

__device__ double dist_to_line(double px, double py, double pz, const double S[3],
                               const double e[3])
{
    const double dx = px - S[0], dy = py - S[1], dz = pz - S[2];
    const double t = dx * e[0] + dy * e[1] + dz * e[2];
    const double rx = dx - t * e[0], ry = dy - t * e[1], rz = dz - t * e[2];
    return sqrt(rx * rx + ry * ry + rz * rz);
}

// One warp per view: cvs[view] = smallest safe row gap (nv if none).
__global__ void __launch_bounds__(32) k_art_rows(const float* __restrict__ geom, Grid G, Grid GA,
                                                int twovol, int nv, float dv, float v0,
                                                int* __restrict__ cvs)
{
    const int view = blockIdx.x, lane = threadIdx.x;
    const float* f = geom + 18 * view;
    const double S[3] = {f[0], f[1], f[2]};
    const double D[3] = {f[6], f[7], f[8]};
    const double eu[3] = {f[9], f[10], f[11]}, ev[3] = {f[12], f[13], f[14]};
    const double ew[3] = {f[15], f[16], f[17]};
    const double nu2 = sqrt(eu[0] * eu[0] + eu[1] * eu[1] + eu[2] * eu[2]);
    const double e[3] = {eu[0] / nu2, eu[1] / nu2, eu[2] / nu2};
    // the volume's box and voxel sides (both volumes in the two-volume form)
    double lo[3], hi[3], dd[3];
    for (int i = 0; i < 3; i++) {
        lo[i] = (double)G.o[i];
        hi[i] = (double)G.o[i] + (double)G.n[i] * (double)G.d[i];
        dd[i] = fabs((double)G.d[i]);
        if (twovol) {
            lo[i] = fmin(lo[i], (double)GA.o[i]);
            hi[i] = fmax(hi[i], (double)GA.o[i] + (double)GA.n[i] * (double)GA.d[i]);
            dd[i] = fmax(dd[i], fabs((double)GA.d[i]));
        }
    }
    // min distance from the box to L: sampled on the six faces, less the
    // sampling's Lipschitz margin (distance to a line is 1-Lipschitz)
    constexpr int M = 64;
    double rho = INFINITY, hstep = 0.0;
    for (int face = 0; face < 6; face++) {
        const int ax = face >> 1, a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
        const double c = (face & 1) ? hi[ax] : lo[ax];
        const double h1 = (hi[a1] - lo[a1]) / (M - 1), h2 = (hi[a2] - lo[a2]) / (M - 1);
        hstep = fmax(hstep, sqrt(h1 * h1 + h2 * h2));
        for (int idx = lane; idx < M * M; idx += 32) {
            double p[3];
            p[ax] = c;
            p[a1] = lo[a1] + (idx / M) * h1;
            p[a2] = lo[a2] + (idx % M) * h2;
            rho = fmin(rho, dist_to_line(p[0], p[1], p[2], S, e));
        }
    }
    for (int o = 16; o > 0; o >>= 1) rho = fmin(rho, __shfl_xor_sync(0xffffffffu, rho, o));
    rho -= 0.5 * hstep;
    // row angles in the plane across L: row k's line sits at (a_v + v_k, a_w)
    const double av = (D[0] - S[0]) * ev[0] + (D[1] - S[1]) * ev[1] + (D[2] - S[2]) * ev[2];
    const double aw = (D[0] - S[0]) * ew[0] + (D[1] - S[1]) * ew[1] + (D[2] - S[2]) * ew[2];
    // |(P - Q).n| <= (Chebyshev index distance) * sum_i |n_i| d_i for a unit
    // n, and |(P - Q).n_k| = dist(P, row plane k) for Q on that plane: the
    // separation needed is kSep times the largest sum_i |n_k,i| d_i over the
    // rows' unit normals n_k = (aw ev - (av + v_k) ew) / norm
    double wmax = 0.0;
    for (int k = lane; k < nv; k += 32) {
        const double vk = (double)v0 + ((double)k + 0.5) * (double)dv;
        const double a = aw, b = -(av + vk), nn = sqrt(a * a + b * b);
        double w = 0.0;
        for (int i = 0; i < 3; i++) w += fabs((a * ev[i] + b * ew[i]) / nn) * dd[i];
        wmax = fmax(wmax, w);
    }
    for (int o = 16; o > 0; o >>= 1) wmax = fmax(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
    const double need = kSep * wmax;
    // the row-plane argument needs an orthonormal detector frame
    const double dots[6] = {eu[0] * eu[0] + eu[1] * eu[1] + eu[2] * eu[2] - 1.0,
                            ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2] - 1.0,
                            ew[0] * ew[0] + ew[1] * ew[1] + ew[2] * ew[2] - 1.0,
                            eu[0] * ev[0] + eu[1] * ev[1] + eu[2] * ev[2],
                            eu[0] * ew[0] + eu[1] * ew[1] + eu[2] * ew[2],
                            ev[0] * ew[0] + ev[1] * ew[1] + ev[2] * ew[2]};
    bool frame_ok = true;
    for (int i = 0; i < 6; i++) frame_ok = frame_ok && fabs(dots[i]) < 1e-5;
    int best = nv;
    if (frame_ok && rho > 0.0 && isfinite(rho)) {
        for (int cv = 1; cv < nv && best == nv; cv++) {
            double dmin = INFINITY;
            for (int k = lane; k + cv < nv; k += 32) {
                const double v1 = (double)v0 + ((double)k + 0.5) * (double)dv;
                const double v2 = (double)v0 + ((double)(k + cv) + 0.5) * (double)dv;
                const double d = fabs(atan2(av + v2, aw) - atan2(av + v1, aw));
                dmin = fmin(dmin, d);
            }
            for (int o = 16; o > 0; o >>= 1)
                dmin = fmin(dmin, __shfl_xor_sync(0xffffffffu, dmin, o));
            if (dmin < 1.5 && rho * sin(dmin) >= need) best = cv;
        }
    }
    if (lane == 0) cvs[view] = best;
}

// Warps of the wave's single CTA: each takes one ray of a step at a time
// (measured on config 0: 169 ms with 32, 187 ms with 16).
constexpr int kWaveWarps = 32;

// Set-ups of the rays of views [view0, view0 + nviews), one thread per ray,
// over the whole GPU: geometry only (no volume access), written once and
// read by k_art_wave, which then spends its serial steps on the volume
// passes alone.
template <int MODE, int FORCE, bool TWOVOL>
__global__ void __launch_bounds__(256) k_art_setup(ArtArgs a, int view0, int nviews,
                                                   Ray* __restrict__ rays, Ray* __restrict__ raysA)
{
    const long long per_view = (long long)a.nu * a.nv;
    const long long n = per_view * nviews;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int view = view0 + (int)(i / per_view);
        const long long rem = i - (long long)(view - view0) * per_view;
        const int ju = (int)(rem / a.nv), kv = (int)(rem - (long long)ju * a.nv);
        float f[18];
#pragma unroll
        for (int k = 0; k < 18; k++) f[k] = __ldg(a.geom + 18 * view + k);
        const float S[3] = {f[0], f[1], f[2]};
        float B[3];
        view_bin(f, ju, kv, a.du, a.dv, a.u0, a.v0, B);
        Ray R = ray_setup(a.G, S, B, FORCE, MODE);
        if (MODE == MODE_LINEAR) {
            int s0, s1;
            exact_interval(R, R.np, &s0, &s1);
        }
        rays[i] = R;
        if (TWOVOL) {
            Ray RA = ray_setup(a.GA, S, B, FORCE, MODE);
            if (MODE == MODE_LINEAR) {
                int s0, s1;
                exact_interval(RA, RA.np, &s0, &s1);
            }
            raysA[i] = RA;
        }
    }
}

// The steps of views [view0, view0 + nviews) in order, rays set up by
// k_art_setup (ray i of the chunk: (view - view0) * nu * nv + ju * nv + kv).
template <int MODE, int FORCE, bool TWOVOL>
__global__ void __launch_bounds__(32 * kWaveWarps) k_art_wave(ArtArgs a, const int* __restrict__ cvs,
                                                             int view0, int nviews,
                                                             const Ray* __restrict__ rays,
                                                             const Ray* __restrict__ raysA)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    VolRef V{a.G, a.x};
    VolRef VA{a.GA, a.xa};
    const long long per_view = (long long)a.nu * a.nv;
    for (int view = view0; view < view0 + nviews; view++) {
        const int cv = cvs[view];
        const long long nsteps = (long long)(a.nv - 1) + (long long)cv * (a.nu - 1) + 1;
        const long long base = (long long)(view - view0) * per_view;
        for (long long s = 0; s < nsteps; s++) {
            // columns j with 0 <= s - cv*j < nv
            const long long jlo = s >= a.nv ? (s - a.nv) / cv + 1 : 0;
            const long long jhi = min((long long)a.nu - 1, s / cv);
            for (long long j = jlo + warp; j <= jhi; j += kWaveWarps) {
                const int ju = (int)j, kv = (int)(s - (long long)cv * j);
                const long long r = (long long)view * per_view + (long long)ju * a.nv + kv;
                if (a.ind != nullptr && a.ind[r] != 1) continue;
                const long long i = base + (long long)ju * a.nv + kv;
                const float y = __ldg(a.y + r);
                const Ray R = rays[i];
                float sm = 0.f, w2 = 0.f;
                lane_sums<MODE>(V, R, lane, sm, w2);
                sm = warp_sum(sm) * R.tvl;
                w2 = warp_sum(w2) * (R.tvl * R.tvl);
                Ray RA;
                if (TWOVOL) {
                    RA = raysA[i];
                    float sa = 0.f, w2a = 0.f;
                    lane_sums<MODE>(VA, RA, lane, sa, w2a);
                    sm += warp_sum(sa) * RA.tvl;
                    w2 += warp_sum(w2a) * (RA.tvl * RA.tvl);
                }
                if (w2 > 0.f) {
                    const float coef = a.reg_fac * (y - sm) / w2;
                    lane_update<MODE>(V, R, lane, coef * R.tvl);
                    if (TWOVOL) lane_update<MODE>(VA, RA, lane, coef * RA.tvl);
                }
            }
            __syncthreads();  // this step's writes before the next step's reads
        }
    }
}

constexpr long long kArtSetupBytes = 256ll << 20;  // ray set-ups held at a time

template <int MODE, bool LIST, int FORCE, bool TWOVOL>
static int launch_art(const ArtArgs& a, cudaStream_t st)
{
    if (LIST) {  // arbitrary rays share no source: strictly one after another
        k_art_ordered<MODE, LIST, FORCE, TWOVOL><<<1, 32, 0, st>>>(a);
        CT2_LAUNCHED();
        return CT2_OK;
    }
    if (a.ns == 0 || a.nu == 0 || a.nv == 0) return CT2_OK;
    const long long per_view = (long long)a.nu * a.nv;
    const long long ray_bytes = (long long)sizeof(Ray) * (TWOVOL ? 2 : 1);
    long long chunk = kArtSetupBytes / (per_view * ray_bytes);
    if (chunk < 1) chunk = 1;
    if (chunk > a.ns) chunk = a.ns;
    int* cvs = nullptr;
    Ray* rays = nullptr;
    CT2_CUDA(cudaMallocAsync((void**)&cvs, sizeof(int) * a.ns, st));
    cudaError_t e = cudaMallocAsync((void**)&rays, (size_t)(chunk * per_view * ray_bytes), st);
    if (e == cudaSuccess) {
        Ray* raysA = TWOVOL ? rays + chunk * per_view : nullptr;
        k_art_rows<<<a.ns, 32, 0, st>>>(a.geom, a.G, a.GA, TWOVOL ? 1 : 0, a.nv, a.dv, a.v0, cvs);
        note_launch();
        e = cudaGetLastError();
        for (int v0 = 0; v0 < a.ns && e == cudaSuccess; v0 += (int)chunk) {
            const int nvw = (int)min(chunk, (long long)a.ns - v0);
            long long blocks = (per_view * nvw + 255) / 256;
            if (blocks > 148ll * 16) blocks = 148ll * 16;
            k_art_setup<MODE, FORCE, TWOVOL><<<(unsigned)blocks, 256, 0, st>>>(a, v0, nvw, rays,
                                                                                raysA);
            note_launch();
            e = cudaGetLastError();
            if (e != cudaSuccess) break;
            k_art_wave<MODE, FORCE, TWOVOL><<<1, 32 * kWaveWarps, 0, st>>>(a, cvs, v0, nvw, rays,
                                                                            raysA);
            note_launch();
            e = cudaGetLastError();
        }
        cudaFreeAsync(rays, st);
    }
    cudaFreeAsync(cvs, st);
    if (e != cudaSuccess) return set_error(CT2_ECUDA, "ART launch: %s", cudaGetErrorString(e));
    return CT2_OK;
}

int art_ordered(const ArtArgs& a, int mode, bool list, bool force_z, bool twovol, cudaStream_t st)
{
    if (twovol) {
        if (list || !force_z || mode != MODE_LINEAR)
            return set_error(CT2_EINVAL, "two-volume ART is the z-driven linear view form only");
        return launch_art<MODE_LINEAR, false, 2, true>(a, st);
    }
    if (list) {
        if (mode == MODE_LINEAR) return launch_art<MODE_LINEAR, true, -1, false>(a, st);
        if (mode == MODE_NEAREST_LT) return launch_art<MODE_NEAREST_LT, true, -1, false>(a, st);
        if (mode == MODE_NEAREST_LE) return launch_art<MODE_NEAREST_LE, true, -1, false>(a, st);
        return set_error(CT2_EINVAL, "unsupported ART mode");
    }
    if (force_z) {
        if (mode != MODE_LINEAR) return set_error(CT2_EINVAL, "z-driven ART is linear only");
        return launch_art<MODE_LINEAR, false, 2, false>(a, st);
    }
    if (mode == MODE_LINEAR) return launch_art<MODE_LINEAR, false, -1, false>(a, st);
    if (mode == MODE_NEAREST_LE) return launch_art<MODE_NEAREST_LE, false, -1, false>(a, st);
    return set_error(CT2_EINVAL, "unsupported ART mode");
}

}  // namespace ct2
