// All-pairs tangent-point energy and its adjoint gradient, FP64.
//
// Reference: calculateEnergy / gradientAnalytical / kernelDerivs in
// src/core/tangentPointEnergy.ts:50-392. Ordered disjoint pairs (I, J) are
// never materialised: the J edges stream through shared memory in tiles and
// disjointness is tested from endpoint indices.
//
// The context's energy and gradient use the symmetric tile-pair form: each
// unordered pair is evaluated once for both orders (I, J) and (J, I), which
// share |d|, d_hat and (|d|+eps)^b. The adjoint gradient recomputes the pair
// terms (nothing of size E^2 is stored) and uses no atomics: every
// contribution lands in a fixed (edge, partner tile) slot and slots are summed
// in a fixed order (deterministic). energy_kernel, the edge-owner form, serves
// the allocation-free entry point, whose scratch is sized for it.
#include <math.h>

#include <algorithm>

#include "tpe_internal.h"

namespace tpe {
namespace {

constexpr int kThreads = 128;   // edges I per block
constexpr int kTile = 128;      // edges J per shared-memory tile

template <int MODE>
__device__ __forceinline__ double pow_a(double x, double a) {
    if (MODE == 1) return x * x * x;  // a = 3
    return pow(x, a);
}
template <int MODE>
__device__ __forceinline__ double pow_a1(double x, double a) {
    if (MODE == 1) return x * x;  // a - 1 = 2
    return pow(x, a - 1.0);
}
template <int MODE>
__device__ __forceinline__ double pow_b(double x, double b) {
    if (MODE == 1) {
        const double x2 = x * x;
        return x2 * x2 * x2;  // b = 6
    }
    return pow(x, b);
}

// s = sqrt(x), inv_s = 1/s (0 below 1e-14) and inv_se = 1/(s + eps) for x >= 0,
// from one reciprocal square root r: s = x r and 1/(s + eps) = r / (1 + t) with
// t = eps r, summed as r (1 - t + t^2) when t < 2^-20 (the first term left out
// is below 2^-60 relative). Distances within about 1e6 eps of zero (and
// non-finite input) take the square root and the divisions themselves.
__device__ __forceinline__ void dist_terms(double x, double eps, double& s, double& inv_s,
                                           double& inv_se) {
    const double r = rsqrt(x);
    const double t = eps * r;
    if (t < 9.5367431640625e-07) {
        s = x * r;
        inv_s = r;
        inv_se = fma(-r, t * (1.0 - t), r);
    } else {
        s = sqrt(x);
        inv_s = s < 1e-14 ? 0.0 : 1.0 / s;
        inv_se = 1.0 / (s + eps);
    }
}

// sqrt(x) for x >= 0 from a reciprocal square root (0 at x = 0).
__device__ __forceinline__ double sqrt_r(double x) { return x > 0.0 ? x * rsqrt(x) : sqrt(x); }

__device__ __forceinline__ bool disjoint(int2 a, int2 b) {
    return a.x != b.x && a.x != b.y && a.y != b.x && a.y != b.y;
}

// Per-edge records: a = (p1, |e|+eps), b = (p2, (|e|+eps)^(1-alpha)).
__global__ void edge_prep_kernel(const double* __restrict__ pos, const int2* __restrict__ edges,
                                 int32_t E, int32_t V, int32_t ncurves, double eps, double alpha,
                                 double4* __restrict__ ea, double4* __restrict__ eb) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)E * ncurves) return;
    const int32_t c = (int32_t)(t / E), I = (int32_t)(t % E);
    const double* p = pos + (int64_t)c * 3 * V;
    const int2 e = edges[I];
    const double x1 = p[3 * e.x], y1 = p[3 * e.x + 1], z1 = p[3 * e.x + 2];
    const double x2 = p[3 * e.y], y2 = p[3 * e.y + 1], z2 = p[3 * e.y + 2];
    const double ex = x2 - x1, ey = y2 - y1, ez = z2 - z1;
    const double ell = sqrt(ex * ex + ey * ey + ez * ez) + eps;
    ea[t] = make_double4(x1, y1, z1, ell);
    eb[t] = make_double4(x2, y2, z2, pow(ell, 1.0 - alpha));
}

template <int MODE>
__global__ void __launch_bounds__(kThreads)
energy_kernel(const double4* __restrict__ ea, const double4* __restrict__ eb,
              const int2* __restrict__ edges, int32_t E, int32_t jchunk, double alpha,
              double beta, double eps, double* __restrict__ partial) {
    __shared__ double4 sa[kTile], sb[kTile];
    __shared__ int2 se[kTile];
    __shared__ double red[kThreads / 32];
    const int32_t c = blockIdx.z;
    ea += (int64_t)c * E;
    eb += (int64_t)c * E;
    const int32_t I = blockIdx.x * kThreads + threadIdx.x;
    const bool valid = I < E;
    double4 a = make_double4(0, 0, 0, 0), b = a;
    int2 ei = make_int2(-1, -1);
    if (valid) {
        a = ea[I];
        b = eb[I];
        ei = edges[I];
    }
    const double eIx = b.x - a.x, eIy = b.y - a.y, eIz = b.z - a.z;
    const double powI = b.w;  // (l_I)^(1-alpha)
    double acc = 0.0;
    const int32_t j0 = blockIdx.y * jchunk;
    const int32_t j1 = min(E, j0 + jchunk);
    for (int32_t t0 = j0; t0 < j1; t0 += kTile) {
        const int32_t nt = min(kTile, j1 - t0);
        __syncthreads();
        if (threadIdx.x < nt) {
            sa[threadIdx.x] = ea[t0 + threadIdx.x];
            sb[threadIdx.x] = eb[t0 + threadIdx.x];
            se[threadIdx.x] = edges[t0 + threadIdx.x];
        }
        __syncthreads();
        if (!valid) continue;
        for (int32_t jj = 0; jj < nt; jj++) {
            const int2 ej = se[jj];
            if (!disjoint(ei, ej) ) continue;
            const double4 qa = sa[jj], qb = sb[jj];
            double sumK = 0.0;
#pragma unroll
            for (int s = 0; s < 4; s++) {
                const double px = (s < 2) ? a.x : b.x, py = (s < 2) ? a.y : b.y,
                             pz = (s < 2) ? a.z : b.z;
                const double qx = (s & 1) ? qb.x : qa.x, qy = (s & 1) ? qb.y : qa.y,
                             qz = (s & 1) ? qb.z : qa.z;
                const double dx = px - qx, dy = py - qy, dz = pz - qz;
                const double invDn = 1.0 / (sqrt(dx * dx + dy * dy + dz * dz) + eps);
                const double cx = eIy * dz - eIz * dy;
                const double cy = eIz * dx - eIx * dz;
                const double cz = eIx * dy - eIy * dx;
                const double cn = sqrt(cx * cx + cy * cy + cz * cz) + eps;
                sumK += (MODE == 1) ? pow_a<1>(cn, alpha) * pow_b<1>(invDn, beta)
                                    : pow(cn, alpha) / pow(1.0 / invDn, beta);
            }
            acc += powI * qa.w * sumK;
        }
    }
    // block reduction (fixed order)
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; w++) s += red[w];
        partial[((int64_t)c * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
    }
}

// Sums nparts partials per curve in a fixed order: out[c] = scale * sum.
__global__ void reduce_partials(const double* __restrict__ partial, int32_t nparts, double scale,
                                double* __restrict__ out) {
    __shared__ double red[32];
    const int32_t c = blockIdx.x;
    double s = 0.0;
    for (int32_t i = threadIdx.x; i < nparts; i += blockDim.x) s += partial[(int64_t)c * nparts + i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        out[c] = scale * t;
    }
}

// edge_prep_kernel for edge indices that were never checked on the host (the
// allocation-free entry point): an endpoint outside [0, V) skips the position
// loads, leaves a NaN record and sets *bad.
__global__ void edge_prep_checked_kernel(const double* __restrict__ p, const int2* __restrict__ edges,
                                         int32_t E, int32_t V, double eps, double alpha,
                                         double4* __restrict__ ea, double4* __restrict__ eb,
                                         int32_t* __restrict__ bad) {
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= E) return;
    const int2 e = edges[I];
    if (e.x < 0 || e.x >= V || e.y < 0 || e.y >= V) {
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        ea[I] = make_double4(nan, nan, nan, nan);
        eb[I] = make_double4(nan, nan, nan, nan);
        atomicOr(bad, 1);
        return;
    }
    const double x1 = p[3 * e.x], y1 = p[3 * e.x + 1], z1 = p[3 * e.x + 2];
    const double x2 = p[3 * e.y], y2 = p[3 * e.y + 1], z2 = p[3 * e.y + 2];
    const double ex = x2 - x1, ey = y2 - y1, ez = z2 - z1;
    const double ell = sqrt(ex * ex + ey * ey + ez * ez) + eps;
    ea[I] = make_double4(x1, y1, z1, ell);
    eb[I] = make_double4(x2, y2, z2, pow(ell, 1.0 - alpha));
}

// reduce_partials for one curve, NaN when *bad is set.
__global__ void reduce_partials_checked(const double* __restrict__ partial, int32_t nparts,
                                        double scale, const int32_t* __restrict__ bad,
                                        double* __restrict__ out) {
    __shared__ double red[32];
    double s = 0.0;
    for (int32_t i = threadIdx.x; i < nparts; i += blockDim.x) s += partial[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        out[0] = *bad ? __longlong_as_double(0x7ff8000000000000LL) : scale * t;
    }
}

// ---- symmetric (tile-pair) forms ---------------------------------------------
//
// Each unordered pair {I, J} of edges is evaluated once: the grid covers the
// tiles (bi, bj), bi <= bj, of 128 x 128 edges; thread t owns I = 128 bi + t and
// walks the J of tile bj (J > I inside a diagonal tile). Both orders (I, J) and
// (J, I) share |d|, d_hat and (|d|+eps)^-b per endpoint combination, so the
// pair work is about half of the edge-owner form. Deterministic: the J-side
// gradient contributions of a warp's 32 lanes are summed by a fixed shuffle
// tree, the four warps' sums in a fixed order, and every (edge, partner tile)
// partial is written exactly once.

// Upper tile (bi <= bj) of the packed index x over a T x T tile grid.
__device__ __forceinline__ void upper_tile(int x, int& bi, int& bj) {
    int t = (int)((sqrt(8.0 * (double)x + 1.0) - 1.0) * 0.5);
    while ((t + 1) * (t + 2) / 2 <= x) t++;
    while (t * (t + 1) / 2 > x) t--;
    bj = t;
    bi = x - t * (t + 1) / 2;
}

template <int MODE>
__global__ void __launch_bounds__(kThreads)
energy_sym_kernel(const double4* __restrict__ ea, const double4* __restrict__ eb,
                  const int2* __restrict__ edges, int32_t E, double alpha, double beta, double eps,
                  double* __restrict__ partial) {
    __shared__ double4 sa[kTile], sb[kTile];
    __shared__ int2 se[kTile];
    __shared__ double red[kThreads / 32];
    const int32_t c = blockIdx.z;
    ea += (int64_t)c * E;
    eb += (int64_t)c * E;
    int bi, bj;
    upper_tile(blockIdx.x, bi, bj);
    const int32_t I = bi * kTile + threadIdx.x;
    const bool valid = I < E;
    double4 a = make_double4(0, 0, 0, 0), b = a;
    int2 ei = make_int2(-1, -1);
    if (valid) {
        a = ea[I];
        b = eb[I];
        ei = edges[I];
    }
    {
        const int32_t J = bj * kTile + threadIdx.x;
        if (J < E) {
            sa[threadIdx.x] = ea[J];
            sb[threadIdx.x] = eb[J];
            se[threadIdx.x] = edges[J];
        }
    }
    __syncthreads();
    const double eIx = b.x - a.x, eIy = b.y - a.y, eIz = b.z - a.z;
    const double powI = b.w, ellI = a.w;
    const int32_t nt = min(kTile, E - bj * kTile);
    const int32_t js = (bi == bj) ? (int32_t)threadIdx.x + 1 : 0;
    double acc = 0.0;
    if (valid) {
        for (int32_t jj = js; jj < nt; jj++) {
            if (!disjoint(ei, se[jj])) continue;
            const double4 qa = sa[jj], qb = sb[jj];
            const double eJx = qb.x - qa.x, eJy = qb.y - qa.y, eJz = qb.z - qa.z;
            double sumF = 0.0, sumF2 = 0.0;
#pragma unroll
            for (int s2 = 0; s2 < 4; s2++) {
                const double px = (s2 < 2) ? a.x : b.x, py = (s2 < 2) ? a.y : b.y,
                             pz = (s2 < 2) ? a.z : b.z;
                const double qx = (s2 & 1) ? qb.x : qa.x, qy = (s2 & 1) ? qb.y : qa.y,
                             qz = (s2 & 1) ? qb.z : qa.z;
                const double dx = px - qx, dy = py - qy, dz = pz - qz;
                double dn, invD, invDn;
                dist_terms(dx * dx + dy * dy + dz * dz, eps, dn, invD, invDn);
                const double iDb = (MODE == 1) ? pow_b<1>(invDn, beta) : 0.0;
                const double cx = eIy * dz - eIz * dy, cy = eIz * dx - eIx * dz,
                             cz = eIx * dy - eIy * dx;
                const double cn = sqrt_r(cx * cx + cy * cy + cz * cz) + eps;
                const double kx = eJy * dz - eJz * dy, ky = eJz * dx - eJx * dz,
                             kz = eJx * dy - eJy * dx;
                const double kn = sqrt_r(kx * kx + ky * ky + kz * kz) + eps;
                if (MODE == 1) {
                    sumF += pow_a<1>(cn, alpha) * iDb;
                    sumF2 += pow_a<1>(kn, alpha) * iDb;
                } else {
                    const double den = pow(dn + eps, beta);
                    sumF += pow(cn, alpha) / den;
                    sumF2 += pow(kn, alpha) / den;
                }
            }
            acc += powI * qa.w * sumF + qb.w * ellI * sumF2;
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; w++) t += red[w];
        partial[(int64_t)c * gridDim.x + blockIdx.x] = t;
    }
}

// f, d-derivative and e-derivative of one kernelDerivs evaluation
// (tangentPointEnergy.ts:165-244) as vectors.
template <int MODE>
__device__ __forceinline__ double kd_vec(double ex, double ey, double ez, double dx, double dy,
                                         double dz, double hx, double hy, double hz,
                                         double invDPowB, double invDe, double alpha, double beta,
                                         double eps, double (&dd)[3], double (&de)[3]) {
    const double cx = ey * dz - ez * dy;
    const double cy = ez * dx - ex * dz;
    const double cz = ex * dy - ey * dx;
    const double c2 = cx * cx + cy * cy + cz * cz;
    double rc, inv = 0.0;
    if (c2 >= 1e-28) {
        inv = rsqrt(c2);
        rc = c2 * inv;
    } else {
        rc = sqrt(c2);
    }
    const double ce = rc + eps;
    const double f = pow_a<MODE>(ce, alpha) * invDPowB;
    const double coeff_c = alpha * pow_a1<MODE>(ce, alpha) * invDPowB;
    const double coeff_d = -beta * f * invDe;
    double ux = 0, uy = 0, uz = 0, vx = 0, vy = 0, vz = 0;
    if (c2 >= 1e-28) {
        ux = inv * (cy * ez - cz * ey);
        uy = inv * (cz * ex - cx * ez);
        uz = inv * (cx * ey - cy * ex);
        vx = inv * (dy * cz - dz * cy);
        vy = inv * (dz * cx - dx * cz);
        vz = inv * (dx * cy - dy * cx);
    }
    dd[0] = coeff_c * ux + coeff_d * hx;
    dd[1] = coeff_c * uy + coeff_d * hy;
    dd[2] = coeff_c * uz + coeff_d * hz;
    de[0] = coeff_c * vx;
    de[1] = coeff_c * vy;
    de[2] = coeff_c * vz;
    return f;
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Shared memory of one 128-thread tile worker.
struct GradSmem {
    double4 sa[kTile], sb[kTile];
    double4 sh[kTile];  // J: unit tangent xyz, (1-a) l^-a
    int2 se[kTile];
    double accJ[kThreads / 32][kTile][6];
    double red[kThreads / 32];
};

// Barrier over the 128 threads of one tile worker (named barrier bar; 0 is the
// whole-block barrier of a 128-thread block).
__device__ __forceinline__ void worker_sync(int bar) {
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(kThreads) : "memory");
}

// Gradient partials edge_acc[slot][K][6] (endpoint 1 xyz, endpoint 2 xyz) and
// energy partials of upper tile x: the tile (bi, bj) writes slot bj of its I
// edges and slot bi of its J edges (both slot bi on a diagonal tile). The
// gather sums all slots. tid < 128 is the thread's index in its worker.
template <int MODE>
__device__ __forceinline__ void grad_sym_tile(int x, int tid, int bar, GradSmem& sm,
                                              const double4* __restrict__ ea,
                                              const double4* __restrict__ eb,
                                              const int2* __restrict__ edges, int32_t E,
                                              double alpha, double beta, double eps,
                                              double* __restrict__ edge_acc,
                                              double* __restrict__ partial) {
    double4* sa = sm.sa;
    double4* sb = sm.sb;
    double4* sh = sm.sh;
    int2* se = sm.se;
    double(*accJ)[kTile][6] = sm.accJ;
    double* red = sm.red;
    const int lane = tid & 31, warp = tid >> 5;
    int bi, bj;
    upper_tile(x, bi, bj);
    const bool diag = bi == bj;
    const int32_t I = bi * kTile + tid;
    const bool valid = I < E;
    double4 a = make_double4(0, 0, 0, 1), b = make_double4(0, 0, 0, 1);
    int2 ei = make_int2(-1, -1);
    if (valid) {
        a = ea[I];
        b = eb[I];
        ei = edges[I];
    }
    const double eIx = b.x - a.x, eIy = b.y - a.y, eIz = b.z - a.z;
    double hIx = 0, hIy = 0, hIz = 0;
    {
        const double reI = sqrt(eIx * eIx + eIy * eIy + eIz * eIz);
        if (!(reI < 1e-14)) {
            const double inv = 1.0 / reI;
            hIx = inv * eIx;
            hIy = inv * eIy;
            hIz = inv * eIz;
        }
    }
    const double ellI = a.w, powI = b.w;
    const double dPowI = (1.0 - alpha) * pow(ellI, -alpha);
    {
        const int32_t J = bj * kTile + tid;
        double4 qa = make_double4(0, 0, 0, 1), qb = make_double4(0, 0, 0, 1);
        int2 ej = make_int2(-2, -2);
        if (J < E) {
            qa = ea[J];
            qb = eb[J];
            ej = edges[J];
        }
        sa[tid] = qa;
        sb[tid] = qb;
        se[tid] = ej;
        const double ex = qb.x - qa.x, ey = qb.y - qa.y, ez = qb.z - qa.z;
        const double re = sqrt(ex * ex + ey * ey + ez * ez);
        double4 h = make_double4(0, 0, 0, (1.0 - alpha) * pow(qa.w, -alpha));
        if (!(re < 1e-14)) {
            const double inv = 1.0 / re;
            h.x = inv * ex;
            h.y = inv * ey;
            h.z = inv * ez;
        }
        sh[tid] = h;
    }
    worker_sync(bar);
    const int32_t nt = min(kTile, E - bj * kTile);
    double g1[3] = {0, 0, 0}, g2[3] = {0, 0, 0};
    double en = 0.0;
    for (int32_t jj = 0; jj < nt; jj++) {
        const int2 ej = se[jj];
        const bool act = valid && (!diag || jj > (int32_t)tid) && disjoint(ei, ej);
        double cJ[6] = {0, 0, 0, 0, 0, 0};
        if (act) {
            const double4 qa = sa[jj], qb = sb[jj], hJ = sh[jj];
            const double eJx = qb.x - qa.x, eJy = qb.y - qa.y, eJz = qb.z - qa.z;
            const double ellJ = qa.w, powJ = qb.w;
            double sumF = 0.0, sumF2 = 0.0;
            double ownI[2][3] = {{0, 0, 0}, {0, 0, 0}}, othI[2][3] = {{0, 0, 0}, {0, 0, 0}};
            double ownJ[2][3] = {{0, 0, 0}, {0, 0, 0}}, othJ[2][3] = {{0, 0, 0}, {0, 0, 0}};
            double deI[3] = {0, 0, 0}, deJ[3] = {0, 0, 0};
#pragma unroll
            for (int s2 = 0; s2 < 4; s2++) {
                const int ai = s2 >> 1, bk = s2 & 1;
                const double px = ai ? b.x : a.x, py = ai ? b.y : a.y, pz = ai ? b.z : a.z;
                const double qx = bk ? qb.x : qa.x, qy = bk ? qb.y : qa.y, qz = bk ? qb.z : qa.z;
                const double dx = px - qx, dy = py - qy, dz = pz - qz;  // p_I - p_J
                double rd, inv, invDe;
                dist_terms(dx * dx + dy * dy + dz * dz, eps, rd, inv, invDe);
                const double hx = inv * dx, hy = inv * dy, hz = inv * dz;
                const double invDPowB = (MODE == 1) ? pow_b<1>(invDe, beta) : 1.0 / pow(rd + eps, beta);
                double ddIJ[3], deIJ[3], ddJI[3], deJI[3];
                sumF += kd_vec<MODE>(eIx, eIy, eIz, dx, dy, dz, hx, hy, hz, invDPowB, invDe, alpha,
                                     beta, eps, ddIJ, deIJ);
                sumF2 += kd_vec<MODE>(eJx, eJy, eJz, -dx, -dy, -dz, -hx, -hy, -hz, invDPowB, invDe,
                                      alpha, beta, eps, ddJI, deJI);
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    ownI[ai][q] += ddIJ[q];
                    othI[ai][q] += ddJI[q];
                    deI[q] += deIJ[q];
                    ownJ[bk][q] += ddJI[q];
                    othJ[bk][q] += ddIJ[q];
                    deJ[q] += deJI[q];
                }
            }
            const double baseIJ = 0.25 * powI * ellJ;  // weight of (I, J)
            const double baseJI = 0.25 * powJ * ellI;  // weight of (J, I)
            en += baseIJ * sumF + baseJI * sumF2;
            // I side (the edge-owner form's terms)
            const double tI = 0.25 * ellJ * sumF * dPowI;
            const double sI2 = 0.25 * powJ * sumF2;
            // J side, roles swapped
            const double tJ = 0.25 * ellI * sumF2 * hJ.w;
            const double sJ2 = 0.25 * powI * sumF;
            const double hI[3] = {hIx, hIy, hIz};
            const double hJv[3] = {hJ.x, hJ.y, hJ.z};
#pragma unroll
            for (int q = 0; q < 3; q++) {
                g1[q] += -tI * hI[q] + baseIJ * ownI[0][q] - baseJI * othI[0][q] - baseIJ * deI[q] -
                         sI2 * hI[q];
                g2[q] += tI * hI[q] + baseIJ * ownI[1][q] - baseJI * othI[1][q] + baseIJ * deI[q] +
                         sI2 * hI[q];
                cJ[q] = -tJ * hJv[q] + baseJI * ownJ[0][q] - baseIJ * othJ[0][q] - baseJI * deJ[q] -
                        sJ2 * hJv[q];
                cJ[3 + q] = tJ * hJv[q] + baseJI * ownJ[1][q] - baseIJ * othJ[1][q] +
                            baseJI * deJ[q] + sJ2 * hJv[q];
            }
        }
        if (__any_sync(0xffffffffu, act)) {
#pragma unroll
            for (int q = 0; q < 6; q++) cJ[q] = warp_sum(cJ[q]);
        }
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < 6; q++) accJ[warp][jj][q] = cJ[q];
        }
    }
    worker_sync(bar);
    // J side of this tile (fixed warp order), and on a diagonal tile the I side
    // of the same edge added to it
    {
        const int32_t J = bj * kTile + tid;
        if (J < E) {
            double v[6];
#pragma unroll
            for (int q = 0; q < 6; q++) {
                double t = 0.0;
                if ((int32_t)tid < nt)
                    for (int w = 0; w < kThreads / 32; w++) t += accJ[w][tid][q];
                v[q] = t;
            }
            if (diag) {
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    v[q] += g1[q];
                    v[3 + q] += g2[q];
                }
            }
            double* o = edge_acc + ((int64_t)bi * E + J) * 6;
#pragma unroll
            for (int q = 0; q < 6; q++) o[q] = v[q];
        }
        if (!diag && valid) {
            double* o = edge_acc + ((int64_t)bj * E + I) * 6;
            o[0] = g1[0];
            o[1] = g1[1];
            o[2] = g1[2];
            o[3] = g2[0];
            o[4] = g2[1];
            o[5] = g2[2];
        }
    }
    en = warp_sum(en);
    if (lane == 0) red[warp] = en;
    worker_sync(bar);
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; w++) t += red[w];
        partial[x] = t;
    }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads)
grad_sym_kernel(const double4* __restrict__ ea, const double4* __restrict__ eb,
                const int2* __restrict__ edges, int32_t E, double alpha, double beta, double eps,
                double* __restrict__ edge_acc, double* __restrict__ partial) {
    __shared__ GradSmem sm;
    grad_sym_tile<MODE>(blockIdx.x, threadIdx.x, 0, sm, ea, eb, edges, E, alpha, beta, eps,
                        edge_acc, partial);
}

// The same tiles on a bounded number of SMs: kGradWorkers independent 128-thread
// workers per block (one block per SM: the registers of three workers fill it)
// take tiles from a global counter until all ntiles are done. Every tile writes
// its own partial slots, so the result does not depend on which worker took it.
// Used for the gradient that runs beside the factorization, which then keeps
// the remaining SMs for its latency-bound chain.
constexpr int kGradWorkers = 3;

template <int MODE>
__global__ void __launch_bounds__(kThreads * kGradWorkers, 1)
grad_sym_persist_kernel(const double4* __restrict__ ea, const double4* __restrict__ eb,
                        const int2* __restrict__ edges, int32_t E, double alpha, double beta,
                        double eps, double* __restrict__ edge_acc, double* __restrict__ partial,
                        int32_t ntiles, int32_t* __restrict__ counter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w = threadIdx.x / kThreads, tid = threadIdx.x % kThreads;
    GradSmem& sm = reinterpret_cast<GradSmem*>(smem_raw)[w];
    __shared__ int next[kGradWorkers];
    for (;;) {
        if (tid == 0) next[w] = atomicAdd(counter, 1);
        worker_sync(1 + w);
        const int x = next[w];
        worker_sync(1 + w);
        if (x >= ntiles) break;
        grad_sym_tile<MODE>(x, tid, 1 + w, sm, ea, eb, edges, E, alpha, beta, eps, edge_acc,
                            partial);
    }
}

// grad[v] = 0.5 * sum over chunks and incident (edge, slot) of edge_acc.
__global__ void gather_vertex_grad(const double* __restrict__ edge_acc, int32_t nchunks,
                                   int32_t E, const int32_t* __restrict__ inc_off,
                                   const int32_t* __restrict__ inc, int32_t V,
                                   double* __restrict__ grad) {
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    double g[3] = {0, 0, 0};
    for (int32_t k = inc_off[v]; k < inc_off[v + 1]; k++) {
        const int32_t I = inc[k] >> 1, slot = inc[k] & 1;
        for (int32_t ch = 0; ch < nchunks; ch++) {
            const double* o = edge_acc + ((int64_t)ch * E + I) * 6 + 3 * slot;
            g[0] += o[0];
            g[1] += o[1];
            g[2] += o[2];
        }
    }
    grad[3 * v] = 0.5 * g[0];
    grad[3 * v + 1] = 0.5 * g[1];
    grad[3 * v + 2] = 0.5 * g[2];
}

inline int exp_mode(double alpha, double beta) { return (alpha == 3.0 && beta == 6.0) ? 1 : 0; }


}  // namespace

int32_t reduce_partials_launch(tpe_ctx* ctx, const double* partial, int32_t nparts, int32_t ncurves,
                               double scale, double* out) {
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    reduce_partials<<<ncurves, 256, 0, ctx->stream>>>(partial, nparts, scale, out);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t edge_prep(tpe_ctx* ctx, const double* d_pos, int32_t ncurves, double eps,
                  double alpha) {
    const int32_t E = ctx->E;
    TPE_TRY(ensure(ctx, ctx->edge_a, sizeof(double4) * (size_t)E * ncurves));
    TPE_TRY(ensure(ctx, ctx->edge_b, sizeof(double4) * (size_t)E * ncurves));
    const int64_t n = (int64_t)E * ncurves;
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    edge_prep_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(
        d_pos, ctx->d_edges.as<int2>(), E, ctx->V, ncurves, eps, alpha,
        ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>());
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t energy_fp64(tpe_ctx* ctx, int32_t ncurves, double alpha, double beta, double eps,
                    double* d_energy) {
    const int32_t E = ctx->E;
    const int32_t T = (E + kTile - 1) / kTile;
    const int32_t ntiles = T * (T + 1) / 2;
    TPE_TRY(ensure(ctx, ctx->partial, sizeof(double) * (size_t)ntiles * ncurves));
    dim3 grid(ntiles, 1, ncurves);
    KernelScope ks(ctx, TPE_KGROUP_ENERGY, 2);
    if (exp_mode(alpha, beta) == 1)
        energy_sym_kernel<1><<<grid, kThreads, 0, ctx->stream>>>(
            ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E,
            alpha, beta, eps, ctx->partial.as<double>());
    else
        energy_sym_kernel<0><<<grid, kThreads, 0, ctx->stream>>>(
            ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E,
            alpha, beta, eps, ctx->partial.as<double>());
    TPE_CUDA_TRY(cudaGetLastError());
    // total = sum over ordered pairs of 0.25 * l^(1-a) * l * sumK, halved
    reduce_partials<<<ncurves, 256, 0, ctx->stream>>>(ctx->partial.as<double>(), ntiles, 0.125,
                                                      d_energy);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

// Energy of one curve with caller-provided scratch (no context, no allocation):
// edge records ea/eb (E each), partial[max_parts] and one int flag *bad.
// Returns TPE_ERR_TOO_LARGE if the partials do not fit. The J range is split
// into at most 16 chunks. The caller's edge indices are checked on the device
// (this path has no host copy of them): an index outside [0, V) skips its
// loads, sets *bad, and the energy comes out NaN. Each launch is checked on its
// own; an error pending from the caller's earlier work is reported (and
// cleared) by the first check.
int32_t energy_fp64_scratch(cudaStream_t stream, const double* d_pos, const int2* d_edges,
                            int32_t V, int32_t E, double alpha, double beta, double eps,
                            double4* ea, double4* eb, double* partial, int32_t max_parts,
                            int32_t* bad, double* d_energy) {
    const int32_t xb = (E + kThreads - 1) / kThreads;
    int32_t ny = (E + kTile - 1) / kTile;
    ny = ny < 16 ? ny : 16;
    const int32_t jchunk = ((E + ny - 1) / ny + kTile - 1) / kTile * kTile;
    const int32_t nyy = (E + jchunk - 1) / jchunk;
    const int32_t nparts = xb * nyy;
    if (nparts > max_parts) return TPE_ERR_TOO_LARGE;
    if (cudaMemsetAsync(bad, 0, sizeof(int32_t), stream) != cudaSuccess) return TPE_ERR_CUDA;
    edge_prep_checked_kernel<<<(E + 255) / 256, 256, 0, stream>>>(d_pos, d_edges, E, V, eps, alpha,
                                                                  ea, eb, bad);
    if (cudaGetLastError() != cudaSuccess) return TPE_ERR_CUDA;
    dim3 grid(xb, nyy, 1);
    if (exp_mode(alpha, beta) == 1)
        energy_kernel<1><<<grid, kThreads, 0, stream>>>(ea, eb, d_edges, E, jchunk, alpha, beta,
                                                        eps, partial);
    else
        energy_kernel<0><<<grid, kThreads, 0, stream>>>(ea, eb, d_edges, E, jchunk, alpha, beta,
                                                        eps, partial);
    if (cudaGetLastError() != cudaSuccess) return TPE_ERR_CUDA;
    reduce_partials_checked<<<1, 256, 0, stream>>>(partial, nparts, 0.125, bad, d_energy);
    return cudaGetLastError() == cudaSuccess ? TPE_OK : TPE_ERR_CUDA;
}

int32_t energy_grad_fp64(tpe_ctx* ctx, double alpha, double beta, double eps, double* d_energy,
                         double* d_grad, int32_t max_blocks) {
    const int32_t E = ctx->E, V = ctx->V;
    const int32_t T = (E + kTile - 1) / kTile;
    const int32_t ntiles = T * (T + 1) / 2;
    TPE_TRY(ensure(ctx, ctx->edge_acc, sizeof(double) * 6 * (size_t)E * T));
    TPE_TRY(ensure(ctx, ctx->partial, sizeof(double) * (size_t)ntiles));
    KernelScope ks(ctx, TPE_KGROUP_GRADIENT, 1 + (d_grad ? 1 : 0) + (d_energy ? 1 : 0));
    const int mode = exp_mode(alpha, beta);
    if (max_blocks > 0) {
        TPE_TRY(ensure(ctx, ctx->grad_ctr, sizeof(int32_t)));
        TPE_CUDA_TRY(cudaMemsetAsync(ctx->grad_ctr.ptr, 0, sizeof(int32_t), ctx->stream));
        const size_t smem = sizeof(GradSmem) * kGradWorkers;
        const unsigned nb = (unsigned)std::min<int64_t>(max_blocks, (ntiles + kGradWorkers - 1) / kGradWorkers);
        auto kern = mode == 1 ? grad_sym_persist_kernel<1> : grad_sym_persist_kernel<0>;
        TPE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<nb, kThreads * kGradWorkers, smem, ctx->stream>>>(
            ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E, alpha,
            beta, eps, ctx->edge_acc.as<double>(), ctx->partial.as<double>(), ntiles,
            ctx->grad_ctr.as<int32_t>());
    } else if (mode == 1) {
        grad_sym_kernel<1><<<ntiles, kThreads, 0, ctx->stream>>>(
            ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E, alpha,
            beta, eps, ctx->edge_acc.as<double>(), ctx->partial.as<double>());
    } else {
        grad_sym_kernel<0><<<ntiles, kThreads, 0, ctx->stream>>>(
            ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E, alpha,
            beta, eps, ctx->edge_acc.as<double>(), ctx->partial.as<double>());
    }
    TPE_CUDA_TRY(cudaGetLastError());
    if (d_grad) {
        gather_vertex_grad<<<(V + 127) / 128, 128, 0, ctx->stream>>>(
            ctx->edge_acc.as<double>(), T, E, ctx->d_inc_off.as<int32_t>(),
            ctx->d_inc.as<int32_t>(), V, d_grad);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    if (d_energy) {
        // the partials already carry the 1/4 weight: halve for the ordered-pair sum
        reduce_partials<<<1, 256, 0, ctx->stream>>>(ctx->partial.as<double>(), ntiles, 0.5,
                                                    d_energy);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    return TPE_OK;
}

}  // namespace tpe
