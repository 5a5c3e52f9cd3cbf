// Mixed-precision all-pairs kernels: FP32 pair arithmetic, FP64 accumulation.
//
// Same sums as pair_kernels.cu / assembly.cu (tangentPointEnergy.ts:50-392,
// innerProduct.ts:38-350). Positions are stored as two floats per coordinate
// (hi = fl32(p), lo = fl32(p - hi)), so a difference of two nearby points,
// (hi_i - hi_j) + (lo_i - lo_j), keeps its full relative accuracy even when the
// points nearly touch (hi_i - hi_j is exact there). Per-pair terms use IEEE
// FP32 sqrt and division; every per-thread and per-tile sum is accumulated in
// FP64, so rounding does not grow with the number of pairs.
#include <math.h>

#include "tpe_internal.h"

namespace tpe {
namespace {

constexpr int kThreads = 128;
constexpr int kTile = 128;

// Edge record: a = (hi1, l^eps), b = (hi2, l^(1-alpha)), c = (lo1, -), d = (lo2, -).
struct MEdge {
    float4 a, b, c, d;
};

__device__ __forceinline__ bool disjoint(int2 a, int2 b) {
    return a.x != b.x && a.x != b.y && a.y != b.x && a.y != b.y;
}

__global__ void edge_prep_mixed_kernel(const double* __restrict__ pos,
                                       const int2* __restrict__ edges, int32_t E, int32_t V,
                                       int32_t ncurves, double eps, double alpha,
                                       MEdge* __restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)E * ncurves) return;
    const int32_t c = (int32_t)(t / E), I = (int32_t)(t % E);
    const double* p = pos + (int64_t)c * 3 * V;
    const int2 e = edges[I];
    double p1[3], p2[3];
    for (int q = 0; q < 3; q++) {
        p1[q] = p[3 * e.x + q];
        p2[q] = p[3 * e.y + q];
    }
    const double ex = p2[0] - p1[0], ey = p2[1] - p1[1], ez = p2[2] - p1[2];
    const double ell = sqrt(ex * ex + ey * ey + ez * ez) + eps;
    float h1[3], h2[3], l1[3], l2[3];
    for (int q = 0; q < 3; q++) {
        h1[q] = (float)p1[q];
        l1[q] = (float)(p1[q] - (double)h1[q]);
        h2[q] = (float)p2[q];
        l2[q] = (float)(p2[q] - (double)h2[q]);
    }
    MEdge m;
    m.a = make_float4(h1[0], h1[1], h1[2], (float)ell);
    m.b = make_float4(h2[0], h2[1], h2[2], (float)pow(ell, 1.0 - alpha));
    m.c = make_float4(l1[0], l1[1], l1[2], 0.0f);
    m.d = make_float4(l2[0], l2[1], l2[2], 0.0f);
    out[t] = m;
}

// p_I(ai) - p_J(bj) from two-float parts.
__device__ __forceinline__ void diff(const MEdge& I, const MEdge& J, int ai, int bj, float& dx,
                                     float& dy, float& dz) {
    const float4 hi = ai ? I.b : I.a, lo = ai ? I.d : I.c;
    const float4 hj = bj ? J.b : J.a, lj = bj ? J.d : J.c;
    dx = (hi.x - hj.x) + (lo.x - lj.x);
    dy = (hi.y - hj.y) + (lo.y - lj.y);
    dz = (hi.z - hj.z) + (lo.z - lj.z);
}

__device__ __forceinline__ void edge_vec(const MEdge& I, float& ex, float& ey, float& ez) {
    ex = (I.b.x - I.a.x) + (I.d.x - I.c.x);
    ey = (I.b.y - I.a.y) + (I.d.y - I.c.y);
    ez = (I.b.z - I.a.z) + (I.d.z - I.c.z);
}

template <int MODE>
__global__ void __launch_bounds__(kThreads)
energy_mixed_kernel(const MEdge* __restrict__ em, const int2* __restrict__ edges, int32_t E,
                    int32_t jchunk, float alpha, float beta, float eps,
                    double* __restrict__ partial) {
    __shared__ MEdge sj[kTile];
    __shared__ int2 se[kTile];
    __shared__ double red[kThreads / 32];
    const int32_t c = blockIdx.z;
    em += (int64_t)c * E;
    const int32_t I = blockIdx.x * kThreads + threadIdx.x;
    const bool valid = I < E;
    MEdge a;
    int2 ei = make_int2(-1, -1);
    if (valid) {
        a = em[I];
        ei = edges[I];
    } else {
        a.a = a.b = a.c = a.d = make_float4(0, 0, 0, 0);
    }
    float eIx, eIy, eIz;
    edge_vec(a, eIx, eIy, eIz);
    const float powI = a.b.w;
    double acc = 0.0;
    const int32_t j0 = blockIdx.y * jchunk, j1 = min(E, j0 + jchunk);
    for (int32_t t0 = j0; t0 < j1; t0 += kTile) {
        const int32_t nt = min(kTile, j1 - t0);
        __syncthreads();
        if (threadIdx.x < nt) {
            sj[threadIdx.x] = em[t0 + threadIdx.x];
            se[threadIdx.x] = edges[t0 + threadIdx.x];
        }
        __syncthreads();
        if (!valid) continue;
        for (int32_t jj = 0; jj < nt; jj++) {
            if (!disjoint(ei, se[jj])) continue;
            const MEdge& b = sj[jj];
            float sumK = 0.0f;
#pragma unroll
            for (int s = 0; s < 4; s++) {
                float dx, dy, dz;
                diff(a, b, s >> 1, s & 1, dx, dy, dz);
                const float invDn = 1.0f / (sqrtf(dx * dx + dy * dy + dz * dz) + eps);
                const float cx = eIy * dz - eIz * dy;
                const float cy = eIz * dx - eIx * dz;
                const float cz = eIx * dy - eIy * dx;
                const float cn = sqrtf(cx * cx + cy * cy + cz * cz) + eps;
                if (MODE == 1) {
                    // (|c|/|d|)^3 |d|^-3 keeps every intermediate inside the FP32 range
                    const float t = cn * invDn, i3 = invDn * invDn * invDn;
                    sumK += (t * t * t) * i3;
                } else {
                    sumK += powf(cn, alpha) * powf(invDn, beta);
                }
            }
            acc += (double)(powI * b.a.w * sumK);
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; w++) s += red[w];
        partial[((int64_t)c * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
    }
}

template <int MODE, bool DE>
__device__ __forceinline__ float kderiv32(float ex, float ey, float ez, float dx, float dy,
                                          float dz, float hx, float hy, float hz, float invDPowB,
                                          float invDe, float alpha, float beta, float eps,
                                          float* dd, float* de) {
    const float cx = ey * dz - ez * dy;
    const float cy = ez * dx - ex * dz;
    const float cz = ex * dy - ey * dx;
    const float rc = sqrtf(cx * cx + cy * cy + cz * cz);
    const float ce = rc + eps;
    float f, coeff_c;
    if (MODE == 1) {
        // f = (ce/de)^3 de^-3, coeff_c = 3 ce^2 de^-6 = 3 (ce/de)^2 de^-4
        const float t = ce * invDe, i2 = invDe * invDe;
        f = (t * t * t) * (i2 * invDe);
        coeff_c = alpha * (t * t) * (i2 * i2);
    } else {
        f = powf(ce, alpha) * invDPowB;
        coeff_c = alpha * powf(ce, alpha - 1.0f) * invDPowB;
    }
    const float coeff_d = -beta * f * invDe;
    float ux = 0, uy = 0, uz = 0, vx = 0, vy = 0, vz = 0;
    if (rc >= 1e-14f) {
        const float inv = 1.0f / rc;
        ux = inv * (cy * ez - cz * ey);
        uy = inv * (cz * ex - cx * ez);
        uz = inv * (cx * ey - cy * ex);
        if (DE) {
            vx = inv * (dy * cz - dz * cy);
            vy = inv * (dz * cx - dx * cz);
            vz = inv * (dx * cy - dy * cx);
        }
    }
    dd[0] += coeff_c * ux + coeff_d * hx;
    dd[1] += coeff_c * uy + coeff_d * hy;
    dd[2] += coeff_c * uz + coeff_d * hz;
    if (DE) {
        de[0] += coeff_c * vx;
        de[1] += coeff_c * vy;
        de[2] += coeff_c * vz;
    }
    return f;
}

// Adjoint gradient, same ordering as grad_kernel (pair_kernels.cu): the thread
// that owns I gathers every contribution landing on I's endpoints from (I,J)
// and (J,I); pair terms in FP32, the per-pair combination and the running
// sums in FP64.
template <int MODE>
__global__ void __launch_bounds__(kThreads)
grad_mixed_kernel(const MEdge* __restrict__ em, const int2* __restrict__ edges, int32_t E,
                  int32_t jchunk, float alpha, float beta, float eps,
                  double* __restrict__ edge_acc, double* __restrict__ partial) {
    __shared__ MEdge sj[kTile];
    __shared__ int2 se[kTile];
    __shared__ double red[kThreads / 32];
    const int32_t I = blockIdx.x * kThreads + threadIdx.x;
    const bool valid = I < E;
    MEdge a;
    int2 ei = make_int2(-1, -1);
    if (valid) {
        a = em[I];
        ei = edges[I];
    } else {
        a.a = a.b = a.c = a.d = make_float4(0, 0, 0, 1);
    }
    float eIx, eIy, eIz;
    edge_vec(a, eIx, eIy, eIz);
    const float reI = sqrtf(eIx * eIx + eIy * eIy + eIz * eIz);
    float hIx = 0, hIy = 0, hIz = 0;
    if (!(reI < 1e-14f)) {
        const float inv = 1.0f / reI;
        hIx = inv * eIx;
        hIy = inv * eIy;
        hIz = inv * eIz;
    }
    const double ellI = a.a.w, powI = a.b.w;
    const double dPowCoeff = (1.0 - (double)alpha) * pow(ellI, -(double)alpha);
    double g1[3] = {0, 0, 0}, g2[3] = {0, 0, 0};
    double en = 0.0;
    const int32_t j0 = blockIdx.y * jchunk, j1 = min(E, j0 + jchunk);
    for (int32_t t0 = j0; t0 < j1; t0 += kTile) {
        const int32_t nt = min(kTile, j1 - t0);
        __syncthreads();
        if (threadIdx.x < nt) {
            sj[threadIdx.x] = em[t0 + threadIdx.x];
            se[threadIdx.x] = edges[t0 + threadIdx.x];
        }
        __syncthreads();
        if (!valid) continue;
        for (int32_t jj = 0; jj < nt; jj++) {
            if (!disjoint(ei, se[jj])) continue;
            const MEdge& b = sj[jj];
            float eJx, eJy, eJz;
            edge_vec(b, eJx, eJy, eJz);
            float sumF = 0.0f, sumF2 = 0.0f;
            float dd_own[2][3] = {{0, 0, 0}, {0, 0, 0}};
            float dd_oth[2][3] = {{0, 0, 0}, {0, 0, 0}};
            float de[3] = {0, 0, 0};
#pragma unroll
            for (int s = 0; s < 4; s++) {
                const int ai = s >> 1, bj = s & 1;
                float dx, dy, dz;
                diff(a, b, ai, bj, dx, dy, dz);
                const float rd = sqrtf(dx * dx + dy * dy + dz * dz);
                float hx = 0, hy = 0, hz = 0;
                if (!(rd < 1e-14f)) {
                    const float inv = 1.0f / rd;
                    hx = inv * dx;
                    hy = inv * dy;
                    hz = inv * dz;
                }
                const float invDe = 1.0f / (rd + eps);
                const float invDPowB = (MODE == 1) ? 0.0f : powf(invDe, beta);
                sumF += kderiv32<MODE, true>(eIx, eIy, eIz, dx, dy, dz, hx, hy, hz, invDPowB, invDe,
                                             alpha, beta, eps, dd_own[ai], de);
                sumF2 += kderiv32<MODE, false>(eJx, eJy, eJz, -dx, -dy, -dz, -hx, -hy, -hz,
                                               invDPowB, invDe, alpha, beta, eps, dd_oth[ai],
                                               nullptr);
            }
            const double ellJ = b.a.w, powJ = b.b.w;
            const double base = 0.25 * powI * ellJ;
            const double base2 = 0.25 * powJ * ellI;
            const double sI = 0.25 * ellJ * (double)sumF;
            const double sJ2 = 0.25 * powJ * (double)sumF2;
            en += base * (double)sumF;
            const double t1 = sI * dPowCoeff;
#pragma unroll
            for (int q = 0; q < 3; q++) {
                const double h = (q == 0) ? hIx : (q == 1) ? hIy : hIz;
                g1[q] += -t1 * h + base * dd_own[0][q] - base2 * dd_oth[0][q] - base * de[q] -
                         sJ2 * h;
                g2[q] += t1 * h + base * dd_own[1][q] - base2 * dd_oth[1][q] + base * de[q] +
                         sJ2 * h;
            }
        }
    }
    if (valid) {
        double* o = edge_acc + ((int64_t)blockIdx.y * E + I) * 6;
        o[0] = g1[0];
        o[1] = g1[1];
        o[2] = g1[2];
        o[3] = g2[0];
        o[4] = g2[1];
        o[5] = g2[2];
    }
    for (int o = 16; o > 0; o >>= 1) en += __shfl_down_sync(0xffffffffu, en, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = en;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; w++) s += red[w];
        partial[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
}

inline int exp_mode(double alpha, double beta) { return (alpha == 3.0 && beta == 6.0) ? 1 : 0; }

inline int32_t pick_chunks(const tpe_ctx* ctx, int32_t E, int32_t ncurves) {
    const int32_t xb = (E + kThreads - 1) / kThreads;
    int32_t want = (4 * ctx->num_sms + xb * ncurves - 1) / (xb * ncurves);
    want = max(1, min(want, (E + kTile - 1) / kTile));
    return want;
}

}  // namespace

// Reductions shared with the FP64 path (pair_kernels.cu).
int32_t reduce_partials_launch(tpe_ctx* ctx, const double* partial, int32_t nparts, int32_t ncurves,
                               double scale, double* out);
int32_t gather_vertex_grad_launch(tpe_ctx* ctx, const double* edge_acc, int32_t nchunks,
                                  double* grad);

int32_t edge_prep_mixed(tpe_ctx* ctx, const double* d_pos, int32_t ncurves, double eps,
                        double alpha) {
    const int32_t E = ctx->E;
    TPE_TRY(ensure(ctx, ctx->edge_m, sizeof(MEdge) * (size_t)E * ncurves));
    const int64_t n = (int64_t)E * ncurves;
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    edge_prep_mixed_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(
        d_pos, ctx->d_edges.as<int2>(), E, ctx->V, ncurves, eps, alpha, ctx->edge_m.as<MEdge>());
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t energy_mixed(tpe_ctx* ctx, int32_t ncurves, double alpha, double beta, double eps,
                     double* d_energy) {
    const int32_t E = ctx->E;
    const int32_t xb = (E + kThreads - 1) / kThreads;
    const int32_t ny = pick_chunks(ctx, E, ncurves);
    const int32_t jchunk = ((E + ny - 1) / ny + kTile - 1) / kTile * kTile;
    const int32_t nyy = (E + jchunk - 1) / jchunk;
    const int32_t nparts = xb * nyy;
    TPE_TRY(ensure(ctx, ctx->partial, sizeof(double) * (size_t)nparts * ncurves));
    dim3 grid(xb, nyy, ncurves);
    {
        KernelScope ks(ctx, TPE_KGROUP_ENERGY, 1);
        if (exp_mode(alpha, beta) == 1)
            energy_mixed_kernel<1><<<grid, kThreads, 0, ctx->stream>>>(
                ctx->edge_m.as<MEdge>(), ctx->d_edges.as<int2>(), E, jchunk, (float)alpha,
                (float)beta, (float)eps, ctx->partial.as<double>());
        else
            energy_mixed_kernel<0><<<grid, kThreads, 0, ctx->stream>>>(
                ctx->edge_m.as<MEdge>(), ctx->d_edges.as<int2>(), E, jchunk, (float)alpha,
                (float)beta, (float)eps, ctx->partial.as<double>());
        TPE_CUDA_TRY(cudaGetLastError());
    }
    return reduce_partials_launch(ctx, ctx->partial.as<double>(), nparts, ncurves, 0.125, d_energy);
}

int32_t energy_grad_mixed(tpe_ctx* ctx, double alpha, double beta, double eps, double* d_energy,
                          double* d_grad) {
    const int32_t E = ctx->E;
    const int32_t xb = (E + kThreads - 1) / kThreads;
    const int32_t ny = pick_chunks(ctx, E, 1);
    const int32_t jchunk = ((E + ny - 1) / ny + kTile - 1) / kTile * kTile;
    const int32_t nyy = (E + jchunk - 1) / jchunk;
    TPE_TRY(ensure(ctx, ctx->edge_acc, sizeof(double) * 6 * (size_t)E * nyy));
    TPE_TRY(ensure(ctx, ctx->partial, sizeof(double) * (size_t)xb * nyy));
    dim3 grid(xb, nyy, 1);
    {
        KernelScope ks(ctx, TPE_KGROUP_GRADIENT, 1);
        if (exp_mode(alpha, beta) == 1)
            grad_mixed_kernel<1><<<grid, kThreads, 0, ctx->stream>>>(
                ctx->edge_m.as<MEdge>(), ctx->d_edges.as<int2>(), E, jchunk, (float)alpha,
                (float)beta, (float)eps, ctx->edge_acc.as<double>(), ctx->partial.as<double>());
        else
            grad_mixed_kernel<0><<<grid, kThreads, 0, ctx->stream>>>(
                ctx->edge_m.as<MEdge>(), ctx->d_edges.as<int2>(), E, jchunk, (float)alpha,
                (float)beta, (float)eps, ctx->edge_acc.as<double>(), ctx->partial.as<double>());
        TPE_CUDA_TRY(cudaGetLastError());
    }
    if (d_grad) TPE_TRY(gather_vertex_grad_launch(ctx, ctx->edge_acc.as<double>(), nyy, d_grad));
    if (d_energy)
        TPE_TRY(reduce_partials_launch(ctx, ctx->partial.as<double>(), xb * nyy, 1, 0.5, d_energy));
    return TPE_OK;
}

// ---- Gram pair weights -----------------------------------------------------------

namespace {

constexpr int kT = 32;

struct MRec {
    float4 h1, h2, l1, l2;  // two-float endpoints; h1.w = l^eps
    float4 T;               // unit tangent (0 below 1e-14)
    int2 ij;
};

__device__ __forceinline__ void load_mrec(const MEdge* __restrict__ em, const int2* __restrict__ edges,
                                          int32_t E, int32_t I, MRec& r) {
    if (I >= E) {
        r.h1 = r.h2 = r.l1 = r.l2 = make_float4(0, 0, 0, 1);
        r.T = make_float4(0, 0, 0, 0);
        r.ij = make_int2(-1, -1);
        return;
    }
    const MEdge m = em[I];
    r.h1 = m.a;
    r.h2 = m.b;
    r.l1 = m.c;
    r.l2 = m.d;
    r.ij = edges[I];
    float ex, ey, ez;
    edge_vec(m, ex, ey, ez);
    const float len = sqrtf(ex * ex + ey * ey + ez * ez);
    if (len < 1e-14f) {
        r.T = make_float4(0, 0, 0, 0);
    } else {
        const float inv = 1.0f / len;
        r.T = make_float4(ex * inv, ey * inv, ez * inv, 0);
    }
}

template <int MODE>
__device__ __forceinline__ float inv_dist_pow32(float dn, float distExp) {
    if (MODE == 1) return 1.0f / (dn * dn * cbrtf(dn));
    return 1.0f / powf(dn, distExp);
}

template <int MODE>
__global__ void __launch_bounds__(256)
pair_weights_mixed_kernel(const MEdge* __restrict__ em, const int2* __restrict__ edges, int32_t E,
                          float distExp, float eps, double2* __restrict__ M,
                          double2* __restrict__ rowpart) {
    __shared__ MRec sI[kT], sJ[kT];
    __shared__ double2 tile[kT][kT + 1];
    __shared__ double2 colred[8][kT];
    const int64_t t = blockIdx.x;
    int32_t it = (int32_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((int64_t)it * (it + 1) / 2 > t) it--;
    while ((int64_t)(it + 1) * (it + 2) / 2 <= t) it++;
    const int32_t ti = (int32_t)(t - (int64_t)it * (it + 1) / 2), tj = it;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    if (threadIdx.x < kT) load_mrec(em, edges, E, ti * kT + threadIdx.x, sI[threadIdx.x]);
    else if (threadIdx.x < 2 * kT)
        load_mrec(em, edges, E, tj * kT + threadIdx.x - kT, sJ[threadIdx.x - kT]);
    __syncthreads();
    const int32_t J = tj * kT + tx;
    const MRec& b = sJ[tx];
    double2 colsum = make_double2(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int li = ty + 8 * r;
        const int32_t I = ti * kT + li;
        const MRec& a = sI[li];
        double2 out = make_double2(0.0, 0.0);
        double2 w = make_double2(0.0, 0.0);
        const bool ok = I < E && J < E && I != J && a.ij.x != b.ij.x && a.ij.x != b.ij.y &&
                        a.ij.y != b.ij.x && a.ij.y != b.ij.y;
        if (ok) {
            float sumDist = 0.0f, sumLowIJ = 0.0f, sumLowJI = 0.0f;
#pragma unroll
            for (int s = 0; s < 4; s++) {
                const int ai = s >> 1, bj = s & 1;
                const float4 hi = ai ? a.h2 : a.h1, lo = ai ? a.l2 : a.l1;
                const float4 hj = bj ? b.h2 : b.h1, lj = bj ? b.l2 : b.l1;
                const float dx = (hi.x - hj.x) + (lo.x - lj.x);
                const float dy = (hi.y - hj.y) + (lo.y - lj.y);
                const float dz = (hi.z - hj.z) + (lo.z - lj.z);
                const float dn = sqrtf(dx * dx + dy * dy + dz * dz) + eps;
                const float kd = inv_dist_pow32<MODE>(dn, distExp);
                sumDist += kd;
                const float dn2 = dn * dn;
                const float kq = kd / (dn2 * dn2);
                float cx = a.T.y * dz - a.T.z * dy, cy = a.T.z * dx - a.T.x * dz,
                      cz = a.T.x * dy - a.T.y * dx;
                float cn = sqrtf(cx * cx + cy * cy + cz * cz) + eps;
                sumLowIJ += cn * cn * kq;
                cx = b.T.y * dz - b.T.z * dy;
                cy = b.T.z * dx - b.T.x * dz;
                cz = b.T.x * dy - b.T.y * dx;
                cn = sqrtf(cx * cx + cy * cy + cz * cz) + eps;
                sumLowJI += cn * cn * kq;
            }
            const double ll = (double)a.h1.w * (double)b.h1.w;
            w = make_double2(0.5 * ll * (double)sumDist, 0.0625 * ll * ((double)sumLowIJ + sumLowJI));
            const double dotT = (double)(a.T.x * b.T.x + a.T.y * b.T.y + a.T.z * b.T.z);
            out = make_double2(-w.x * dotT / ll, -w.y);
        }
        if (I < E && J < E) M[(int64_t)I * E + J] = out;
        tile[li][tx] = out;
        colsum.x += w.x;
        colsum.y += w.y;
        double2 rs = w;
        for (int o = 16; o > 0; o >>= 1) {
            rs.x += __shfl_down_sync(0xffffffffu, rs.x, o);
            rs.y += __shfl_down_sync(0xffffffffu, rs.y, o);
        }
        if (tx == 0 && I < E) rowpart[(int64_t)tj * E + I] = rs;
    }
    if (ti == tj) return;
    colred[ty][tx] = colsum;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int lj = ty + 8 * r;
        const int32_t Jr = tj * kT + lj;
        const int32_t Ic = ti * kT + tx;
        if (Jr < E && Ic < E) M[(int64_t)Jr * E + Ic] = tile[tx][lj];
    }
    if (ty == 0 && J < E) {
        double2 s = colred[0][tx];
        for (int g = 1; g < 8; g++) {
            s.x += colred[g][tx].x;
            s.y += colred[g][tx].y;
        }
        rowpart[(int64_t)ti * E + J] = s;
    }
}

}  // namespace

namespace {
__global__ void pair_diag_mixed_kernel(const MEdge* __restrict__ em, int32_t E, int32_t nt,
                                       const double2* __restrict__ rowpart,
                                       double2* __restrict__ M) {
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= E) return;
    double sx = 0.0, sy = 0.0;
    for (int32_t s = 0; s < nt; s++) {
        const double2 p = rowpart[(int64_t)s * E + I];
        sx += p.x;
        sy += p.y;
    }
    const double ell = em[I].a.w;
    M[(int64_t)I * E + I] = make_double2(sx / (ell * ell), sy);
}
}  // namespace

int32_t gather_A_launch(tpe_ctx* ctx, double* d_A, double* d_B, double* d_B0);

int32_t pair_weights_mixed(tpe_ctx* ctx, double alpha, double beta, double eps, int32_t* ntp_out) {
    const int32_t E = ctx->E;
    TPE_TRY(ensure(ctx, ctx->pairM, sizeof(double2) * (size_t)E * E));
    const double s = (beta - 1.0) / alpha;
    const double distExp = 2.0 * (s - 1.0) + 1.0;
    const int32_t ntp = (E + kT - 1) / kT;
    TPE_TRY(ensure(ctx, ctx->tmp, sizeof(double2) * (size_t)ntp * E));
    const int64_t tiles = (int64_t)ntp * (ntp + 1) / 2;
    KernelScope ks(ctx, TPE_KGROUP_PAIR_WEIGHTS, 1);
    if (exp_mode(alpha, beta) == 1)
        pair_weights_mixed_kernel<1><<<(unsigned)tiles, 256, 0, ctx->stream>>>(
            ctx->edge_m.as<MEdge>(), ctx->d_edges.as<int2>(), E, (float)distExp, (float)eps,
            ctx->pairM.as<double2>(), ctx->tmp.as<double2>());
    else
        pair_weights_mixed_kernel<0><<<(unsigned)tiles, 256, 0, ctx->stream>>>(
            ctx->edge_m.as<MEdge>(), ctx->d_edges.as<int2>(), E, (float)distExp, (float)eps,
            ctx->pairM.as<double2>(), ctx->tmp.as<double2>());
    TPE_CUDA_TRY(cudaGetLastError());
    *ntp_out = ntp;
    return TPE_OK;
}

// A = B + B0 (FP64) from FP32 pair weights; edge records already prepared.
int32_t assemble_mixed(tpe_ctx* ctx, double alpha, double beta, double eps, double* d_A) {
    int32_t ntp = 0;
    TPE_TRY(pair_weights_mixed(ctx, alpha, beta, eps, &ntp));
    {
        KernelScope ks(ctx, TPE_KGROUP_PAIR_WEIGHTS, 1);
        pair_diag_mixed_kernel<<<(ctx->E + 255) / 256, 256, 0, ctx->stream>>>(
            ctx->edge_m.as<MEdge>(), ctx->E, ntp, ctx->tmp.as<double2>(), ctx->pairM.as<double2>());
        TPE_CUDA_TRY(cudaGetLastError());
    }
    return gather_A_launch(ctx, d_A, nullptr, nullptr);
}

}  // namespace tpe
