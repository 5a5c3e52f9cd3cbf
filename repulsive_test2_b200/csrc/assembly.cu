// Fractional-Sobolev Gram assembly, FP64: A = B + B0 (V x V).
//
// Reference: assembleBHighFlat / assembleBLowFlat / assembleAFlat in
// src/core/sobolev/innerProduct.ts:38-350. The reference scatters 16
// increments per ordered pair into V x V; here the same sum is written in
// matrix form and evaluated as two gathers, with no atomics:
//
//   B  = S (diag(d) - Mb) S^T,   S column I = e_{i1} - e_{i2}
//   B0 = U (diag(d0) - M0) U^T,  U column I = e_{i1} + e_{i2}
//
// with, for disjoint I != J (w_IJ = w_JI = 1/4 l_I l_J sum 1/(|d|+eps)^(2s+1),
// q_IJ = 1/4 * 1/4 l_I l_J sum (|T_I x d|+eps)^2/(|d|+eps)^4/(|d|+eps)^(2s+1)):
//   Mb[I][J] = (w_IJ + w_JI) (T_I . T_J) / (l_I l_J),   d_I  = sum_J (w_IJ + w_JI) / l_I^2
//   M0[I][J] = q_IJ + q_JI,                             d0_I = sum_J (q_IJ + q_JI)
// Kernel 1 writes the E x E pair matrix (Mb', M0') with the diagonal sums on
// its diagonal and minus signs folded in; kernel 2 forms each A[v][u] from the
// incident edges of v and u (4 entries for a closed polyline) and writes A and
// its mirror, so A is exactly symmetric as after the reference's explicit
// symmetrisation.
#include <math.h>

#include "tpe_internal.h"

namespace tpe {
namespace {

constexpr int kThreads = 128;
constexpr int kTile = 128;

__device__ __forceinline__ bool disjoint(int2 a, int2 b) {
    return a.x != b.x && a.x != b.y && a.y != b.x && a.y != b.y;
}

// (|d|+eps)^(-(2 sigma + 1)); MODE 1: alpha = 3, beta = 6 -> exponent 7/3.
template <int MODE>
__device__ __forceinline__ double inv_dist_pow(double dn, double distExp) {
    if (MODE == 1) return rcbrt(dn) / (dn * dn);
    return 1.0 / pow(dn, distExp);
}

template <int MODE>
__global__ void __launch_bounds__(kThreads)
pair_weights_kernel(const double4* __restrict__ ea, const double4* __restrict__ eb,
                    const int2* __restrict__ edges, int32_t E, double distExp, double eps,
                    double2* __restrict__ M) {
    __shared__ double4 sa[kTile], sb[kTile];
    __shared__ int2 se[kTile];
    const int32_t I = blockIdx.x * kThreads + threadIdx.x;
    const bool valid = I < E;
    double4 a = make_double4(0, 0, 0, 1), b = make_double4(0, 0, 0, 1);
    int2 ei = make_int2(-1, -1);
    if (valid) {
        a = ea[I];
        b = eb[I];
        ei = edges[I];
    }
    const double eIx = b.x - a.x, eIy = b.y - a.y, eIz = b.z - a.z;
    const double rI = sqrt(eIx * eIx + eIy * eIy + eIz * eIz);
    double TIx = 0, TIy = 0, TIz = 0;
    if (!(rI < 1e-14)) {
        const double inv = 1.0 / rI;
        TIx = eIx * inv;
        TIy = eIy * inv;
        TIz = eIz * inv;
    }
    const double ellI = a.w;
    double dsum = 0.0, d0sum = 0.0;
    double2* row = M + (int64_t)I * E;
    for (int32_t t0 = 0; t0 < E; t0 += kTile) {
        const int32_t nt = min(kTile, E - t0);
        __syncthreads();
        if (threadIdx.x < nt) {
            sa[threadIdx.x] = ea[t0 + threadIdx.x];
            sb[threadIdx.x] = eb[t0 + threadIdx.x];
            se[threadIdx.x] = edges[t0 + threadIdx.x];
        }
        __syncthreads();
        if (!valid) continue;
        for (int32_t jj = 0; jj < nt; jj++) {
            const int32_t J = t0 + jj;
            const int2 ej = se[jj];
            double2 out = make_double2(0.0, 0.0);
            if (J != I && disjoint(ei, ej)) {
                const double4 qa = sa[jj], qb = sb[jj];
                const double eJx = qb.x - qa.x, eJy = qb.y - qa.y, eJz = qb.z - qa.z;
                const double rJ = sqrt(eJx * eJx + eJy * eJy + eJz * eJz);
                double TJx = 0, TJy = 0, TJz = 0;
                if (!(rJ < 1e-14)) {
                    const double inv = 1.0 / rJ;
                    TJx = eJx * inv;
                    TJy = eJy * inv;
                    TJz = eJz * inv;
                }
                const double ellJ = qa.w;
                double sumDist = 0.0, sumLowIJ = 0.0, sumLowJI = 0.0;
#pragma unroll
                for (int s = 0; s < 4; s++) {
                    const int ai = s >> 1, bj = s & 1;
                    const double dx = (ai ? b.x : a.x) - (bj ? qb.x : qa.x);
                    const double dy = (ai ? b.y : a.y) - (bj ? qb.y : qa.y);
                    const double dz = (ai ? b.z : a.z) - (bj ? qb.z : qa.z);
                    const double dn = sqrt(dx * dx + dy * dy + dz * dz) + eps;
                    const double kd = inv_dist_pow<MODE>(dn, distExp);
                    sumDist += kd;
                    const double dn2 = dn * dn;
                    const double kq = kd / (dn2 * dn2);
                    double cx = TIy * dz - TIz * dy, cy = TIz * dx - TIx * dz,
                           cz = TIx * dy - TIy * dx;
                    double cn = sqrt(cx * cx + cy * cy + cz * cz) + eps;
                    sumLowIJ += cn * cn * kq;
                    cx = TJy * dz - TJz * dy;
                    cy = TJz * dx - TJx * dz;
                    cz = TJx * dy - TJy * dx;
                    cn = sqrt(cx * cx + cy * cy + cz * cz) + eps;
                    sumLowJI += cn * cn * kq;
                }
                const double ll = ellI * ellJ;
                const double w2 = 0.5 * ll * sumDist;             // w_IJ + w_JI
                const double q = 0.0625 * ll * (sumLowIJ + sumLowJI);  // q_IJ + q_JI
                const double dotT = TIx * TJx + TIy * TJy + TIz * TJz;
                dsum += w2;
                d0sum += q;
                out = make_double2(-w2 * dotT / ll, -q);
            }
            row[J] = out;
        }
    }
    if (valid) row[I] = make_double2(dsum / (ellI * ellI), d0sum);
}

// A[v][u] = sum_{(I,a) in inc(v)} sum_{(J,b) in inc(u)} (s_a s_b Mb'[I][J] + M0'[I][J]),
// s_0 = +1 (v is the edge's first vertex), s_1 = -1. Lower-triangle tiles only;
// each entry is written with its mirror.
__global__ void gather_A_kernel(const double2* __restrict__ M, int32_t E,
                                const int32_t* __restrict__ inc_off,
                                const int32_t* __restrict__ inc, int32_t V, int32_t tiles,
                                double* __restrict__ A, double* __restrict__ B,
                                double* __restrict__ B0) {
    // blockIdx.x enumerates lower-triangular 32x32 tiles (ti >= tj)
    const int32_t t = blockIdx.x;
    int32_t ti = (int32_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((int64_t)ti * (ti + 1) / 2 > t) ti--;
    while ((int64_t)(ti + 1) * (ti + 2) / 2 <= t) ti++;
    const int32_t tj = t - ti * (ti + 1) / 2;
    const int32_t v = ti * 32 + threadIdx.y;
    const int32_t u = tj * 32 + threadIdx.x;
    (void)tiles;
    if (v >= V || u >= V || u > v) return;
    double sb = 0.0, s0 = 0.0;
    for (int32_t p = inc_off[v]; p < inc_off[v + 1]; p++) {
        const int32_t I = inc[p] >> 1;
        const double sa = (inc[p] & 1) ? -1.0 : 1.0;
        const double2* row = M + (int64_t)I * E;
        for (int32_t q = inc_off[u]; q < inc_off[u + 1]; q++) {
            const int32_t J = inc[q] >> 1;
            const double sgn = (inc[q] & 1) ? -sa : sa;
            const double2 m = row[J];
            sb += sgn * m.x;
            s0 += m.y;
        }
    }
    const double a = sb + s0;
    A[(int64_t)v * V + u] = a;
    A[(int64_t)u * V + v] = a;
    if (B) {
        B[(int64_t)v * V + u] = sb;
        B[(int64_t)u * V + v] = sb;
    }
    if (B0) {
        B0[(int64_t)v * V + u] = s0;
        B0[(int64_t)u * V + v] = s0;
    }
}

}  // namespace

int32_t assemble_fp64(tpe_ctx* ctx, double alpha, double beta, double eps, double* d_A,
                      double* d_B, double* d_B0) {
    const int32_t E = ctx->E, V = ctx->V;
    TPE_TRY(ensure(ctx, ctx->pairM, sizeof(double2) * (size_t)E * E));
    const double s = (beta - 1.0) / alpha;
    const double sigma = s - 1.0;
    const double distExp = 2.0 * sigma + 1.0;
    const int mode = (alpha == 3.0 && beta == 6.0) ? 1 : 0;
    const int32_t xb = (E + kThreads - 1) / kThreads;
    {
    KernelScope ks(ctx, TPE_KGROUP_PAIR_WEIGHTS, 1);
    if (mode == 1)
        pair_weights_kernel<1><<<xb, kThreads, 0, ctx->stream>>>(
            ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E,
            distExp, eps, ctx->pairM.as<double2>());
    else
        pair_weights_kernel<0><<<xb, kThreads, 0, ctx->stream>>>(
            ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E,
            distExp, eps, ctx->pairM.as<double2>());
    TPE_CUDA_TRY(cudaGetLastError());
    }
    const int32_t nt = (V + 31) / 32;
    KernelScope ks(ctx, TPE_KGROUP_GATHER_A, 1);
    const int32_t tiles = nt * (nt + 1) / 2;
    gather_A_kernel<<<tiles, dim3(32, 32), 0, ctx->stream>>>(
        ctx->pairM.as<double2>(), E, ctx->d_inc_off.as<int32_t>(), ctx->d_inc.as<int32_t>(), V,
        tiles, d_A, d_B, d_B0);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

}  // namespace tpe
