// Mixed-precision energy: FP32 pair arithmetic, FP64 accumulation.
//
// Same sum as pair_kernels.cu's energy (calculateEnergy,
// tangentPointEnergy.ts:50-111), reached through tpe_energy_batch with
// TPE_PRECISION_MIXED as an explicitly lower-accuracy energy (the descent step
// keeps FP64 pair terms in every precision mode). Positions are stored as two floats per coordinate
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

}  // namespace tpe
