// All-pairs tangent-point energy and its adjoint gradient, FP64.
//
// Reference: calculateEnergy / gradientAnalytical / kernelDerivs in
// src/core/tangentPointEnergy.ts:50-392. Ordered disjoint pairs (I, J) are
// never materialised: each thread owns one edge I, the J edges stream through
// shared memory in tiles, and disjointness is tested from endpoint indices.
//
// Gradient (adjoint) form: the thread that owns I accumulates every
// contribution that lands on I's endpoints -- from the ordered pair (I, J)
// (I first: the l_I^(1-a) chain, the d and e_I terms) and from (J, I) (I
// second: the l_I chain and the d terms). Pair terms are recomputed, nothing
// of size E^2 is stored, and no atomics are used (deterministic). The two
// orders share |d|, d_hat and (|d|+eps)^b.
#include <math.h>

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

// One kernelDerivs evaluation (tangentPointEnergy.ts:165-244) for edge vector e
// and a distance vector whose norm pieces are shared: returns f, adds the d
// derivative into dd and the e derivative into de (when DE).
template <int MODE, bool DE>
__device__ __forceinline__ double kernel_derivs(double ex, double ey, double ez, double dx,
                                                double dy, double dz, double hx, double hy,
                                                double hz, double invDPowB, double invDe,
                                                double alpha, double beta, double eps,
                                                double* dd, double* de) {
    const double cx = ey * dz - ez * dy;
    const double cy = ez * dx - ex * dz;
    const double cz = ex * dy - ey * dx;
    const double rc = sqrt(cx * cx + cy * cy + cz * cz);
    const double ce = rc + eps;
    const double cPowA = pow_a<MODE>(ce, alpha);
    const double f = cPowA * invDPowB;
    const double coeff_c = alpha * pow_a1<MODE>(ce, alpha) * invDPowB;
    const double coeff_d = -beta * f * invDe;
    double ux = 0, uy = 0, uz = 0, vx = 0, vy = 0, vz = 0;
    if (rc >= 1e-14) {
        const double inv = 1.0 / rc;
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

template <int MODE>
__global__ void __launch_bounds__(kThreads)
grad_kernel(const double4* __restrict__ ea, const double4* __restrict__ eb,
            const int2* __restrict__ edges, int32_t E, int32_t jchunk, double alpha, double beta,
            double eps, double* __restrict__ edge_acc, double* __restrict__ partial) {
    __shared__ double4 sa[kTile], sb[kTile];
    __shared__ int2 se[kTile];
    __shared__ double red[kThreads / 32];
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
    const double reI = sqrt(eIx * eIx + eIy * eIy + eIz * eIz);
    double hIx = 0, hIy = 0, hIz = 0;
    if (!(reI < 1e-14)) {
        const double inv = 1.0 / reI;
        hIx = inv * eIx;
        hIy = inv * eIy;
        hIz = inv * eIz;
    }
    const double ellI = a.w, powI = b.w;
    const double dPowCoeff = (1.0 - alpha) * pow(ellI, -alpha);
    double g1[3] = {0, 0, 0}, g2[3] = {0, 0, 0};
    double en = 0.0;
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
            if (!disjoint(ei, ej)) continue;
            const double4 qa = sa[jj], qb = sb[jj];
            const double eJx = qb.x - qa.x, eJy = qb.y - qa.y, eJz = qb.z - qa.z;
            const double ellJ = qa.w, powJ = qb.w;
            double sumF = 0.0, sumF2 = 0.0;
            double dd_own[2][3] = {{0, 0, 0}, {0, 0, 0}};  // (I,J): d-derivative at I endpoint a
            double dd_oth[2][3] = {{0, 0, 0}, {0, 0, 0}};  // (J,I): d-derivative landing on I endpoint a
            double de[3] = {0, 0, 0};
#pragma unroll
            for (int s = 0; s < 4; s++) {
                const int ai = s >> 1, bj = s & 1;
                const double px = ai ? b.x : a.x, py = ai ? b.y : a.y, pz = ai ? b.z : a.z;
                const double qx = bj ? qb.x : qa.x, qy = bj ? qb.y : qa.y, qz = bj ? qb.z : qa.z;
                const double dx = px - qx, dy = py - qy, dz = pz - qz;  // p_I - p_J
                const double rd = sqrt(dx * dx + dy * dy + dz * dz);
                double hx = 0, hy = 0, hz = 0;
                if (!(rd < 1e-14)) {
                    const double inv = 1.0 / rd;
                    hx = inv * dx;
                    hy = inv * dy;
                    hz = inv * dz;
                }
                const double invDe = 1.0 / (rd + eps);
                const double invDPowB = (MODE == 1) ? pow_b<1>(invDe, beta) : 1.0 / pow(rd + eps, beta);
                // (I, J): e = e_I, d = p_I - p_J
                sumF += kernel_derivs<MODE, true>(eIx, eIy, eIz, dx, dy, dz, hx, hy, hz, invDPowB,
                                                  invDe, alpha, beta, eps, dd_own[ai], de);
                // (J, I): e = e_J, d' = p_J - p_I = -d, d_hat' = -d_hat
                sumF2 += kernel_derivs<MODE, false>(eJx, eJy, eJz, -dx, -dy, -dz, -hx, -hy, -hz,
                                                    invDPowB, invDe, alpha, beta, eps, dd_oth[ai],
                                                    nullptr);
            }
            const double base = 0.25 * powI * ellJ;   // (I,J) weight
            const double base2 = 0.25 * powJ * ellI;  // (J,I) weight
            const double sI = 0.25 * ellJ * sumF;     // times d(l_I^(1-a))
            const double sJ2 = 0.25 * powJ * sumF2;   // times d(l_I) for (J,I)
            en += base * sumF;
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

// Number of J chunks so that the grid has roughly 4 blocks per SM.
inline int32_t pick_chunks(const tpe_ctx* ctx, int32_t E, int32_t ncurves) {
    const int32_t xb = (E + kThreads - 1) / kThreads;
    int32_t want = (4 * ctx->num_sms + xb * ncurves - 1) / (xb * ncurves);
    want = max(1, min(want, (E + kTile - 1) / kTile));
    return want;
}

}  // namespace

int32_t reduce_partials_launch(tpe_ctx* ctx, const double* partial, int32_t nparts, int32_t ncurves,
                               double scale, double* out) {
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    reduce_partials<<<ncurves, 256, 0, ctx->stream>>>(partial, nparts, scale, out);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t gather_vertex_grad_launch(tpe_ctx* ctx, const double* edge_acc, int32_t nchunks,
                                  double* grad) {
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    gather_vertex_grad<<<(ctx->V + 127) / 128, 128, 0, ctx->stream>>>(
        edge_acc, nchunks, ctx->E, ctx->d_inc_off.as<int32_t>(), ctx->d_inc.as<int32_t>(), ctx->V,
        grad);
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
    const int32_t xb = (E + kThreads - 1) / kThreads;
    const int32_t ny = pick_chunks(ctx, E, ncurves);
    const int32_t jchunk = ((E + ny - 1) / ny + kTile - 1) / kTile * kTile;
    const int32_t nyy = (E + jchunk - 1) / jchunk;
    const int32_t nparts = xb * nyy;
    TPE_TRY(ensure(ctx, ctx->partial, sizeof(double) * (size_t)nparts * ncurves));
    dim3 grid(xb, nyy, ncurves);
    KernelScope ks(ctx, TPE_KGROUP_ENERGY, 2);
    if (exp_mode(alpha, beta) == 1)
        energy_kernel<1><<<grid, kThreads, 0, ctx->stream>>>(
            ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E,
            jchunk, alpha, beta, eps, ctx->partial.as<double>());
    else
        energy_kernel<0><<<grid, kThreads, 0, ctx->stream>>>(
            ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E,
            jchunk, alpha, beta, eps, ctx->partial.as<double>());
    TPE_CUDA_TRY(cudaGetLastError());
    // total = sum(0.25 * l_I^(1-a) * l_J * sumK) / 2
    reduce_partials<<<ncurves, 256, 0, ctx->stream>>>(ctx->partial.as<double>(), nparts, 0.125,
                                                      d_energy);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

// Energy of one curve with caller-provided scratch (no context, no allocation):
// edge records ea/eb (E each) and partial[max_parts]. Returns TPE_ERR_TOO_LARGE if
// the partials do not fit. The J range is split into at most 16 chunks.
int32_t energy_fp64_scratch(cudaStream_t stream, const double* d_pos, const int2* d_edges,
                            int32_t V, int32_t E, double alpha, double beta, double eps,
                            double4* ea, double4* eb, double* partial, int32_t max_parts,
                            double* d_energy) {
    const int32_t xb = (E + kThreads - 1) / kThreads;
    int32_t ny = (E + kTile - 1) / kTile;
    ny = ny < 16 ? ny : 16;
    const int32_t jchunk = ((E + ny - 1) / ny + kTile - 1) / kTile * kTile;
    const int32_t nyy = (E + jchunk - 1) / jchunk;
    const int32_t nparts = xb * nyy;
    if (nparts > max_parts) return TPE_ERR_TOO_LARGE;
    edge_prep_kernel<<<(E + 255) / 256, 256, 0, stream>>>(d_pos, d_edges, E, V, 1, eps, alpha, ea,
                                                          eb);
    dim3 grid(xb, nyy, 1);
    if (exp_mode(alpha, beta) == 1)
        energy_kernel<1><<<grid, kThreads, 0, stream>>>(ea, eb, d_edges, E, jchunk, alpha, beta,
                                                        eps, partial);
    else
        energy_kernel<0><<<grid, kThreads, 0, stream>>>(ea, eb, d_edges, E, jchunk, alpha, beta,
                                                        eps, partial);
    reduce_partials<<<1, 256, 0, stream>>>(partial, nparts, 0.125, d_energy);
    return cudaGetLastError() == cudaSuccess ? TPE_OK : TPE_ERR_CUDA;
}

int32_t energy_grad_fp64(tpe_ctx* ctx, double alpha, double beta, double eps, double* d_energy,
                         double* d_grad) {
    const int32_t E = ctx->E, V = ctx->V;
    const int32_t xb = (E + kThreads - 1) / kThreads;
    const int32_t ny = pick_chunks(ctx, E, 1);
    const int32_t jchunk = ((E + ny - 1) / ny + kTile - 1) / kTile * kTile;
    const int32_t nyy = (E + jchunk - 1) / jchunk;
    TPE_TRY(ensure(ctx, ctx->edge_acc, sizeof(double) * 6 * (size_t)E * nyy));
    TPE_TRY(ensure(ctx, ctx->partial, sizeof(double) * (size_t)xb * nyy));
    dim3 grid(xb, nyy, 1);
    KernelScope ks(ctx, TPE_KGROUP_GRADIENT, 1 + (d_grad ? 1 : 0) + (d_energy ? 1 : 0));
    if (exp_mode(alpha, beta) == 1)
        grad_kernel<1><<<grid, kThreads, 0, ctx->stream>>>(
            ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E,
            jchunk, alpha, beta, eps, ctx->edge_acc.as<double>(), ctx->partial.as<double>());
    else
        grad_kernel<0><<<grid, kThreads, 0, ctx->stream>>>(
            ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E,
            jchunk, alpha, beta, eps, ctx->edge_acc.as<double>(), ctx->partial.as<double>());
    TPE_CUDA_TRY(cudaGetLastError());
    if (d_grad) {
        gather_vertex_grad<<<(V + 127) / 128, 128, 0, ctx->stream>>>(
            ctx->edge_acc.as<double>(), nyy, E, ctx->d_inc_off.as<int32_t>(),
            ctx->d_inc.as<int32_t>(), V, d_grad);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    if (d_energy) {
        reduce_partials<<<1, 256, 0, ctx->stream>>>(ctx->partial.as<double>(), xb * nyy, 0.5,
                                                    d_energy);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    return TPE_OK;
}

}  // namespace tpe
