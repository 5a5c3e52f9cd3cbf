// Constraint rows and soft penalties on the device, FP64.
//
// Reference: barycenterPhiAndC (src/core/sobolev/constraints.ts:67-120),
// totalLengthBlock / edgeLengthsBlock / pointBlock and their scale()
// (src/core/sobolev/constraintSet.ts:119-301), barycenterScale
// (src/core/sobolev/lineSearch.ts:86-109), penaltyEnergy / penaltyGradient
// (src/core/sobolev/penalties.ts:139-241). Raw edge lengths (no epsilon),
// unit tangents zeroed below 1e-14, NaN rows for a missing target.
// Jacobian columns are gathered per vertex over its incident edges in
// ascending edge order (the order the reference accumulates in), so no two
// threads write the same entry.
#include <math.h>

#include "tpe_internal.h"

namespace tpe {
namespace {

constexpr int kBS = 512;

// Math.max semantics: NaN if either argument is NaN.
__device__ __forceinline__ double js_max(double a, double b) {
    if (a != a || b != b) return NAN;
    return a > b ? a : b;
}

struct EdgeGeo {
    double ell, T[3], rvec[3];
};

__device__ __forceinline__ void edge_geo(const double* __restrict__ pos, int2 e, EdgeGeo& g,
                                         const double* x0) {
    const double ex = pos[3 * e.y] - pos[3 * e.x];
    const double ey = pos[3 * e.y + 1] - pos[3 * e.x + 1];
    const double ez = pos[3 * e.y + 2] - pos[3 * e.x + 2];
    g.ell = sqrt(ex * ex + ey * ey + ez * ez);
    if (g.ell < 1e-14) {
        g.T[0] = g.T[1] = g.T[2] = 0.0;
    } else {
        const double inv = 1.0 / g.ell;
        g.T[0] = ex * inv;
        g.T[1] = ey * inv;
        g.T[2] = ez * inv;
    }
    if (x0)
        for (int r = 0; r < 3; r++) g.rvec[r] = 0.5 * (pos[3 * e.x + r] + pos[3 * e.y + r]) - x0[r];
}

template <int N>
__device__ void block_reduce(double (&v)[N], bool is_max_last) {
    __shared__ double red[kBS / 32][8];
    for (int q = 0; q < N; q++)
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = (is_max_last && q == N - 1) ? js_max(v[q], w) : v[q] + w;
        }
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < N; q++) red[threadIdx.x >> 5][q] = v[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < N; q++) v[q] = red[0][q];
        for (int w = 1; w < kBS / 32; w++)
            for (int q = 0; q < N; q++)
                v[q] = (is_max_last && q == N - 1) ? js_max(v[q], red[w][q]) : v[q] + red[w][q];
    }
    __syncthreads();
}

// The constraint rows phi and, per block b, ns[2b] = ||phi_b||^2 and
// ns[2b+1] = scale_b, for position set y (idx[y], or y). kPhiSplit CTAs per
// (block, position set): CTA s takes the edges (or vertices)
// [s E / S, (s+1) E / S) and leaves its reductions in
// part[((y * nblocks + b) * S + s) * 5 + q]; edge-length rows are written
// directly. phi_final_kernel then combines the S partials in order (sums in
// order, the maxima by Math.max) and writes the block rows, norms and scales.
constexpr int kPhiSplit = 16;

__global__ void __launch_bounds__(kBS)
phi_part_kernel(const double* __restrict__ pos, const int2* __restrict__ edges, int32_t E,
                int32_t V, const DevBlock* __restrict__ blocks, double* __restrict__ phi,
                int64_t pos_stride, const int32_t* __restrict__ idx, int32_t k,
                double* __restrict__ part) {
    const DevBlock B = blocks[blockIdx.x];
    const int32_t y = blockIdx.y, sp = blockIdx.z;
    pos += (idx ? idx[y] : y) * pos_stride;
    phi += (size_t)y * k;
    double* out = part + ((size_t)(y * gridDim.x + blockIdx.x) * kPhiSplit + sp) * 5;
    const int32_t n = B.kind == TPE_BLOCK_POINT ? V : E;
    const int32_t lo = (int32_t)((int64_t)n * sp / kPhiSplit);
    const int32_t hi = (int32_t)((int64_t)n * (sp + 1) / kPhiSplit);
    if (B.kind == TPE_BLOCK_BARYCENTER) {
        double v[5] = {0, 0, 0, 0, 0};
        for (int32_t I = lo + threadIdx.x; I < hi; I += kBS) {
            const int2 e = edges[I];
            EdgeGeo g;
            edge_geo(pos, e, g, B.target);
            for (int r = 0; r < 3; r++) v[r] += g.ell * g.rvec[r];
            v[3] += g.ell;
            double d1 = 0, d2 = 0;
            for (int r = 0; r < 3; r++) {
                const double a = pos[3 * e.x + r] - B.target[r];
                const double b = pos[3 * e.y + r] - B.target[r];
                d1 += a * a;
                d2 += b * b;
            }
            v[4] = js_max(js_max(v[4], sqrt(d1)), sqrt(d2));
        }
        block_reduce<5>(v, true);
        if (threadIdx.x == 0)
            for (int q = 0; q < 5; q++) out[q] = v[q];
    } else if (B.kind == TPE_BLOCK_TOTAL_LENGTH || B.kind == TPE_BLOCK_EDGE_LENGTHS) {
        double v[2] = {0, 0};
        for (int32_t I = lo + threadIdx.x; I < hi; I += kBS) {
            const int2 e = edges[I];
            EdgeGeo g;
            edge_geo(pos, e, g, nullptr);
            v[0] += g.ell;
            if (B.kind == TPE_BLOCK_EDGE_LENGTHS) {
                const double p = B.ell0[I] - g.ell;
                phi[B.row0 + I] = p;
                v[1] += p * p;
            }
        }
        block_reduce<2>(v, false);
        if (threadIdx.x == 0) {
            out[0] = v[0];
            out[1] = v[1];
        }
    } else if (B.kind == TPE_BLOCK_POINT) {
        double v[1] = {0};
        for (int32_t i = lo + threadIdx.x; i < hi; i += kBS) {
            double d = 0;
            for (int r = 0; r < 3; r++) {
                const double a = pos[3 * i + r] - B.target[r];
                d += a * a;
            }
            v[0] = js_max(v[0], sqrt(d));
        }
        block_reduce<1>(v, true);
        if (threadIdx.x == 0) out[0] = v[0];
    }
}

// One thread per (block, position set): the partials of phi_part_kernel in
// order, then the block's rows, squared norm and scale.
__global__ void phi_final_kernel(const double* __restrict__ pos, int32_t V,
                                 const DevBlock* __restrict__ blocks, int32_t nblocks,
                                 double* __restrict__ phi, double* __restrict__ ns,
                                 int64_t pos_stride, const int32_t* __restrict__ idx, int32_t k,
                                 int32_t n, const double* __restrict__ part) {
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * nblocks) return;
    const int32_t y = t / nblocks, b = t % nblocks;
    const DevBlock B = blocks[b];
    pos += (idx ? idx[y] : y) * pos_stride;
    phi += (size_t)y * k;
    ns += (size_t)y * 2 * nblocks;
    const double* in = part + (size_t)(y * nblocks + b) * kPhiSplit * 5;
    if (B.kind == TPE_BLOCK_BARYCENTER) {
        double v[5] = {in[0], in[1], in[2], in[3], in[4]};
        for (int sp = 1; sp < kPhiSplit; sp++) {
            for (int q = 0; q < 4; q++) v[q] += in[sp * 5 + q];
            v[4] = js_max(v[4], in[sp * 5 + 4]);
        }
        for (int r = 0; r < 3; r++) phi[B.row0 + r] = v[r];
        ns[2 * b] = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        ns[2 * b + 1] = js_max(1.0, v[3] * js_max(1.0, v[4]));
    } else if (B.kind == TPE_BLOCK_TOTAL_LENGTH || B.kind == TPE_BLOCK_EDGE_LENGTHS) {
        double v[2] = {in[0], in[1]};
        for (int sp = 1; sp < kPhiSplit; sp++) {
            v[0] += in[sp * 5];
            v[1] += in[sp * 5 + 1];
        }
        if (B.kind == TPE_BLOCK_TOTAL_LENGTH) {
            const double p = B.L0 - v[0];
            phi[B.row0] = p;
            ns[2 * b] = p * p;
        } else {
            ns[2 * b] = v[1];
        }
        ns[2 * b + 1] = js_max(1.0, v[0]);
    } else if (B.kind == TPE_BLOCK_POINT) {
        double v = in[0];
        for (int sp = 1; sp < kPhiSplit; sp++) v = js_max(v, in[sp * 5]);
        double s2 = 0.0;
        for (int r = 0; r < 3; r++) {
            const double p = (B.vertex >= 0 && B.vertex < V) ? pos[3 * B.vertex + r] - B.target[r] : NAN;
            phi[B.row0 + r] = p;
            s2 += p * p;
        }
        ns[2 * b] = s2;
        ns[2 * b + 1] = js_max(1.0, v);
    }
}

// Dense C (k x 3V): one thread per vertex, all blocks.
__global__ void jacobian_kernel(const double* __restrict__ pos, const int2* __restrict__ edges,
                                const int32_t* __restrict__ inc_off,
                                const int32_t* __restrict__ inc, int32_t V,
                                const DevBlock* __restrict__ blocks, int32_t nblocks,
                                double* __restrict__ C) {
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const int64_t m = 3 * (int64_t)V;
    for (int32_t b = 0; b < nblocks; b++) {
        const DevBlock B = blocks[b];
        if (B.kind == TPE_BLOCK_BARYCENTER) {
            double acc[3][3] = {};
            for (int32_t p = inc_off[v]; p < inc_off[v + 1]; p++) {
                const int32_t I = inc[p] >> 1;
                const double sg = (inc[p] & 1) ? 1.0 : -1.0;  // -T at i1, +T at i2
                EdgeGeo g;
                edge_geo(pos, edges[I], g, B.target);
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++)
                        acc[r][c] += sg * g.T[c] * g.rvec[r] + 0.5 * g.ell * (r == c ? 1.0 : 0.0);
            }
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) C[(int64_t)(B.row0 + r) * m + (int64_t)c * V + v] = acc[r][c];
        } else if (B.kind == TPE_BLOCK_TOTAL_LENGTH) {
            double acc[3] = {0, 0, 0};
            for (int32_t p = inc_off[v]; p < inc_off[v + 1]; p++) {
                const int32_t I = inc[p] >> 1;
                const double sg = (inc[p] & 1) ? -1.0 : 1.0;  // +T at i1, -T at i2
                EdgeGeo g;
                edge_geo(pos, edges[I], g, nullptr);
                for (int c = 0; c < 3; c++) acc[c] += sg * g.T[c];
            }
            for (int c = 0; c < 3; c++) C[(int64_t)B.row0 * m + (int64_t)c * V + v] = acc[c];
        } else if (B.kind == TPE_BLOCK_EDGE_LENGTHS) {
            for (int32_t p = inc_off[v]; p < inc_off[v + 1]; p++) {
                const int32_t I = inc[p] >> 1;
                const double sg = (inc[p] & 1) ? -1.0 : 1.0;
                EdgeGeo g;
                edge_geo(pos, edges[I], g, nullptr);
                for (int c = 0; c < 3; c++)
                    C[(int64_t)(B.row0 + I) * m + (int64_t)c * V + v] += sg * g.T[c];
            }
        } else if (B.kind == TPE_BLOCK_POINT) {
            if (v == B.vertex)
                for (int r = 0; r < 3; r++) C[(int64_t)(B.row0 + r) * m + (int64_t)r * V + v] = 1.0;
        }
    }
}

// ---- penalties ---------------------------------------------------------------

struct PenW {
    double wl, wd, wf, X[3];
};

__device__ __forceinline__ void pen_edge(const double* __restrict__ pos, int2 e, double& len,
                                         double T[3]) {
    const double ex = pos[3 * e.y] - pos[3 * e.x];
    const double ey = pos[3 * e.y + 1] - pos[3 * e.x + 1];
    const double ez = pos[3 * e.y + 2] - pos[3 * e.x + 2];
    len = sqrt(ex * ex + ey * ey + ez * ez);
    if (len < 1e-14) {
        T[0] = T[1] = T[2] = 0.0;
    } else {
        T[0] = ex / len;
        T[1] = ey / len;
        T[2] = ez / len;
    }
}

__device__ __forceinline__ double edge_len(const double* __restrict__ pos, int2 e) {
    double len, T[3];
    pen_edge(pos, e, len, T);
    return len;
}

// Interior (degree-2) vertex v: its two incident edges in ascending order.
__device__ __forceinline__ bool interior(const int32_t* inc_off, const int32_t* inc, int32_t v,
                                         int32_t& I, int32_t& J) {
    if (inc_off[v + 1] - inc_off[v] != 2) return false;
    I = inc[inc_off[v]] >> 1;
    J = inc[inc_off[v] + 1] >> 1;
    return true;
}

// terms[0..E) edge terms (w_len*l + w_field*l|TxX|^2), terms[E..E+V) vertex terms.
__global__ void pen_energy_terms(const double* __restrict__ pos, const int2* __restrict__ edges,
                                 int32_t E, const int32_t* __restrict__ inc_off,
                                 const int32_t* __restrict__ inc, int32_t V, PenW w,
                                 double* __restrict__ terms) {
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < E) {
        double len, T[3];
        pen_edge(pos, edges[t], len, T);
        double s = 0.0;
        if (w.wl != 0.0) s += w.wl * len;
        if (w.wf != 0.0) {
            const double cx = T[1] * w.X[2] - T[2] * w.X[1];
            const double cy = T[2] * w.X[0] - T[0] * w.X[2];
            const double cz = T[0] * w.X[1] - T[1] * w.X[0];
            s += w.wf * (len * (cx * cx + cy * cy + cz * cz));
        }
        terms[t] = s;
    } else if (t < E + V) {
        const int32_t v = t - E;
        int32_t I, J;
        double s = 0.0;
        if (w.wd != 0.0 && interior(inc_off, inc, v, I, J)) {
            const double d = edge_len(pos, edges[I]) - edge_len(pos, edges[J]);
            s = w.wd * (d * d);
        }
        terms[t] = s;
    }
}

// Per-edge stencil coefficient: g at the edge's second vertex is +coef*T + field, first -.
__global__ void pen_edge_coef(const double* __restrict__ pos, const int2* __restrict__ edges,
                              int32_t E, const int32_t* __restrict__ inc_off,
                              const int32_t* __restrict__ inc, PenW w, double* __restrict__ out) {
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= E) return;
    const int2 e = edges[I];
    double len, T[3];
    pen_edge(pos, e, len, T);
    double coef = 0.0;
    if (w.wl != 0.0) coef += w.wl;
    if (w.wd != 0.0) {
        const int32_t ends[2] = {e.x, e.y};
        for (int k = 0; k < 2; k++) {
            int32_t Iv, Jv;
            if (!interior(inc_off, inc, ends[k], Iv, Jv)) continue;
            const double s = 2.0 * w.wd * (edge_len(pos, edges[Iv]) - edge_len(pos, edges[Jv]));
            if (Iv == I) coef += s;
            if (Jv == I) coef -= s;
        }
    }
    double g[3] = {coef * T[0], coef * T[1], coef * T[2]};
    if (w.wf != 0.0 && !(len < 1e-14)) {
        const double u = T[0] * w.X[0] + T[1] * w.X[1] + T[2] * w.X[2];
        const double c = 1.0 + u * u;
        for (int q = 0; q < 3; q++) g[q] += w.wf * (c * T[q] - 2.0 * u * w.X[q]);
    }
    out[3 * I] = g[0];
    out[3 * I + 1] = g[1];
    out[3 * I + 2] = g[2];
}

__global__ void pen_gather(const double* __restrict__ coef, const int32_t* __restrict__ inc_off,
                           const int32_t* __restrict__ inc, int32_t V, double* __restrict__ grad,
                           int accumulate) {
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    double g[3] = {0, 0, 0};
    for (int32_t p = inc_off[v]; p < inc_off[v + 1]; p++) {
        const int32_t I = inc[p] >> 1;
        const double sg = (inc[p] & 1) ? 1.0 : -1.0;
        for (int q = 0; q < 3; q++) g[q] += sg * coef[3 * I + q];
    }
    for (int q = 0; q < 3; q++) grad[3 * v + q] = accumulate ? grad[3 * v + q] + g[q] : g[q];
}

}  // namespace

int32_t upload_set(tpe_ctx* ctx, const tpe_constraint* set, int32_t nblocks, int32_t* k_out) {
    const int32_t E = ctx->E;
    std::vector<DevBlock> h((size_t)(nblocks > 0 ? nblocks : 1));
    int32_t k = 0, nedge = 0;
    for (int32_t b = 0; b < nblocks; b++) {
        const tpe_constraint& c = set[b];
        int32_t rows;
        switch (c.kind) {
            case TPE_BLOCK_BARYCENTER: rows = 3; break;
            case TPE_BLOCK_TOTAL_LENGTH: rows = 1; break;
            case TPE_BLOCK_EDGE_LENGTHS: rows = E; nedge++; break;
            case TPE_BLOCK_POINT: rows = 3; break;
            default:
                set_error(ctx, TPE_ERR_BAD_ARG, "unknown constraint block kind");
                return TPE_ERR_BAD_ARG;
        }
        h[b] = DevBlock{c.kind, k, c.vertex, rows, {c.target[0], c.target[1], c.target[2]},
                        c.L0, nullptr};
        k += rows;
    }
    TPE_TRY(ensure(ctx, ctx->con_ell0, sizeof(double) * (size_t)E * (nedge > 0 ? nedge : 1)));
    int32_t ei = 0;
    for (int32_t b = 0; b < nblocks; b++) {
        if (set[b].kind != TPE_BLOCK_EDGE_LENGTHS) continue;
        std::vector<double> ell((size_t)E, NAN);
        for (int32_t r = 0; r < E && set[b].ell0 && r < set[b].n_ell0; r++) ell[r] = set[b].ell0[r];
        double* dst = ctx->con_ell0.as<double>() + (size_t)ei * E;
        TPE_CUDA_TRY(cudaMemcpyAsync(dst, ell.data(), sizeof(double) * E, cudaMemcpyHostToDevice,
                                     ctx->stream));
        TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        h[b].ell0 = dst;
        ei++;
    }
    TPE_TRY(ensure(ctx, ctx->con_blocks, sizeof(DevBlock) * h.size()));
    TPE_CUDA_TRY(cudaMemcpyAsync(ctx->con_blocks.ptr, h.data(), sizeof(DevBlock) * h.size(),
                                 cudaMemcpyHostToDevice, ctx->stream));
    TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    *k_out = k;
    return TPE_OK;
}

int32_t eval_constraints_batch(tpe_ctx* ctx, const double* d_pos, int64_t stride,
                               const int32_t* d_idx, int32_t n, int32_t nblocks, int32_t k,
                               double* d_phi, double* d_ns) {
    if (nblocks == 0 || n == 0) return TPE_OK;
    TPE_TRY(ensure(ctx, ctx->con_part, sizeof(double) * (size_t)n * nblocks * kPhiSplit * 5));
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 2);
    phi_part_kernel<<<dim3((unsigned)nblocks, (unsigned)n, kPhiSplit), kBS, 0, ctx->stream>>>(
        d_pos, ctx->d_edges.as<int2>(), ctx->E, ctx->V, ctx->con_blocks.as<DevBlock>(), d_phi,
        stride, d_idx, k, ctx->con_part.as<double>());
    phi_final_kernel<<<(unsigned)((n * nblocks + 127) / 128), 128, 0, ctx->stream>>>(
        d_pos, ctx->V, ctx->con_blocks.as<DevBlock>(), nblocks, d_phi, d_ns, stride, d_idx, k, n,
        ctx->con_part.as<double>());
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t eval_constraints(tpe_ctx* ctx, const double* d_pos, int32_t nblocks, int32_t k,
                         double* d_C, std::vector<double>& phi, std::vector<double>& ns) {
    const int32_t V = ctx->V, E = ctx->E;
    phi.assign((size_t)k, 0.0);
    ns.assign((size_t)2 * nblocks, 0.0);
    if (nblocks == 0) return TPE_OK;
    TPE_TRY(ensure(ctx, ctx->con_phi, sizeof(double) * (size_t)(k + 2 * nblocks + 1)));
    double* dphi = ctx->con_phi.as<double>();
    double* dns = dphi + k;
    TPE_TRY(ensure(ctx, ctx->con_part, sizeof(double) * (size_t)nblocks * kPhiSplit * 5));
    { KernelScope ks(ctx, TPE_KGROUP_OTHER, 2);
    phi_part_kernel<<<dim3((unsigned)nblocks, 1, kPhiSplit), kBS, 0, ctx->stream>>>(
        d_pos, ctx->d_edges.as<int2>(), E, V, ctx->con_blocks.as<DevBlock>(), dphi, 0, nullptr, k,
        ctx->con_part.as<double>());
    phi_final_kernel<<<(unsigned)((nblocks + 127) / 128), 128, 0, ctx->stream>>>(
        d_pos, V, ctx->con_blocks.as<DevBlock>(), nblocks, dphi, dns, 0, nullptr, k, 1,
        ctx->con_part.as<double>()); }
    TPE_CUDA_TRY(cudaGetLastError());
    if (d_C) {
        TPE_CUDA_TRY(cudaMemsetAsync(d_C, 0, sizeof(double) * (size_t)k * 3 * V, ctx->stream));
        KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
        jacobian_kernel<<<(V + 127) / 128, 128, 0, ctx->stream>>>(
            d_pos, ctx->d_edges.as<int2>(), ctx->d_inc_off.as<int32_t>(), ctx->d_inc.as<int32_t>(),
            V, ctx->con_blocks.as<DevBlock>(), nblocks, d_C);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    const HostCopy cp[2] = {{phi.data(), dphi, k > 0 ? sizeof(double) * k : 0},
                            {ns.data(), dns, sizeof(double) * 2 * nblocks}};
    return download_many(ctx, ctx->stream, cp, 2);
}

static PenW resolve(const tpe_penalties* p, bool* active) {
    PenW w{p->total_length, p->length_diff, p->field_weight, {0, 0, 0}};
    if (w.wf != 0.0) {
        const double x = p->field_X[0], y = p->field_X[1], z = p->field_X[2];
        const double n = sqrt(x * x + y * y + z * z);
        if (n < 1e-14) {
            w.wf = 0.0;
        } else {
            w.X[0] = x / n;
            w.X[1] = y / n;
            w.X[2] = z / n;
        }
    }
    *active = (w.wl != 0.0 || w.wd != 0.0 || w.wf != 0.0);
    return w;
}

bool penalties_active(const tpe_penalties* p) {
    bool a = false;
    resolve(p, &a);
    return a;
}

int32_t penalty_energy_dev(tpe_ctx* ctx, const double* d_pos, const tpe_penalties* p,
                           double* out) {
    bool active = false;
    const PenW w = resolve(p, &active);
    if (!active) {
        *out = 0.0;
        return TPE_OK;
    }
    const int32_t E = ctx->E, V = ctx->V;
    TPE_TRY(ensure(ctx, ctx->flat3, sizeof(double) * (size_t)(E + V + 8)));
    double* terms = ctx->flat3.as<double>();
    { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    pen_energy_terms<<<(E + V + 255) / 256, 256, 0, ctx->stream>>>(
        d_pos, ctx->d_edges.as<int2>(), E, ctx->d_inc_off.as<int32_t>(), ctx->d_inc.as<int32_t>(),
        V, w, terms); }
    TPE_CUDA_TRY(cudaGetLastError());
    return dot(ctx, E + V, terms, nullptr, out);
}

int32_t penalty_gradient_dev(tpe_ctx* ctx, const double* d_pos, const tpe_penalties* p,
                             double* d_grad, int accumulate) {
    bool active = false;
    const PenW w = resolve(p, &active);
    const int32_t E = ctx->E, V = ctx->V;
    if (!active) {
        if (!accumulate) TPE_CUDA_TRY(cudaMemsetAsync(d_grad, 0, sizeof(double) * 3 * V, ctx->stream));
        return TPE_OK;
    }
    TPE_TRY(ensure(ctx, ctx->flat3, sizeof(double) * (size_t)(3 * E + 8)));
    double* coef = ctx->flat3.as<double>();
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 2);
    pen_edge_coef<<<(E + 255) / 256, 256, 0, ctx->stream>>>(
        d_pos, ctx->d_edges.as<int2>(), E, ctx->d_inc_off.as<int32_t>(), ctx->d_inc.as<int32_t>(),
        w, coef);
    pen_gather<<<(V + 255) / 256, 256, 0, ctx->stream>>>(coef, ctx->d_inc_off.as<int32_t>(),
                                                          ctx->d_inc.as<int32_t>(), V, d_grad,
                                                          accumulate);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

}  // namespace tpe
