// Saddle solves with a large constraint set (k rows, e.g. one edge-length row
// per edge: k = E + 3 with the barycenter), on the device.
//
// The reference eliminates the constraints inside one dense factorization of
// the (3V + k)^2 saddle matrix (src/core/sobolev/linsolve.ts:431-589, called
// from src/core/optimizer.ts:231-440). The structured solve replaces it with the
// Schur complement S = C A3^{-1} C^T (A3 = A_rho per coordinate block), which the
// small-k path forms from k x 3 solves and factors on the host. For large k that
// is k^3 host work and 3k solves; here instead:
//   Ainv = A_rho^{-1} explicitly (FP64: Cholesky, recursive triangular
//   inverse, X^T X), then Y = A3^{-1} C^T row by row as a gather of at most
//   kNZ rows of Ainv per coordinate block (an edge-length row has two nonzeros
//   per block); rows with more nonzeros (barycenter) go through one multi-RHS
//   product with Ainv;
//   S[r][s] = C_r . Y_s as the same gather (dense rows r: full dot products),
//   symmetrized, factored and inverted on the device (Sinv), so that every
//   multiplier solve is one product with Sinv.
#include <algorithm>

#include "tpe_internal.h"

namespace tpe {
namespace {

constexpr int kNZ = 4;  // nonzeros per (row, coordinate block) kept as a sparse row

// Per row s and coordinate block c: the nonzero entries in index order when
// there are at most kNZ, else dense[s] = 1.
__global__ void __launch_bounds__(256)
sparse_rows_kernel(const double* __restrict__ C, int32_t V, int32_t* __restrict__ nz_idx,
                   double* __restrict__ nz_val, int32_t* __restrict__ nz_cnt,
                   int32_t* __restrict__ dense) {
    const int32_t s = blockIdx.x;
    __shared__ int cnt[3];
    __shared__ int idx[3][kNZ];
    __shared__ double val[3][kNZ];
    if (threadIdx.x < 3) cnt[threadIdx.x] = 0;
    __syncthreads();
    const double* row = C + (int64_t)s * 3 * V;
    for (int64_t t = threadIdx.x; t < 3 * (int64_t)V; t += blockDim.x) {
        const double x = row[t];
        if (x != 0.0) {
            const int c = (int)(t / V);
            const int q = atomicAdd(&cnt[c], 1);
            if (q < kNZ) {
                idx[c][q] = (int)(t - (int64_t)c * V);
                val[c][q] = x;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        bool dn = false;
        for (int c = 0; c < 3; c++) {
            const int n = cnt[c];
            if (n > kNZ) {
                dn = true;
                continue;
            }
            // index order, so the sums below do not depend on the race above
            for (int a = 1; a < n; a++)
                for (int b = a; b > 0 && idx[c][b - 1] > idx[c][b]; b--) {
                    const int ti = idx[c][b];
                    idx[c][b] = idx[c][b - 1];
                    idx[c][b - 1] = ti;
                    const double tv = val[c][b];
                    val[c][b] = val[c][b - 1];
                    val[c][b - 1] = tv;
                }
            for (int q = 0; q < kNZ; q++) {
                nz_idx[((int64_t)s * 3 + c) * kNZ + q] = q < n ? idx[c][q] : 0;
                nz_val[((int64_t)s * 3 + c) * kNZ + q] = q < n ? val[c][q] : 0.0;
            }
            nz_cnt[(int64_t)s * 3 + c] = n;
        }
        dense[s] = dn ? 1 : 0;
    }
}

// Y[s][c][u] = sum_q val[s][c][q] Ainv[idx[s][c][q]][u] for the sparse rows s
// (Ainv symmetric: row idx is column idx). Grid (k, 3, V / 256).
__global__ void __launch_bounds__(256)
y_sparse_kernel(const double* __restrict__ Ainv, int32_t V, const int32_t* __restrict__ nz_idx,
                const double* __restrict__ nz_val, const int32_t* __restrict__ nz_cnt,
                const int32_t* __restrict__ dense, double* __restrict__ Y) {
    const int32_t s = blockIdx.x, c = blockIdx.y;
    if (dense[s]) return;
    const int32_t u = blockIdx.z * blockDim.x + threadIdx.x;
    if (u >= V) return;
    const int64_t rc = (int64_t)s * 3 + c;
    const int n = nz_cnt[rc];
    double acc = 0.0;
    for (int q = 0; q < n; q++)
        acc += nz_val[rc * kNZ + q] * Ainv[(int64_t)nz_idx[rc * kNZ + q] * V + u];
    Y[rc * V + u] = acc;
}

// S[r][s] = sum_c sum_q val[r][c][q] Y[s][c][idx[r][c][q]] for sparse rows r;
// 32 x 32 tiles (r, s), transposed through shared memory so that the gathers
// (consecutive r of one s) and the stores (consecutive s of one r) coalesce.
__global__ void __launch_bounds__(256)
s_sparse_kernel(const double* __restrict__ Y, int32_t V, int32_t k,
                const int32_t* __restrict__ nz_idx, const double* __restrict__ nz_val,
                const int32_t* __restrict__ nz_cnt, const int32_t* __restrict__ dense,
                double* __restrict__ S) {
    __shared__ double t[32][33];
    const int32_t r0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int32_t r = r0 + tx;
    const bool rv = r < k && !dense[r];
    int ix[3][kNZ];
    double vv[3][kNZ];
    int nn[3] = {0, 0, 0};
    if (rv) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const int64_t rc = (int64_t)r * 3 + c;
            nn[c] = nz_cnt[rc];
#pragma unroll
            for (int q = 0; q < kNZ; q++) {
                ix[c][q] = nz_idx[rc * kNZ + q];
                vv[c][q] = nz_val[rc * kNZ + q];
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int sl = ty + 8 * i;
        const int32_t s = s0 + sl;
        double acc = 0.0;
        if (rv && s < k) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const double* ys = Y + ((int64_t)s * 3 + c) * V;
#pragma unroll
                for (int q = 0; q < kNZ; q++)
                    if (q < nn[c]) acc += vv[c][q] * ys[ix[c][q]];
            }
        }
        t[sl][tx] = acc;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int rl = ty + 8 * i;
        const int32_t rr = r0 + rl, s = s0 + tx;
        if (rr < k && s < k && !dense[rr]) S[(int64_t)rr * k + s] = t[tx][rl];
    }
}

// S = (S + S^T) / 2, one pair of 32 x 32 tiles per block (bi >= bj).
__global__ void symmetrize_kernel(double* __restrict__ S, int32_t n) {
    __shared__ double a[32][33], b[32][33];
    const int32_t bi = blockIdx.y, bj = blockIdx.x;
    if (bj > bi) return;
    const int32_t i0 = bi * 32, j0 = bj * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int32_t i = i0 + r, j = j0 + threadIdx.x;
        if (i < n && j < n) a[r][threadIdx.x] = S[(int64_t)i * n + j];
        const int32_t i2 = j0 + r, j2 = i0 + threadIdx.x;
        if (i2 < n && j2 < n) b[r][threadIdx.x] = S[(int64_t)i2 * n + j2];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int32_t i = i0 + r, j = j0 + threadIdx.x;
        // a[r][x] = S[i0 + r][j0 + x], b[x][r] = S[j0 + x][i0 + r]
        if (i < n && j < n) {
            const double m = 0.5 * (a[r][threadIdx.x] + b[threadIdx.x][r]);
            S[(int64_t)i * n + j] = m;
        }
        const int32_t i2 = j0 + r, j2 = i0 + threadIdx.x;
        if (i2 < n && j2 < n && bi != bj) {
            const double m = 0.5 * (b[r][threadIdx.x] + a[threadIdx.x][r]);
            S[(int64_t)i2 * n + j2] = m;
        }
    }
}

}  // namespace

int32_t large_schur_build(tpe_ctx* ctx, SaddleOp& op, const double* b_flat, bool* singular) {
    const int32_t V = op.V, k = op.k;
    const cudaStream_t st = ctx->stream;
    *singular = false;
    const int32_t nmax = std::max(V, k);
    const size_t nn = (size_t)nmax * nmax;
    const size_t half = (size_t)(nmax / 2 + kNB) * (nmax / 2 + kNB);
    TPE_TRY(ensure(ctx, ctx->mat_Ainv, sizeof(double) * (size_t)V * V));
    TPE_TRY(ensure(ctx, ctx->inv_X, sizeof(double) * nn));
    TPE_TRY(ensure(ctx, ctx->inv_W, sizeof(double) * nn));
    TPE_TRY(ensure(ctx, ctx->inv_T, sizeof(double) * half));
    double* Ainv = ctx->mat_Ainv.as<double>();
    if (op.int8) {
        // op.L holds A_rho unfactored; it is overwritten
        bool sing = false;
        TPE_TRY(spd_inverse_int8(ctx, op.L, V, op.chol_tol, ctx->inv_X.as<double>(),
                                 ctx->inv_W.as<double>(), ctx->inv_T.as<double>(), Ainv, &sing));
        if (sing) {
            *singular = true;
            return TPE_OK;
        }
    } else {
        TPE_TRY(spd_inverse_fp64(ctx, op.L, op.Linv, V, ctx->inv_X.as<double>(),
                                 ctx->inv_W.as<double>(), ctx->inv_T.as<double>(), Ainv));
    }
    op.Ainv = Ainv;
    // sparse structure of C
    TPE_TRY(ensure(ctx, ctx->sch_nz, (sizeof(int32_t) + sizeof(double)) * (size_t)k * 3 * kNZ +
                                         sizeof(int32_t) * (size_t)k * 4));
    double* nz_val = ctx->sch_nz.as<double>();
    int32_t* nz_idx = reinterpret_cast<int32_t*>(nz_val + (size_t)k * 3 * kNZ);
    int32_t* nz_cnt = nz_idx + (size_t)k * 3 * kNZ;
    int32_t* dense = nz_cnt + (size_t)k * 3;
    {
        KernelScope ks(ctx, TPE_KGROUP_OTHER, 2);
        sparse_rows_kernel<<<k, 256, 0, st>>>(op.C, V, nz_idx, nz_val, nz_cnt, dense);
        y_sparse_kernel<<<dim3(k, 3, (V + 255) / 256), 256, 0, st>>>(Ainv, V, nz_idx, nz_val, nz_cnt,
                                                                     dense, op.Y);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    std::vector<int32_t> hdense((size_t)k);
    TPE_CUDA_TRY(cudaMemcpyAsync(hdense.data(), dense, sizeof(int32_t) * k, cudaMemcpyDeviceToHost, st));
    TPE_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<int32_t> drows;
    for (int32_t s = 0; s < k; s++)
        if (hdense[s]) drows.push_back(s);
    // dense rows: Y_s = Ainv C_s per coordinate block (3 right-hand sides each)
    for (int32_t s : drows)
        TPE_TRY(mrhs_fp64(ctx, Ainv, V, op.C + (size_t)s * 3 * V, V, 3, op.Y + (size_t)s * 3 * V));
    // the gradient right-hand side: w = A3^{-1} b
    if (b_flat) {
        TPE_TRY(finish_gradient(ctx));
        TPE_TRY(mrhs_fp64(ctx, Ainv, V, b_flat, V, 3, op.W));
    }
    // S = C Y (k x k)
    TPE_TRY(ensure(ctx, ctx->sch_S, sizeof(double) * (size_t)k * k));
    TPE_TRY(ensure(ctx, ctx->sch_L, sizeof(double) * (size_t)k * k));
    TPE_TRY(ensure(ctx, ctx->sch_Linv, sizeof(double) * (size_t)((k + kNB - 1) / kNB) * kNB * kNB));
    TPE_TRY(ensure(ctx, ctx->sch_Sinv, sizeof(double) * (size_t)k * k));
    double* S = ctx->sch_S.as<double>();
    {
        KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
        const unsigned tk = (unsigned)((k + 31) / 32);
        s_sparse_kernel<<<dim3(tk, tk), dim3(32, 8), 0, st>>>(op.Y, V, k, nz_idx, nz_val, nz_cnt,
                                                             dense, S);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    for (int32_t r : drows)
        TPE_TRY(gram_dots(ctx, op.C + (size_t)r * 3 * V, 1, op.Y, k, 3 * (int64_t)V,
                          S + (size_t)r * k));
    {
        KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
        const unsigned tk = (unsigned)((k + 31) / 32);
        symmetrize_kernel<<<dim3(tk, tk), dim3(32, 8), 0, st>>>(S, k);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    double* Ls = ctx->sch_L.as<double>();
    TPE_CUDA_TRY(cudaMemcpyAsync(Ls, S, sizeof(double) * (size_t)k * k, cudaMemcpyDeviceToDevice, st));
    if (op.int8) {
        bool sing = false;
        TPE_TRY(spd_inverse_int8(ctx, Ls, k, 0.0, ctx->inv_X.as<double>(), ctx->inv_W.as<double>(),
                                 ctx->inv_T.as<double>(), ctx->sch_Sinv.as<double>(), &sing));
        if (sing) {
            *singular = true;
            return TPE_OK;
        }
    } else {
        int32_t bad = 0;
        TPE_TRY(cholesky_fp64(ctx, Ls, ctx->sch_Linv.as<double>(), k, 0.0, &bad));
        if (bad) {
            *singular = true;
            return TPE_OK;
        }
        TPE_TRY(spd_inverse_fp64(ctx, Ls, ctx->sch_Linv.as<double>(), k, ctx->inv_X.as<double>(),
                                 ctx->inv_W.as<double>(), ctx->inv_T.as<double>(),
                                 ctx->sch_Sinv.as<double>()));
    }
    op.Sinv = ctx->sch_Sinv.as<double>();
    return TPE_OK;
}

int32_t large_schur_apply(tpe_ctx* ctx, const SaddleOp& op, const double* rc, int32_t nr,
                          double* out) {
    const int32_t k = op.k;
    TPE_TRY(ensure(ctx, ctx->sch_vec, sizeof(double) * 2 * 16 * (size_t)k));
    double* din = ctx->sch_vec.as<double>();
    double* dout = din + (size_t)16 * k;
    for (int32_t c0 = 0; c0 < nr; c0 += 16) {
        const int32_t n = std::min(16, nr - c0);
        TPE_CUDA_TRY(cudaMemcpyAsync(din, rc + (size_t)c0 * k, sizeof(double) * (size_t)n * k,
                                     cudaMemcpyHostToDevice, ctx->stream));
        TPE_TRY(mrhs_fp64(ctx, op.Sinv, k, din, k, n, dout));
        TPE_CUDA_TRY(cudaMemcpyAsync(out + (size_t)c0 * k, dout, sizeof(double) * (size_t)n * k,
                                     cudaMemcpyDeviceToHost, ctx->stream));
        TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    return TPE_OK;
}

}  // namespace tpe
