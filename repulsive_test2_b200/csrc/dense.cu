// Dense FP64 linear algebra for the structured saddle solve.
//
// The reference factors the (3V+k)^2 saddle matrix with Bunch-Kaufman LDL^T
// (src/core/sobolev/linsolve.ts:431-589). Here the only large factorization is
// the SPD V x V matrix A_rho = A + (rho/V) 1 1^T (A is PSD with the constants
// as its kernel), which needs no pivoting: a right-looking blocked Cholesky
// with 64 x 64 blocks. Per block column k: one CTA factors the diagonal block
// and inverts it, one CTA per row block forms the panel as A_ik * inv(L_kk)^T,
// and a tiled kernel applies the symmetric rank-64 update to the trailing
// lower triangle. Triangular solves run block row by block row with the same
// diagonal-block inverses.
#include <math.h>

#include "tpe_internal.h"

namespace tpe {
namespace {

constexpr int NB = kNB;  // 64

// ---- Cholesky --------------------------------------------------------------

// One CTA (256 threads): factor the diagonal block kb (size s <= 64) of the
// lower triangle in place and write its inverse into Linv[kb].
__global__ void __launch_bounds__(256)
potrf_diag_kernel(double* __restrict__ L, double* __restrict__ Linv, int32_t n, int32_t kb,
                  double tol, int32_t* __restrict__ status) {
    extern __shared__ double dsm[];
    double(*a)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm);
    double(*inv)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm + NB * (NB + 1));
    __shared__ int bad;
    const int32_t r0 = kb * NB;
    const int32_t s = min(NB, n - r0);
    const int tid = threadIdx.x;
    if (tid == 0) bad = 0;
    for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
        const int i = idx / NB, j = idx % NB;
        double v;
        if (i < s && j < s)
            v = (j <= i) ? L[(int64_t)(r0 + i) * n + r0 + j] : 0.0;
        else
            v = (i == j) ? 1.0 : 0.0;
        a[i][j] = v;
    }
    __syncthreads();
    for (int j = 0; j < NB; j++) {
        if (tid == 0) {
            const double d = a[j][j];
            if (!(d > tol)) {
                bad = 1;
                a[j][j] = 1.0;
            } else {
                a[j][j] = sqrt(d);
            }
        }
        __syncthreads();
        const double djj = a[j][j];
        for (int i = j + 1 + tid; i < NB; i += blockDim.x) a[i][j] /= djj;
        __syncthreads();
        // trailing update of the lower triangle: a[i][c] -= a[i][j] * a[c][j], j < c <= i
        const int m = NB - j - 1;
        for (int idx = tid; idx < m * m; idx += blockDim.x) {
            const int i = j + 1 + idx / m, c = j + 1 + idx % m;
            if (c <= i) a[i][c] -= a[i][j] * a[c][j];
        }
        __syncthreads();
    }
    // inverse of the lower-triangular factor, one column per thread
    if (tid < NB) {
        const int c = tid;
        for (int i = 0; i < NB; i++) inv[i][c] = 0.0;
        inv[c][c] = 1.0 / a[c][c];
        for (int i = c + 1; i < NB; i++) {
            double acc = 0.0;
            for (int m2 = c; m2 < i; m2++) acc += a[i][m2] * inv[m2][c];
            inv[i][c] = -acc / a[i][i];
        }
    }
    __syncthreads();
    double* Li = Linv + (int64_t)kb * NB * NB;
    for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
        const int i = idx / NB, j = idx % NB;
        Li[idx] = inv[i][j];
        if (i < s && j < s && j <= i) L[(int64_t)(r0 + i) * n + r0 + j] = a[i][j];
    }
    if (tid == 0 && bad) atomicOr(status, 1);
}

// Panel: L_ik = A_ik * inv(L_kk)^T for row blocks i > kb (one CTA each).
__global__ void __launch_bounds__(256)
trsm_panel_kernel(double* __restrict__ L, const double* __restrict__ Linv, int32_t n, int32_t kb) {
    extern __shared__ double dsm[];
    double(*a)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm);
    double(*li)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm + NB * (NB + 1));
    const int32_t ib = kb + 1 + blockIdx.x;
    const int32_t r0 = ib * NB, c0 = kb * NB;
    const int tid = threadIdx.x;
    const double* Lk = Linv + (int64_t)kb * NB * NB;
    for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
        const int i = idx / NB, j = idx % NB;
        a[i][j] = (r0 + i < n) ? L[(int64_t)(r0 + i) * n + c0 + j] : 0.0;
        li[i][j] = Lk[idx];
    }
    __syncthreads();
    // out[i][c] = sum_{m <= c} a[i][m] * li[c][m]
    const int tx = tid % 16, ty = tid / 16;
    double acc[4][4] = {};
    for (int m = 0; m < NB; m++) {
        double av[4], bv[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            av[q] = a[ty * 4 + q][m];
            bv[q] = li[tx * 4 + q][m];
        }
#pragma unroll
        for (int p = 0; p < 4; p++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[p][q] += av[p] * bv[q];
    }
#pragma unroll
    for (int p = 0; p < 4; p++) {
        const int i = ty * 4 + p;
        if (r0 + i >= n) continue;
#pragma unroll
        for (int q = 0; q < 4; q++) L[(int64_t)(r0 + i) * n + c0 + tx * 4 + q] = acc[p][q];
    }
}

// Trailing update A_ij -= L_ik L_jk^T over the lower triangle of the trailing
// matrix, in 128 x 128 tiles (rank-64 update, K = the panel). 256 threads, each
// an 8 x 8 register tile; the two 128 x 64 panels are staged transposed in
// shared memory; a thread owns rows 8ty..8ty+7 and columns 2tx + 32q + {0,1}.
constexpr int ST = 128;
constexpr int SP = ST + 2;
__global__ void __launch_bounds__(256)
syrk_update_kernel(double* __restrict__ L, int32_t n, int32_t kb) {
    extern __shared__ double dsm[];
    double* at = dsm;            // at[m * SP + r] = L[r0 + r][k0 + m]
    double* bt = dsm + NB * SP;  // bt[m * SP + c] = L[c0 + c][k0 + m]
    const int64_t t = blockIdx.x;
    int32_t ti = (int32_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((int64_t)ti * (ti + 1) / 2 > t) ti--;
    while ((int64_t)(ti + 1) * (ti + 2) / 2 <= t) ti++;
    const int32_t tj = (int32_t)(t - (int64_t)ti * (ti + 1) / 2);
    const int32_t rs = (kb + 1) * NB;  // trailing start
    const int32_t r0 = rs + ti * ST, c0 = rs + tj * ST, k0 = kb * NB;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < ST * NB; idx += 256) {
        const int i = idx / NB, m = idx % NB;
        at[m * SP + i] = (r0 + i < n) ? L[(int64_t)(r0 + i) * n + k0 + m] : 0.0;
        bt[m * SP + i] = (c0 + i < n) ? L[(int64_t)(c0 + i) * n + k0 + m] : 0.0;
    }
    __syncthreads();
    const int tx = tid % 16, ty = tid / 16;
    double acc[8][8];
#pragma unroll
    for (int p = 0; p < 8; p++)
#pragma unroll
        for (int q = 0; q < 8; q++) acc[p][q] = 0.0;
#pragma unroll 2
    for (int m = 0; m < NB; m++) {
        double av[8], bv[8];
        const double2* ap = reinterpret_cast<const double2*>(at + m * SP + ty * 8);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            // columns 2*tx + 32*q + {0,1}: a warp's 16 lanes read 256 contiguous bytes
            const double2 a2 = ap[q];
            const double2 b2 = *reinterpret_cast<const double2*>(bt + m * SP + 32 * q + 2 * tx);
            av[2 * q] = a2.x;
            av[2 * q + 1] = a2.y;
            bv[2 * q] = b2.x;
            bv[2 * q + 1] = b2.y;
        }
#pragma unroll
        for (int p = 0; p < 8; p++)
#pragma unroll
            for (int q = 0; q < 8; q++) acc[p][q] = fma(av[p], bv[q], acc[p][q]);
    }
#pragma unroll
    for (int p = 0; p < 8; p++) {
        const int32_t i = r0 + ty * 8 + p;
        if (i >= n) continue;
        double* row = L + (int64_t)i * n;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int32_t c = c0 + 32 * (q >> 1) + 2 * tx + (q & 1);
            if (c < n && c <= i) row[c] -= acc[p][q];
        }
    }
}

// ---- triangular solves: B[nrhs][n] ------------------------------------------

// Triangular-solve block steps. Dynamic shared memory: the 64x64 diagonal
// inverse, one 64x64 tile of L and the block of right-hand sides, all staged
// with coalesced loads.
constexpr int TP = NB + 1;

// Forward step kb: y = inv(L_kk) b_kk (every CTA recomputes it from shared
// memory), CTA 0 stores y into Y; CTA j updates the 64 rows after block kb it
// owns: b_row -= L[row][kb block] y.
__global__ void __launch_bounds__(256)
trsv_fwd_kernel(const double* __restrict__ L, const double* __restrict__ Linv, int32_t n,
                int32_t kb, double* __restrict__ B, double* __restrict__ Y, int32_t nrhs) {
    extern __shared__ double sm[];
    double* li = sm;              // [NB][TP]
    double* lt = li + NB * TP;    // [NB][TP]
    double* bb = lt + NB * TP;    // [nrhs][NB]
    double* y = bb + nrhs * NB;   // [nrhs][NB]
    const int32_t r0 = kb * NB;
    const int32_t s = min(NB, n - r0);
    const int tid = threadIdx.x;
    const double* Li = Linv + (int64_t)kb * NB * NB;
    for (int idx = tid; idx < NB * NB; idx += 256) li[(idx / NB) * TP + idx % NB] = Li[idx];
    for (int idx = tid; idx < nrhs * NB; idx += 256) {
        const int q = idx / NB, m = idx % NB;
        bb[idx] = (m < s) ? B[(int64_t)q * n + r0 + m] : 0.0;
    }
    const int32_t row0 = r0 + NB + blockIdx.x * NB;
    for (int idx = tid; idx < NB * NB; idx += 256) {
        const int rr = idx / NB, m = idx % NB;
        lt[rr * TP + m] = (row0 + rr < n && m < s) ? L[(int64_t)(row0 + rr) * n + r0 + m] : 0.0;
    }
    __syncthreads();
    for (int idx = tid; idx < nrhs * NB; idx += 256) {
        const int q = idx / NB, i = idx % NB;
        double acc = 0.0;
        for (int m = 0; m <= i; m++) acc += li[i * TP + m] * bb[q * NB + m];
        y[idx] = acc;
    }
    __syncthreads();
    if (blockIdx.x == 0)
        for (int idx = tid; idx < nrhs * NB; idx += 256) {
            const int q = idx / NB, i = idx % NB;
            if (i < s) Y[(int64_t)q * n + r0 + i] = y[idx];
        }
    if (row0 >= n) return;
    for (int idx = tid; idx < nrhs * NB; idx += 256) {
        const int q = idx / NB, rr = idx % NB;
        if (row0 + rr >= n) continue;
        double acc = 0.0;
#pragma unroll 8
        for (int m = 0; m < NB; m++) acc += lt[rr * TP + m] * y[q * NB + m];
        B[(int64_t)q * n + row0 + rr] -= acc;
    }
}

// Backward step kb: x = inv(L_kk)^T y_kk, CTA 0 stores x into X; CTA j updates
// the 64 columns it owns before block kb: y_c -= sum_r L[kb*64 + r][c] x_r.
__global__ void __launch_bounds__(256)
trsv_bwd_kernel(const double* __restrict__ L, const double* __restrict__ Linv, int32_t n,
                int32_t kb, double* __restrict__ Yv, double* __restrict__ X, int32_t nrhs) {
    extern __shared__ double sm[];
    double* li = sm;
    double* lt = li + NB * TP;
    double* yb = lt + NB * TP;
    double* x = yb + nrhs * NB;
    const int32_t r0 = kb * NB;
    const int32_t s = min(NB, n - r0);
    const int tid = threadIdx.x;
    const double* Li = Linv + (int64_t)kb * NB * NB;
    for (int idx = tid; idx < NB * NB; idx += 256) li[(idx / NB) * TP + idx % NB] = Li[idx];
    for (int idx = tid; idx < nrhs * NB; idx += 256) {
        const int q = idx / NB, m = idx % NB;
        yb[idx] = (m < s) ? Yv[(int64_t)q * n + r0 + m] : 0.0;
    }
    const int32_t col0 = blockIdx.x * NB;
    const bool upd = col0 < r0;
    if (upd)
        for (int idx = tid; idx < NB * NB; idx += 256) {
            const int r = idx / NB, cc = idx % NB;
            lt[r * TP + cc] = (r < s) ? L[(int64_t)(r0 + r) * n + col0 + cc] : 0.0;
        }
    __syncthreads();
    for (int idx = tid; idx < nrhs * NB; idx += 256) {
        const int q = idx / NB, i = idx % NB;
        double acc = 0.0;
        for (int m = i; m < NB; m++) acc += li[m * TP + i] * yb[q * NB + m];
        x[idx] = acc;
    }
    __syncthreads();
    if (blockIdx.x == 0)
        for (int idx = tid; idx < nrhs * NB; idx += 256) {
            const int q = idx / NB, i = idx % NB;
            if (i < s) X[(int64_t)q * n + r0 + i] = x[idx];
        }
    if (!upd) return;
    for (int idx = tid; idx < nrhs * NB; idx += 256) {
        const int q = idx / NB, cc = idx % NB;
        double acc = 0.0;
#pragma unroll 8
        for (int r = 0; r < NB; r++) acc += lt[r * TP + cc] * x[q * NB + r];
        Yv[(int64_t)q * n + col0 + cc] -= acc;
    }
}

// ---- reductions and vector helpers -----------------------------------------

template <int BS>
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double red[BS / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < BS / 32; w++) t += red[w];
    __syncthreads();
    return t;  // valid on thread 0
}

// out[i*ny + j] = sum_t X[i][t] * Y[j][t]; one CTA per (i, j).
__global__ void __launch_bounds__(256)
gram_dots_kernel(const double* __restrict__ X, const double* __restrict__ Y, int32_t ny,
                 int64_t len, double* __restrict__ out) {
    const int32_t i = blockIdx.x / ny, j = blockIdx.x % ny;
    const double* x = X + (int64_t)i * len;
    const double* y = Y + (int64_t)j * len;
    double s = 0.0;
    for (int64_t t = threadIdx.x; t < len; t += blockDim.x) s += x[t] * y[t];
    s = block_sum<256>(s);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

__global__ void shift_copy_kernel(const double* __restrict__ A, double* __restrict__ L, int32_t n,
                                  double shift) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * n) return;
    const int32_t i = (int32_t)(t / n), j = (int32_t)(t % n);
    L[t] = (j <= i) ? A[t] + shift : 0.0;
}

__global__ void trace_kernel(const double* __restrict__ A, int32_t n, double* __restrict__ out) {
    double s = 0.0;
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) s += A[(int64_t)i * n + i];
    s = block_sum<256>(s);
    if (threadIdx.x == 0) *out = s;
}

__global__ void to_block_kernel(const double* __restrict__ v3, double* __restrict__ f, int32_t V) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    f[i] = v3[3 * i];
    f[V + i] = v3[3 * i + 1];
    f[2 * V + i] = v3[3 * i + 2];
}

__global__ void to_interleaved_kernel(const double* __restrict__ f, double* __restrict__ v3,
                                      int32_t V) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    v3[3 * i] = f[i];
    v3[3 * i + 1] = f[V + i];
    v3[3 * i + 2] = f[2 * V + i];
}

__global__ void axpby_kernel(int64_t n, double a, const double* __restrict__ x, double b,
                             double* __restrict__ y) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) y[t] = a * x[t] + b * y[t];
}

// Two-stage deterministic dot / non-finite count (partials then one CTA).
__global__ void __launch_bounds__(256)
dot_partial_kernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                   double* __restrict__ part) {
    double s = 0.0;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        s += x[t] * (y ? y[t] : 1.0);
    s = block_sum<256>(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256)
nonfinite_partial_kernel(int64_t n, const double* __restrict__ x, double* __restrict__ part) {
    double s = 0.0;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        s += isfinite(x[t]) ? 0.0 : 1.0;
    s = block_sum<256>(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256)
sum_kernel(const double* __restrict__ part, int32_t n, double* __restrict__ out) {
    double s = 0.0;
    for (int32_t t = threadIdx.x; t < n; t += blockDim.x) s += part[t];
    s = block_sum<256>(s);
    if (threadIdx.x == 0) *out = s;
}

// Per-edge l2CurveNorm terms (lineSearch.ts:53-75).
__global__ void l2_terms_kernel(const double* __restrict__ vals, const double* __restrict__ pos,
                                const int2* __restrict__ edges, int32_t E,
                                double* __restrict__ terms) {
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= E) return;
    const int2 e = edges[I];
    const double ex = pos[3 * e.y] - pos[3 * e.x];
    const double ey = pos[3 * e.y + 1] - pos[3 * e.x + 1];
    const double ez = pos[3 * e.y + 2] - pos[3 * e.x + 2];
    const double ell = sqrt(ex * ex + ey * ey + ez * ez);
    const double* v1 = vals + 3 * e.x;
    const double* v2 = vals + 3 * e.y;
    terms[I] = 0.5 * ell *
               (v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2] +
                (v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2]));
}

// x = w - sum_s Y[s] lam[s] - (mu_c / (rho sqrt(V))) in block c.
__global__ void combine_kernel(const double* __restrict__ w, const double* __restrict__ Y,
                               int32_t k, const double* __restrict__ coef, int32_t V,
                               double* __restrict__ x) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t m = 3 * (int64_t)V;
    if (t >= m) return;
    double v = w ? w[t] : 0.0;
    for (int32_t s = 0; s < k; s++) v -= Y[(int64_t)s * m + t] * coef[s];
    v -= coef[k + (int32_t)(t / V)];
    x[t] = v;
}

// Residual rows: top (3V): A x_c + (C^T lam)_c - rhs ; one thread per (c, i),
// grouped so each A row is read once for the three blocks.
__global__ void __launch_bounds__(256)
residual_top_kernel(const double* __restrict__ A, int32_t V, const double* __restrict__ C,
                    int32_t k, const double* __restrict__ x, const double* __restrict__ lam,
                    const double* __restrict__ rhs, double* __restrict__ out_res,
                    double* __restrict__ out_rhs) {
    // one CTA per row i: 256 threads stride the row
    const int32_t i = blockIdx.x;
    const double* Ai = A + (int64_t)i * V;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int32_t j = threadIdx.x; j < V; j += blockDim.x) {
        const double a = Ai[j];
        s0 += a * x[j];
        s1 += a * x[V + j];
        s2 += a * x[2 * V + j];
    }
    s0 = block_sum<256>(s0);
    s1 = block_sum<256>(s1);
    s2 = block_sum<256>(s2);
    if (threadIdx.x == 0) {
        const int64_t m = 3 * (int64_t)V;
        double r2 = 0.0, b2 = 0.0;
        double s[3] = {s0, s1, s2};
        for (int c = 0; c < 3; c++) {
            const int64_t row = (int64_t)c * V + i;
            double v = s[c];
            for (int32_t r = 0; r < k; r++) v += C[(int64_t)r * m + row] * lam[r];
            const double d = v - rhs[row];
            r2 += d * d;
            b2 += rhs[row] * rhs[row];
        }
        out_res[i] = r2;
        out_rhs[i] = b2;
    }
}

inline int32_t grid_for(int64_t n, int bs) { return (int32_t)((n + bs - 1) / bs); }

}  // namespace

int32_t cholesky_fp64(tpe_ctx* ctx, double* d_L, double* d_Linv, int32_t n, double piv_tol,
                      int32_t* singular) {
    const int32_t nb = (n + NB - 1) / NB;
    TPE_TRY(ensure(ctx, ctx->status, sizeof(int32_t) * 4));
    int32_t* st = ctx->status.as<int32_t>();
    TPE_CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(int32_t), ctx->stream));
    const size_t sm1 = sizeof(double) * 2 * NB * (NB + 1);
    const size_t sm2 = sizeof(double) * 2 * NB * SP;
    TPE_CUDA_TRY(cudaFuncSetAttribute(potrf_diag_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
    TPE_CUDA_TRY(cudaFuncSetAttribute(trsm_panel_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
    TPE_CUDA_TRY(cudaFuncSetAttribute(syrk_update_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
    KernelScope ks(ctx, TPE_KGROUP_CHOLESKY, 3 * (int64_t)nb - 2);
    for (int32_t kb = 0; kb < nb; kb++) {
        potrf_diag_kernel<<<1, 256, sm1, ctx->stream>>>(d_L, d_Linv, n, kb, piv_tol, st);
        const int32_t rest = nb - kb - 1;
        if (rest > 0) {
            trsm_panel_kernel<<<rest, 256, sm1, ctx->stream>>>(d_L, d_Linv, n, kb);
            const int64_t nt2 = ((int64_t)rest * NB + ST - 1) / ST;
            const int64_t tiles = nt2 * (nt2 + 1) / 2;
            syrk_update_kernel<<<(unsigned)tiles, 256, sm2, ctx->stream>>>(d_L, n, kb);
        }
    }
    TPE_CUDA_TRY(cudaGetLastError());
    int32_t h = 0;
    TPE_CUDA_TRY(cudaMemcpyAsync(&h, st, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    *singular = h;
    return TPE_OK;
}

int32_t chol_solve_fp64(tpe_ctx* ctx, const double* d_L, const double* d_Linv, int32_t n,
                        double* d_B, int32_t nrhs) {
    if (nrhs <= 0) return TPE_OK;
    const int32_t nb = (n + NB - 1) / NB;
    TPE_TRY(ensure(ctx, ctx->solve_scratch, sizeof(double) * (size_t)n * nrhs));
    double* Y = ctx->solve_scratch.as<double>();
    const size_t smem = sizeof(double) * (2 * (size_t)NB * TP + 2 * (size_t)nrhs * NB);
    if (nrhs > 64) {
        set_error(ctx, TPE_ERR_TOO_LARGE, "chol_solve: at most 64 right-hand sides per call");
        return TPE_ERR_TOO_LARGE;
    }
    TPE_CUDA_TRY(cudaFuncSetAttribute(trsv_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(double) * (2 * NB * TP + 2 * 64 * NB))));
    TPE_CUDA_TRY(cudaFuncSetAttribute(trsv_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(double) * (2 * NB * TP + 2 * 64 * NB))));
    KernelScope ks(ctx, TPE_KGROUP_TRSV, 2 * (int64_t)nb);
    for (int32_t kb = 0; kb < nb; kb++) {
        const int32_t rows_after = n - (kb + 1) * NB;
        const int32_t g = rows_after > 0 ? (rows_after + NB - 1) / NB : 1;
        trsv_fwd_kernel<<<g, 256, smem, ctx->stream>>>(d_L, d_Linv, n, kb, d_B, Y, nrhs);
    }
    for (int32_t kb = nb - 1; kb >= 0; kb--) {
        const int32_t g = kb > 0 ? kb : 1;
        trsv_bwd_kernel<<<g, 256, smem, ctx->stream>>>(d_L, d_Linv, n, kb, Y, d_B, nrhs);
    }
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t gram_dots(tpe_ctx* ctx, const double* X, int32_t nx, const double* Y, int32_t ny,
                  int64_t len, double* d_out) {
    if (nx <= 0 || ny <= 0) return TPE_OK;
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    gram_dots_kernel<<<nx * ny, 256, 0, ctx->stream>>>(X, Y, ny, len, d_out);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t shift_copy(tpe_ctx* ctx, const double* d_A, double* d_L, int32_t n, double shift) {
    const int64_t nn = (int64_t)n * n;
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    shift_copy_kernel<<<grid_for(nn, 256), 256, 0, ctx->stream>>>(d_A, d_L, n, shift);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t trace(tpe_ctx* ctx, const double* d_A, int32_t n, double* d_out) {
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    trace_kernel<<<1, 256, 0, ctx->stream>>>(d_A, n, d_out);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t interleaved_to_block(tpe_ctx* ctx, const double* d_v3, double* d_flat, int32_t V) {
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    to_block_kernel<<<grid_for(V, 256), 256, 0, ctx->stream>>>(d_v3, d_flat, V);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t block_to_interleaved(tpe_ctx* ctx, const double* d_flat, double* d_v3, int32_t V) {
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    to_interleaved_kernel<<<grid_for(V, 256), 256, 0, ctx->stream>>>(d_flat, d_v3, V);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t axpby(tpe_ctx* ctx, int64_t n, double a, const double* x, double b, double* y) {
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    axpby_kernel<<<grid_for(n, 256), 256, 0, ctx->stream>>>(n, a, x, b, y);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

static int32_t reduce_to_host(tpe_ctx* ctx, double* part, int32_t nparts, double* out) {
    double* dst = part + nparts;
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    sum_kernel<<<1, 256, 0, ctx->stream>>>(part, nparts, dst);
    TPE_CUDA_TRY(cudaGetLastError());
    TPE_CUDA_TRY(cudaMemcpyAsync(out, dst, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return TPE_OK;
}

int32_t dot(tpe_ctx* ctx, int64_t n, const double* x, const double* y, double* out) {
    const int32_t g = 256;
    TPE_TRY(ensure(ctx, ctx->scalars, sizeof(double) * (g + 8)));
    { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    dot_partial_kernel<<<g, 256, 0, ctx->stream>>>(n, x, y, ctx->scalars.as<double>()); }
    TPE_CUDA_TRY(cudaGetLastError());
    return reduce_to_host(ctx, ctx->scalars.as<double>(), g, out);
}

int32_t count_nonfinite(tpe_ctx* ctx, int64_t n, const double* x, int64_t* out) {
    const int32_t g = 256;
    TPE_TRY(ensure(ctx, ctx->scalars, sizeof(double) * (g + 8)));
    { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    nonfinite_partial_kernel<<<g, 256, 0, ctx->stream>>>(n, x, ctx->scalars.as<double>()); }
    TPE_CUDA_TRY(cudaGetLastError());
    double d = 0.0;
    TPE_TRY(reduce_to_host(ctx, ctx->scalars.as<double>(), g, &d));
    *out = (int64_t)d;
    return TPE_OK;
}

int32_t l2_curve_norm(tpe_ctx* ctx, const double* d_vals, const double* d_pos, double* out) {
    const int32_t E = ctx->E;
    TPE_TRY(ensure(ctx, ctx->tmp, sizeof(double) * (size_t)(E + 8)));
    { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    l2_terms_kernel<<<grid_for(E, 256), 256, 0, ctx->stream>>>(d_vals, d_pos,
                                                               ctx->d_edges.as<int2>(), E,
                                                               ctx->tmp.as<double>()); }
    TPE_CUDA_TRY(cudaGetLastError());
    double total = 0.0;
    TPE_TRY(dot(ctx, E, ctx->tmp.as<double>(), nullptr, &total));
    *out = sqrt(total > 0.0 ? total : 0.0);
    if (total != total) *out = NAN;
    return TPE_OK;
}

int32_t combine_solution(tpe_ctx* ctx, const double* d_w, const double* d_Y, int32_t k,
                         const double* lam, const double* mu, double rho, int32_t V, double* d_x) {
    std::vector<double> coef((size_t)k + 3, 0.0);
    for (int32_t s = 0; s < k; s++) coef[s] = lam[s];
    const double su = 1.0 / (rho * sqrt((double)V));
    for (int c = 0; c < 3; c++) coef[(size_t)k + c] = mu ? mu[c] * su : 0.0;
    TPE_TRY(ensure(ctx, ctx->scalars, sizeof(double) * (size_t)(k + 3 + 512)));
    double* dc = ctx->scalars.as<double>() + 264;
    TPE_CUDA_TRY(cudaMemcpyAsync(dc, coef.data(), sizeof(double) * coef.size(),
                                 cudaMemcpyHostToDevice, ctx->stream));
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    combine_kernel<<<grid_for(3 * (int64_t)V, 256), 256, 0, ctx->stream>>>(d_w, d_Y, k, dc, V,
                                                                          d_x);
    TPE_CUDA_TRY(cudaGetLastError());
    TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return TPE_OK;
}

int32_t saddle_residual(tpe_ctx* ctx, const double* d_A, int32_t V, const double* d_C, int32_t k,
                        const double* d_x, const double* lam, const double* d_rhs_top,
                        const double* rhs_bottom, double* out) {
    TPE_TRY(ensure(ctx, ctx->tmp, sizeof(double) * (size_t)(2 * V + 16 + k)));
    TPE_TRY(ensure(ctx, ctx->scalars, sizeof(double) * (size_t)(k + 3 + 512)));
    double* dl = ctx->scalars.as<double>() + 264;
    if (k > 0)
        TPE_CUDA_TRY(cudaMemcpyAsync(dl, lam, sizeof(double) * k, cudaMemcpyHostToDevice,
                                     ctx->stream));
    double* rr = ctx->tmp.as<double>();
    double* rb = rr + V;
    { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    residual_top_kernel<<<V, 256, 0, ctx->stream>>>(d_A, V, d_C, k, d_x, dl, d_rhs_top, rr, rb); }
    TPE_CUDA_TRY(cudaGetLastError());
    double top_r = 0.0, top_b = 0.0;
    TPE_TRY(dot(ctx, V, rr, nullptr, &top_r));
    TPE_TRY(dot(ctx, V, rb, nullptr, &top_b));
    // bottom rows C x - rhs_bottom
    double bot_r = 0.0, bot_b = 0.0;
    if (k > 0) {
        TPE_TRY(ensure(ctx, ctx->tmp, sizeof(double) * (size_t)(2 * V + 16 + k)));
        double* cx = ctx->tmp.as<double>() + 2 * V;
        TPE_TRY(gram_dots(ctx, d_C, k, d_x, 1, 3 * (int64_t)V, cx));
        std::vector<double> h((size_t)k);
        TPE_CUDA_TRY(cudaMemcpyAsync(h.data(), cx, sizeof(double) * k, cudaMemcpyDeviceToHost,
                                     ctx->stream));
        TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        for (int32_t r = 0; r < k; r++) {
            const double b = rhs_bottom ? rhs_bottom[r] : 0.0;
            const double d = h[r] - b;
            bot_r += d * d;
            bot_b += b * b;
        }
    }
    const double rn = sqrt(top_r + bot_r), bn = sqrt(top_b + bot_b);
    *out = rn / (bn > 1.0 ? bn : 1.0);
    return TPE_OK;
}

}  // namespace tpe
