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
#include <cooperative_groups.h>
#include <math.h>

#include "tpe_internal.h"

namespace cg = cooperative_groups;

namespace tpe {
namespace {

constexpr int NB = kNB;  // 64

// ---- Cholesky --------------------------------------------------------------

// One CTA (256 threads): factor the 64x64 diagonal block kb (size s <= 64,
// padded with the identity) in FP64 and write L_kk and inv(L_kk). The block is
// processed in four 16-column panels: warp 0 factors a panel in registers
// (lane l owns panel rows c0+l and c0+l+32, column entries broadcast with
// shuffles), then all warps apply the rank-16 update to the rest of the block.
// The inverse is built from 16x16 diagonal inverses and three block-diagonal
// stages X_ij = -inv(L_ii) sum_{m=j}^{i-1} L_im X_mj. About 15 barriers in all.
template <typename T>
__global__ void __launch_bounds__(256)
potrf_diag_kernel(T* __restrict__ L, T* __restrict__ Linv, int32_t n, int32_t kb, double tol,
                  int32_t* __restrict__ status) {
    extern __shared__ double dsm[];
    double(*a)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm);
    double(*inv)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm + NB * (NB + 1));
    double(*tmp)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm + 2 * NB * (NB + 1));
    __shared__ int bad;
    const int32_t r0 = kb * NB;
    const int32_t s = min(NB, n - r0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) bad = 0;
    for (int idx = tid; idx < NB * NB; idx += 256) {
        const int i = idx / NB, j = idx % NB;
        double v;
        if (i < s && j < s)
            v = (j <= i) ? (double)L[(int64_t)(r0 + i) * n + r0 + j] : 0.0;
        else
            v = (i == j) ? 1.0 : 0.0;
        a[i][j] = v;
        inv[i][j] = 0.0;
    }
    __syncthreads();
    for (int p = 0; p < 4; p++) {
        const int c0 = 16 * p;
        if (warp == 0) {
            const int ra = c0 + lane, rb = c0 + lane + 32;
            const bool va = ra < NB, vb = rb < NB;
            double x[16], y[16];
#pragma unroll
            for (int c = 0; c < 16; c++) {
                x[c] = va ? a[ra][c0 + c] : 0.0;
                y[c] = vb ? a[rb][c0 + c] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < 16; j++) {
                double d = __shfl_sync(0xffffffffu, x[j], j);
                if (!(d > tol)) {
                    if (lane == 0) bad = 1;
                    d = 1.0;
                }
                const double sq = sqrt(d);
                const double iv = 1.0 / sq;
                if (lane > j) x[j] *= iv;
                if (lane == j) x[j] = sq;
                y[j] *= iv;
#pragma unroll
                for (int c = j + 1; c < 16; c++) {
                    const double lcj = __shfl_sync(0xffffffffu, x[j], c);
                    if (lane >= c) x[c] -= x[j] * lcj;
                    y[c] -= y[j] * lcj;
                }
            }
#pragma unroll
            for (int c = 0; c < 16; c++) {
                if (va && ra >= c0 + c) a[ra][c0 + c] = x[c];
                if (vb) a[rb][c0 + c] = y[c];
            }
        }
        __syncthreads();
        const int c1 = c0 + 16, m = NB - c1;
        if (m > 0) {
            for (int idx = tid; idx < m * m; idx += 256) {
                const int i = c1 + idx / m, c = c1 + idx % m;
                if (c > i) continue;
                double acc = a[i][c];
#pragma unroll
                for (int q = 0; q < 16; q++) acc -= a[i][c0 + q] * a[c][c0 + q];
                a[i][c] = acc;
            }
        }
        __syncthreads();
    }
    // 16x16 diagonal inverses: warp w < 4 inverts block w, lane c < 16 owns column c
    if (warp < 4 && lane < 16) {
        const int o = 16 * warp, c = lane;
        for (int i = 0; i < 16; i++) {
            double acc = (i == c) ? 1.0 : 0.0;
            for (int mm = c; mm < i; mm++) acc -= a[o + i][o + mm] * inv[o + mm][o + c];
            inv[o + i][o + c] = (i >= c) ? acc / a[o + i][o + i] : 0.0;
        }
    }
    __syncthreads();
    for (int dgl = 1; dgl < 4; dgl++) {
        // tmp_ij = sum_{m=j}^{i-1} L_im X_mj for the blocks (i, j = i - dgl)
        const int nblk = 4 - dgl;
        for (int idx = tid; idx < nblk * 256; idx += 256) {
            const int bi = idx / 256, e = idx % 256, r = e / 16, c = e % 16;
            const int i = bi + dgl, j = bi;
            double acc = 0.0;
            for (int mb = j; mb < i; mb++)
                for (int q = 0; q < 16; q++) acc += a[16 * i + r][16 * mb + q] * inv[16 * mb + q][16 * j + c];
            tmp[16 * i + r][16 * j + c] = acc;
        }
        __syncthreads();
        for (int idx = tid; idx < nblk * 256; idx += 256) {
            const int bi = idx / 256, e = idx % 256, r = e / 16, c = e % 16;
            const int i = bi + dgl, j = bi;
            double acc = 0.0;
            for (int q = 0; q < 16; q++) acc += inv[16 * i + r][16 * i + q] * tmp[16 * i + q][16 * j + c];
            inv[16 * i + r][16 * j + c] = -acc;
        }
        __syncthreads();
    }
    T* Li = Linv + (int64_t)kb * NB * NB;
    for (int idx = tid; idx < NB * NB; idx += 256) {
        const int i = idx / NB, j = idx % NB;
        Li[idx] = (T)inv[i][j];
        if (i < s && j < s && j <= i) L[(int64_t)(r0 + i) * n + r0 + j] = (T)a[i][j];
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

// Lower-triangle update L[r][c] -= sum_{m<kl} L[r][k0+m] L[c][k0+m] for
// r in [r_s, n), c in [c_s, c_e), c <= r, on the FP64 tensor cores
// (mma.sync m8n8k4 f64). 128x128 output tiles (tiles entirely above the
// diagonal exit at once), 8 warps as 2 (rows) x 4 (cols), each warp 64x32 =
// 8x4 MMA tiles. K runs in chunks of 32 staged by 16-byte cp.async into two
// shared-memory buffers; rows are padded to 36 doubles (72 words = 8 banks
// mod 32) so a fragment load (8 rows x 4 k) takes the minimum two wavefronts.
constexpr int GT = 128;
constexpr int GK = 32;
constexpr int GP = GK + 4;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
// Two doubles into 16-byte aligned shared memory from a source that may be
// only 8-byte aligned (an odd row length).
template <bool kAligned16>
__device__ __forceinline__ void cp_async_pair(void* smem, const double* gmem) {
    if (kAligned16) {
        cp_async16(smem, gmem);
    } else {
        const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s + 8), "l"(gmem + 1));
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <bool kAligned16>  // rows start on 16-byte boundaries (n even)
__global__ void __launch_bounds__(256)
gemm_lower_update_kernel(double* __restrict__ L, int32_t n, int32_t r_s, int32_t c_s, int32_t c_e,
                         int32_t k0, int32_t kl) {
    extern __shared__ double dsm[];
    const int32_t r0 = r_s + blockIdx.y * GT, c0 = c_s + blockIdx.x * GT;
    if (c0 > r0 + GT - 1) return;
    double* As = dsm;                  // [2][GT][GP]
    double* Bs = dsm + 2 * GT * GP;    // [2][GT][GP]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = (warp >> 2) * 64, wc = (warp & 3) * 32;  // warp tile origin in the CTA tile
    const int fr = lane >> 2, fk = lane & 3;                // fragment row / k of this lane
    auto load = [&](int buf, int kc) {
        // 128 rows x 32 doubles = 2048 16-byte pieces per operand, 8 per thread
        for (int idx = tid; idx < GT * (GK / 2); idx += 256) {
            const int rr = idx / (GK / 2), pc = (idx % (GK / 2)) * 2;
            const int32_t ra = min(r0 + rr, n - 1), rb = min(c0 + rr, n - 1);
            cp_async_pair<kAligned16>(As + (size_t)buf * GT * GP + rr * GP + pc,
                                      L + (int64_t)ra * n + k0 + kc + pc);
            cp_async_pair<kAligned16>(Bs + (size_t)buf * GT * GP + rr * GP + pc,
                                      L + (int64_t)rb * n + k0 + kc + pc);
        }
        cp_async_commit();
    };
    double acc[8][4][2];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int nch = kl / GK;
    load(0, 0);
    for (int ch = 0; ch < nch; ch++) {
        if (ch + 1 < nch) {
            load((ch + 1) & 1, (ch + 1) * GK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double* Ab = As + (size_t)(ch & 1) * GT * GP + (wr + fr) * GP + fk;
        const double* Bb = Bs + (size_t)(ch & 1) * GT * GP + (wc + fr) * GP + fk;
#pragma unroll
        for (int kk = 0; kk < GK; kk += 4) {
            double af[8], bf[4];
#pragma unroll
            for (int i = 0; i < 8; i++) af[i] = Ab[i * 8 * GP + kk];
#pragma unroll
            for (int j = 0; j < 4; j++) bf[j] = Bb[j * 8 * GP + kk];
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
        __syncthreads();
    }
    // accumulator (i, j): rows wr + 8i + lane/4, cols wc + 8j + 2(lane%4) + {0,1}
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int32_t row = r0 + wr + 8 * i + fr;
        if (row >= n) continue;
        double* rp = L + (int64_t)row * n;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int32_t col = c0 + wc + 8 * j + 2 * fk;
            if (col < c_e && col <= row) rp[col] -= acc[i][j][0];
            if (col + 1 < c_e && col + 1 <= row) rp[col + 1] -= acc[i][j][1];
        }
    }
}

// C = alpha A B^T + beta C (row-major FP64) with the tile, fragment and staging
// scheme of gemm_lower_update_kernel, separate operands, rows past M / N
// clamped (never stored), a zero-filled K tail and optional structure:
// kDLowerTiles computes only tiles with tile column <= tile row; kDAUpper
// (A[i][k] = 0 for k < i) starts the K loop of tile row t at 128 t, kDALower
// (A[i][k] = 0 for k > i) ends it at 128 (t + 1).
template <bool kAligned16>
__global__ void __launch_bounds__(256) dgemm_nt_kernel(const DGemmArgs g) {
    extern __shared__ double dsm[];
    const int32_t ti = blockIdx.y, tj = blockIdx.x;
    if ((g.mode & kDLowerTiles) && tj > ti) return;
    const int32_t r0 = ti * GT, c0 = tj * GT;
    int32_t kb = 0, ke = g.K;
    if (g.mode & kDAUpper) kb = min(g.K, r0);
    if (g.mode & kDALower) ke = min(g.K, r0 + GT);
    double* As = dsm;                // [2][GT][GP]
    double* Bs = dsm + 2 * GT * GP;  // [2][GT][GP]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = (warp >> 2) * 64, wc = (warp & 3) * 32;
    const int fr = lane >> 2, fk = lane & 3;
    auto load = [&](int buf, int kc) {
        for (int idx = tid; idx < GT * (GK / 2); idx += 256) {
            const int rr = idx / (GK / 2), pc = (idx % (GK / 2)) * 2;
            const int32_t k = kb + kc + pc;
            const int64_t ra = min(r0 + rr, g.M - 1), rb = min(c0 + rr, g.N - 1);
            double* da = As + (size_t)buf * GT * GP + rr * GP + pc;
            double* db = Bs + (size_t)buf * GT * GP + rr * GP + pc;
            if (k + 1 < ke) {
                cp_async_pair<kAligned16>(da, g.A + ra * g.lda + k);
                cp_async_pair<kAligned16>(db, g.B + rb * g.ldb + k);
            } else {
                da[0] = k < ke ? g.A[ra * g.lda + k] : 0.0;
                db[0] = k < ke ? g.B[rb * g.ldb + k] : 0.0;
                da[1] = 0.0;
                db[1] = 0.0;
            }
        }
        cp_async_commit();
    };
    double acc[8][4][2];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int nch = ke > kb ? (ke - kb + GK - 1) / GK : 0;
    if (nch > 0) load(0, 0);
    for (int ch = 0; ch < nch; ch++) {
        if (ch + 1 < nch) {
            load((ch + 1) & 1, (ch + 1) * GK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double* Ab = As + (size_t)(ch & 1) * GT * GP + (wr + fr) * GP + fk;
        const double* Bb = Bs + (size_t)(ch & 1) * GT * GP + (wc + fr) * GP + fk;
#pragma unroll
        for (int kk = 0; kk < GK; kk += 4) {
            double af[8], bf[4];
#pragma unroll
            for (int i = 0; i < 8; i++) af[i] = Ab[i * 8 * GP + kk];
#pragma unroll
            for (int j = 0; j < 4; j++) bf[j] = Bb[j * 8 * GP + kk];
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int32_t row = r0 + wr + 8 * i + fr;
        if (row >= g.M) continue;
        double* cp = g.C + (int64_t)row * g.ldc;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int32_t col = c0 + wc + 8 * j + 2 * fk;
#pragma unroll
            for (int e = 0; e < 2; e++) {
                if (col + e >= g.N) continue;
                double y = g.alpha * acc[i][j][e];
                if (g.beta != 0.0) y += g.beta * cp[col + e];
                cp[col + e] = y;
            }
        }
    }
}

// The 64 x 64 diagonal-block inverses (nb x 64 x 64, lower) onto the diagonals
// of X (lower) and W = X^T (upper), n x n; block b covers min(64, n - 64 b) rows.
__global__ void diag_inverse_kernel(const double* __restrict__ Linv, int32_t n,
                                    double* __restrict__ X, double* __restrict__ W) {
    const int32_t b = blockIdx.x, r0 = b * NB, s = min(NB, n - r0);
    const double* Li = Linv + (int64_t)b * NB * NB;
    for (int idx = threadIdx.x; idx < NB * NB; idx += blockDim.x) {
        const int i = idx / NB, j = idx % NB;
        if (i >= s || j >= s) continue;
        X[(int64_t)(r0 + i) * n + r0 + j] = Li[idx];
        W[(int64_t)(r0 + j) * n + r0 + i] = Li[idx];
    }
}

// dst[j][i] = src[i][j] for an m x c block (row strides lds, ldd), 32 x 32 tiles.
__global__ void transpose_fp64_kernel(const double* __restrict__ src, int64_t lds, int32_t m,
                                      int32_t c, double* __restrict__ dst, int64_t ldd) {
    __shared__ double t[32][33];
    const int32_t i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int32_t i = i0 + r, j = j0 + threadIdx.x;
        if (i < m && j < c) t[r][threadIdx.x] = src[(int64_t)i * lds + j];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int32_t j = j0 + r, i = i0 + threadIdx.x;
        if (i < m && j < c) dst[(int64_t)j * ldd + i] = t[threadIdx.x][r];
    }
}

// M[i][j] = M[j][i] for j > i (the lower triangle mirrored onto the upper),
// one 32 x 32 tile pair per block.
__global__ void mirror_lower_kernel(double* __restrict__ M, int32_t n) {
    __shared__ double t[32][33];
    const int32_t bi = blockIdx.y, bj = blockIdx.x;  // source tile (bi, bj), bi >= bj
    if (bj > bi) return;
    const int32_t i0 = bi * 32, j0 = bj * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int32_t i = i0 + r, j = j0 + threadIdx.x;
        if (i < n && j < n) t[r][threadIdx.x] = M[(int64_t)i * n + j];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int32_t row = j0 + r, col = i0 + threadIdx.x;  // (row, col) = (j, i)
        if (row < n && col < n && col > row) M[(int64_t)row * n + col] = t[threadIdx.x][r];
    }
}

// Triangular solves keep the 64x64 diagonal inverse, one 64x64 tile of L and
// the block of right-hand sides in shared memory, staged with coalesced loads.
constexpr int TP = NB + 1;

// (L L^T) X = B in one cooperative launch. Forward: for each 64-block kb every
// CTA recomputes y = inv(L_kk) b_kk in shared memory, CTA 0 stores it, and the
// CTAs update the row blocks after kb that they own (block j belongs to CTA
// (j - kb - 1) mod G); one grid barrier per block. Backward mirrors it with
// inv(L_kk)^T and the column blocks before kb. B is overwritten with X; W is
// scratch of the same shape. Requires all G CTAs resident (cooperative launch).
__global__ void __launch_bounds__(256)
chol_solve_coop_kernel(const double* __restrict__ L, const double* __restrict__ Linv, int32_t n,
                       double* __restrict__ B, double* __restrict__ W, int32_t nrhs) {
    cg::grid_group grid = cg::this_grid();
    extern __shared__ double sm[];
    double* li = sm;                 // [NB][TP]
    double* lt = li + NB * TP;       // [NB][TP]
    double* yb = lt + NB * TP;       // [nrhs][NB]
    double* y = yb + nrhs * NB;      // [nrhs][NB]
    const int32_t nb = (n + NB - 1) / NB;
    const int tid = threadIdx.x;
    const int G = gridDim.x;
    // forward: W = inv(L) B
    for (int32_t kb = 0; kb < nb; kb++) {
        const int32_t r0 = kb * NB, s = min(NB, n - r0);
        const double* Li = Linv + (int64_t)kb * NB * NB;
        for (int idx = tid; idx < NB * NB; idx += 256) li[(idx / NB) * TP + idx % NB] = Li[idx];
        for (int idx = tid; idx < nrhs * NB; idx += 256) {
            const int q = idx / NB, m = idx % NB;
            yb[idx] = (m < s) ? B[(int64_t)q * n + r0 + m] : 0.0;
        }
        __syncthreads();
        for (int idx = tid; idx < nrhs * NB; idx += 256) {
            const int q = idx / NB, i = idx % NB;
            double acc = 0.0;
            for (int m = 0; m <= i; m++) acc += li[i * TP + m] * yb[q * NB + m];
            y[idx] = acc;
        }
        __syncthreads();
        if (blockIdx.x == 0)
            for (int idx = tid; idx < nrhs * NB; idx += 256) {
                const int q = idx / NB, i = idx % NB;
                if (i < s) W[(int64_t)q * n + r0 + i] = y[idx];
            }
        for (int32_t jb = kb + 1 + blockIdx.x; jb < nb; jb += G) {
            const int32_t row0 = jb * NB;
            __syncthreads();
            for (int idx = tid; idx < NB * NB; idx += 256) {
                const int rr = idx / NB, m = idx % NB;
                lt[rr * TP + m] = (row0 + rr < n && m < s) ? L[(int64_t)(row0 + rr) * n + r0 + m] : 0.0;
            }
            __syncthreads();
            for (int idx = tid; idx < nrhs * NB; idx += 256) {
                const int q = idx / NB, rr = idx % NB;
                if (row0 + rr >= n) continue;
                double acc = 0.0;
#pragma unroll 8
                for (int m = 0; m < NB; m++) acc += lt[rr * TP + m] * y[q * NB + m];
                B[(int64_t)q * n + row0 + rr] -= acc;
            }
        }
        grid.sync();
    }
    // backward: B = inv(L)^T W
    for (int32_t kb = nb - 1; kb >= 0; kb--) {
        const int32_t r0 = kb * NB, s = min(NB, n - r0);
        const double* Li = Linv + (int64_t)kb * NB * NB;
        for (int idx = tid; idx < NB * NB; idx += 256) li[(idx / NB) * TP + idx % NB] = Li[idx];
        for (int idx = tid; idx < nrhs * NB; idx += 256) {
            const int q = idx / NB, m = idx % NB;
            yb[idx] = (m < s) ? W[(int64_t)q * n + r0 + m] : 0.0;
        }
        __syncthreads();
        for (int idx = tid; idx < nrhs * NB; idx += 256) {
            const int q = idx / NB, i = idx % NB;
            double acc = 0.0;
            for (int m = i; m < NB; m++) acc += li[m * TP + i] * yb[q * NB + m];
            y[idx] = acc;
        }
        __syncthreads();
        if (blockIdx.x == 0)
            for (int idx = tid; idx < nrhs * NB; idx += 256) {
                const int q = idx / NB, i = idx % NB;
                if (i < s) B[(int64_t)q * n + r0 + i] = y[idx];
            }
        for (int32_t jb = blockIdx.x; jb < kb; jb += G) {
            const int32_t col0 = jb * NB;
            __syncthreads();
            for (int idx = tid; idx < NB * NB; idx += 256) {
                const int r = idx / NB, cc = idx % NB;
                lt[r * TP + cc] = (r < s) ? L[(int64_t)(r0 + r) * n + col0 + cc] : 0.0;
            }
            __syncthreads();
            for (int idx = tid; idx < nrhs * NB; idx += 256) {
                const int q = idx / NB, cc = idx % NB;
                double acc = 0.0;
#pragma unroll 8
                for (int r = 0; r < NB; r++) acc += lt[r * TP + cc] * y[q * NB + r];
                W[(int64_t)q * n + col0 + cc] -= acc;
            }
        }
        grid.sync();
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
// Y^T coef for nu <= 16 coefficient vectors (coef[q]: k multipliers, then the
// 3 scaled mu), Y k x m (block layout), split over ks chunks of rows s:
// part[ks][q][t] = -sum_{s in chunk ks} Y[s][t] coef[q][s], s in order. The
// number of chunks depends on k only, so every caller sums in the same order.
constexpr int kYcMaxQ = 16;
inline int32_t ycomb_chunks(int32_t k) { return k >= 512 ? min(32, k / 256) : 1; }

__global__ void __launch_bounds__(256)
ycomb_part_kernel(const double* __restrict__ Y, int32_t k, int64_t m,
                  const double* __restrict__ coef, int32_t nu, double* __restrict__ part) {
    constexpr int kChunk = 64;
    __shared__ double cs[kChunk][kYcMaxQ];
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int32_t ks = blockIdx.y, nks = gridDim.y;
    const int32_t per = (k + nks - 1) / nks;
    const int32_t sb = ks * per, se = min(k, sb + per);
    double v[kYcMaxQ];
#pragma unroll
    for (int q = 0; q < kYcMaxQ; q++) v[q] = 0.0;
    for (int32_t s0 = sb; s0 < se; s0 += kChunk) {
        const int32_t n = min(kChunk, se - s0);
        __syncthreads();
        for (int e = threadIdx.x; e < kChunk * kYcMaxQ; e += blockDim.x) {
            const int q = e / kChunk, j = e % kChunk;
            cs[j][q] = (q < nu && j < n) ? coef[(size_t)q * (k + 3) + s0 + j] : 0.0;
        }
        __syncthreads();
        if (t < m) {
            for (int j = 0; j < n; j++) {
                const double y = Y[(int64_t)(s0 + j) * m + t];
#pragma unroll
                for (int q = 0; q < kYcMaxQ; q++)
                    if (q < nu) v[q] -= y * cs[j][q];
            }
        }
    }
    if (t >= m) return;
    for (int q = 0; q < nu; q++) part[((int64_t)ks * nu + q) * m + t] = v[q];
}

// x = w - Y^T coef - mu term (one vector, block layout; w may be null).
__global__ void combine_final_kernel(const double* __restrict__ w, const double* __restrict__ part,
                                     int32_t nks, int32_t k, const double* __restrict__ coef,
                                     int32_t V, double* __restrict__ x) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t m = 3 * (int64_t)V;
    if (t >= m) return;
    double v = w ? w[t] : 0.0;
    for (int32_t ks = 0; ks < nks; ks++) v += part[(int64_t)ks * m + t];
    v -= coef[k + (int32_t)(t / V)];
    x[t] = v;
}

// cur[idx[q]] (interleaved V x 3) += -Y^T coef[q] - mu term, flagging non-finite
// corrections in bad[idx[q]]; the same sums as combine_final_kernel with w = 0.
__global__ void proj_final_kernel(double* __restrict__ cur, int64_t stride,
                                  const double* __restrict__ part, int32_t nks, int32_t nu,
                                  int32_t k, const double* __restrict__ coef,
                                  const int32_t* __restrict__ idx, int32_t V,
                                  int32_t* __restrict__ bad) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t m = 3 * (int64_t)V;
    const int q = blockIdx.y;
    if (t >= m) return;
    double v = 0.0;
    for (int32_t ks = 0; ks < nks; ks++) v += part[((int64_t)ks * nu + q) * m + t];
    const int c = (int)(t / V);
    v -= coef[(size_t)q * (k + 3) + k + c];
    const int a = idx[q];
    if (!isfinite(v)) bad[a] = 1;
    double* p = cur + (int64_t)a * stride + 3 * (t % V) + c;
    *p = *p + v;
}

// Residual rows: top (3V): A x_c + (C^T lam)_c - rhs ; one thread per (c, i),
// grouped so each A row is read once for the three blocks; ctl = C^T lam
// (precomputed, null when k = 0). res (optional) receives rhs - (A x + C^T lam).
__global__ void __launch_bounds__(256)
residual_top_kernel(const double* __restrict__ A, int32_t V, const double* __restrict__ ctl,
                    const double* __restrict__ x, const double* __restrict__ rhs,
                    double* __restrict__ out_res, double* __restrict__ out_rhs,
                    double* __restrict__ res) {
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
        double r2 = 0.0, b2 = 0.0;
        double s[3] = {s0, s1, s2};
        for (int c = 0; c < 3; c++) {
            const int64_t row = (int64_t)c * V + i;
            double v = s[c];
            if (ctl) v += ctl[row];
            const double d = v - rhs[row];
            if (res) res[row] = -d;
            r2 += d * d;
            b2 += rhs[row] * rhs[row];
        }
        out_res[i] = r2;
        out_rhs[i] = b2;
    }
}

// out[row] = sum_r C[r][row] lam[r] (C k x m row-major), r in order.
__global__ void __launch_bounds__(256)
ct_lambda_kernel(const double* __restrict__ C, int32_t k, int64_t m, const double* __restrict__ lam,
                 double* __restrict__ out) {
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    double v = 0.0;
    for (int32_t r = 0; r < k; r++) v += C[(int64_t)r * m + row] * lam[r];
    out[row] = v;
}

inline int32_t grid_for(int64_t n, int bs) { return (int32_t)((n + bs - 1) / bs); }

}  // namespace

int32_t cholesky_fp64(tpe_ctx* ctx, double* d_L, double* d_Linv, int32_t n, double piv_tol,
                      int32_t* singular) {
    // Right-looking, outer panels of 256 columns, with look-ahead. On the main
    // stream: each 64-column block of the panel is factored (potrf_diag), every
    // row below it is solved against the block (trsm_panel: A_ik inv(L_kk)^T)
    // and the rest of the panel gets the rank-64 update. On the second stream:
    // the trailing matrix gets the rank-256 update, first the columns of the
    // next panel (which the main stream waits for) and then the rest, which
    // overlaps the next panel's factorization (disjoint columns).
    const int32_t nb = (n + NB - 1) / NB;
    constexpr int32_t OUT = 4;  // 64-blocks per outer panel
    const int32_t nsteps = (nb + OUT - 1) / OUT;
    TPE_TRY(ensure(ctx, ctx->status, sizeof(int32_t) * 4));
    int32_t* st = ctx->status.as<int32_t>();
    TPE_CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(int32_t), ctx->stream));
    const size_t sm1 = sizeof(double) * 2 * NB * (NB + 1);
    const size_t sm0 = sizeof(double) * 3 * NB * (NB + 1);
    const size_t smg = sizeof(double) * 4 * GT * GP;
    TPE_CUDA_TRY(cudaFuncSetAttribute(potrf_diag_kernel<double>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm0));
    TPE_CUDA_TRY(cudaFuncSetAttribute(trsm_panel_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
    auto update = (n & 1) ? gemm_lower_update_kernel<false> : gemm_lower_update_kernel<true>;
    TPE_CUDA_TRY(cudaFuncSetAttribute(update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smg));
    while ((int32_t)ctx->fac_events.size() < 2 * nsteps + 2) {
        cudaEvent_t e;
        TPE_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->fac_events.push_back(e);
    }
    cudaEvent_t* ev = ctx->fac_events.data();
    int64_t launches = 0;
    for (int32_t K0b = 0; K0b < nb; K0b += OUT) {
        const int32_t kend = min(nb, K0b + OUT);
        for (int32_t kb = K0b; kb < kend; kb++)
            launches += 1 + (nb - kb - 1 > 0 ? 1 : 0) + (kb + 1 < kend ? 1 : 0);
        launches += kend < nb ? 1 : 0;
        launches += (kend + OUT) * NB < n ? 1 : 0;
    }
    KernelScope ks(ctx, TPE_KGROUP_CHOLESKY, launches);
    cudaStream_t sa = ctx->stream, sb = ctx->stream2;
    // the second stream starts after everything already queued on the main one
    TPE_CUDA_TRY(cudaEventRecord(ev[2 * nsteps], sa));
    TPE_CUDA_TRY(cudaStreamWaitEvent(sb, ev[2 * nsteps], 0));
    for (int32_t s = 0; s < nsteps; s++) {
        const int32_t K0b = s * OUT, kend = min(nb, K0b + OUT);
        if (s > 0) TPE_CUDA_TRY(cudaStreamWaitEvent(sa, ev[2 * (s - 1) + 1], 0));
        for (int32_t kb = K0b; kb < kend; kb++) {
            potrf_diag_kernel<double><<<1, 256, sm0, sa>>>(d_L, d_Linv, n, kb, piv_tol, st);
            const int32_t rest = nb - kb - 1;
            if (rest > 0) trsm_panel_kernel<<<rest, 256, sm1, sa>>>(d_L, d_Linv, n, kb);
            if (kb + 1 < kend) {
                const int32_t r_s = (kb + 1) * NB, c_e = min(n, kend * NB);
                dim3 g((c_e - r_s + GT - 1) / GT, (n - r_s + GT - 1) / GT);
                update<<<g, 256, smg, sa>>>(d_L, n, r_s, r_s, c_e, kb * NB, NB);
            }
        }
        TPE_CUDA_TRY(cudaEventRecord(ev[2 * s], sa));
        if (kend < nb) {
            TPE_CUDA_TRY(cudaStreamWaitEvent(sb, ev[2 * s], 0));
            const int32_t r_s = kend * NB, c_next = min(n, (kend + OUT) * NB);
            const int32_t k0 = K0b * NB, kl = (kend - K0b) * NB;
            dim3 g1((c_next - r_s + GT - 1) / GT, (n - r_s + GT - 1) / GT);
            update<<<g1, 256, smg, sb>>>(d_L, n, r_s, r_s, c_next, k0, kl);
            TPE_CUDA_TRY(cudaEventRecord(ev[2 * s + 1], sb));
            if (c_next < n) {
                dim3 g2((n - c_next + GT - 1) / GT, (n - c_next + GT - 1) / GT);
                update<<<g2, 256, smg, sb>>>(d_L, n, c_next, c_next, n, k0, kl);
            }
        }
    }
    TPE_CUDA_TRY(cudaEventRecord(ev[2 * nsteps + 1], sb));
    TPE_CUDA_TRY(cudaStreamWaitEvent(sa, ev[2 * nsteps + 1], 0));
    TPE_CUDA_TRY(cudaGetLastError());
    int32_t h = 0;
    TPE_CUDA_TRY(cudaMemcpyAsync(&h, st, sizeof(int32_t), cudaMemcpyDeviceToHost, sa));
    TPE_CUDA_TRY(cudaStreamSynchronize(sa));
    *singular = h;
    return TPE_OK;
}

int32_t chol_solve_fp64(tpe_ctx* ctx, const double* d_L, const double* d_Linv, int32_t n,
                        double* d_B, int32_t nrhs) {
    if (nrhs <= 0) return TPE_OK;
    if (nrhs > 64) {
        set_error(ctx, TPE_ERR_TOO_LARGE, "chol_solve: at most 64 right-hand sides per call");
        return TPE_ERR_TOO_LARGE;
    }
    const int32_t nb = (n + NB - 1) / NB;
    TPE_TRY(ensure(ctx, ctx->solve_scratch, sizeof(double) * (size_t)n * nrhs));
    double* W = ctx->solve_scratch.as<double>();
    const size_t smem = sizeof(double) * (2 * (size_t)NB * TP + 2 * (size_t)nrhs * NB);
    const int smax = (int)(sizeof(double) * (2 * NB * TP + 2 * 64 * NB));
    TPE_CUDA_TRY(cudaFuncSetAttribute(chol_solve_coop_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
    int per_sm = 0;
    TPE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chol_solve_coop_kernel, 256,
                                                               smem));
    int G = per_sm * ctx->num_sms;
    if (G > nb) G = nb;
    if (G < 1) {
        set_error(ctx, TPE_ERR_CUDA, "chol_solve: cooperative kernel does not fit on an SM");
        return TPE_ERR_CUDA;
    }
    KernelScope ks(ctx, TPE_KGROUP_TRSV, 1);
    void* args[] = {(void*)&d_L, (void*)&d_Linv, (void*)&n, (void*)&d_B, (void*)&W, (void*)&nrhs};
    TPE_CUDA_TRY(cudaLaunchCooperativeKernel((void*)chol_solve_coop_kernel, dim3(G), dim3(256), args,
                                             smem, ctx->stream));
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
    return download_on(ctx, ctx->stream, out, dst, sizeof(double));
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
    const int64_t m = 3 * (int64_t)V;
    const int32_t nks = ycomb_chunks(k);
    TPE_TRY(ensure(ctx, ctx->ycomb_part, sizeof(double) * (size_t)nks * kYcMaxQ * m));
    double* part = ctx->ycomb_part.as<double>();
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 2);
    ycomb_part_kernel<<<dim3(grid_for(m, 256), nks), 256, 0, ctx->stream>>>(d_Y, k, m, dc, 1, part);
    combine_final_kernel<<<grid_for(m, 256), 256, 0, ctx->stream>>>(d_w, part, nks, k, dc, V, d_x);
    TPE_CUDA_TRY(cudaGetLastError());
    TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return TPE_OK;
}

int32_t project_update(tpe_ctx* ctx, const double* d_Y, int32_t k, int32_t V, const double* d_coef,
                       int32_t nu, const int32_t* d_idx, double* d_cur, int64_t stride,
                       int32_t* d_bad) {
    if (nu <= 0) return TPE_OK;
    if (nu > kYcMaxQ) {
        set_error(ctx, TPE_ERR_TOO_LARGE, "project_update: at most 16 trials per update");
        return TPE_ERR_TOO_LARGE;
    }
    const int64_t m = 3 * (int64_t)V;
    const int32_t nks = ycomb_chunks(k);
    TPE_TRY(ensure(ctx, ctx->ycomb_part, sizeof(double) * (size_t)nks * kYcMaxQ * m));
    double* part = ctx->ycomb_part.as<double>();
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 2);
    ycomb_part_kernel<<<dim3(grid_for(m, 256), nks), 256, 0, ctx->stream>>>(d_Y, k, m, d_coef, nu,
                                                                            part);
    proj_final_kernel<<<dim3(grid_for(m, 256), nu), 256, 0, ctx->stream>>>(
        d_cur, stride, part, nks, nu, k, d_coef, d_idx, V, d_bad);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t saddle_residual(tpe_ctx* ctx, const double* d_A, int32_t V, const double* d_C, int32_t k,
                        const double* d_x, const double* lam, const double* d_rhs_top,
                        const double* rhs_bottom, double* out, double* d_res_top,
                        double* res_bottom) {
    const int64_t m = 3 * (int64_t)V;
    TPE_TRY(ensure(ctx, ctx->tmp, sizeof(double) * (size_t)(2 * V + 16 + k + m)));
    TPE_TRY(ensure(ctx, ctx->scalars, sizeof(double) * (size_t)(k + 3 + 512)));
    double* dl = ctx->scalars.as<double>() + 264;
    if (k > 0)
        TPE_CUDA_TRY(cudaMemcpyAsync(dl, lam, sizeof(double) * k, cudaMemcpyHostToDevice,
                                     ctx->stream));
    double* rr = ctx->tmp.as<double>();
    double* rb = rr + V;
    double* ctl = rb + V + 16 + k;
    {
        KernelScope ks(ctx, TPE_KGROUP_OTHER, k > 0 ? 2 : 1);
        if (k > 0)
            ct_lambda_kernel<<<grid_for(m, 256), 256, 0, ctx->stream>>>(d_C, k, m, dl, ctl);
        residual_top_kernel<<<V, 256, 0, ctx->stream>>>(d_A, V, k > 0 ? ctl : nullptr, d_x, d_rhs_top,
                                                        rr, rb, d_res_top);
    }
    TPE_CUDA_TRY(cudaGetLastError());
    double top_r = 0.0, top_b = 0.0;
    TPE_TRY(dot(ctx, V, rr, nullptr, &top_r));
    TPE_TRY(dot(ctx, V, rb, nullptr, &top_b));
    // bottom rows C x - rhs_bottom
    double bot_r = 0.0, bot_b = 0.0;
    if (k > 0) {
        double* cx = ctx->tmp.as<double>() + 2 * V;
        TPE_TRY(gram_dots(ctx, d_C, k, d_x, 1, 3 * (int64_t)V, cx));
        std::vector<double> h((size_t)k);
        TPE_CUDA_TRY(cudaMemcpyAsync(h.data(), cx, sizeof(double) * k, cudaMemcpyDeviceToHost,
                                     ctx->stream));
        TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        for (int32_t r = 0; r < k; r++) {
            const double b = rhs_bottom ? rhs_bottom[r] : 0.0;
            const double d = h[r] - b;
            if (res_bottom) res_bottom[r] = -d;
            bot_r += d * d;
            bot_b += b * b;
        }
    }
    const double rn = sqrt(top_r + bot_r), bn = sqrt(top_b + bot_b);
    *out = rn / (bn > 1.0 ? bn : 1.0);
    return TPE_OK;
}

int32_t dgemm_nt(tpe_ctx* ctx, const DGemmArgs& g, cudaStream_t stream) {
    if (g.M <= 0 || g.N <= 0) return TPE_OK;
    const bool al = ((((uintptr_t)g.A) | ((uintptr_t)g.B)) & 15) == 0 && (g.lda & 1) == 0 &&
                    (g.ldb & 1) == 0;
    auto kern = al ? dgemm_nt_kernel<true> : dgemm_nt_kernel<false>;
    const size_t smem = sizeof(double) * 4 * GT * GP;
    TPE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((g.N + GT - 1) / GT), (unsigned)((g.M + GT - 1) / GT));
    kern<<<grid, 256, smem, stream>>>(g);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

namespace {
// X[r1.., r1..] for the 64-blocks [b0, b0 + nblk): recursive halving,
// X21 = -X22 L21 X11 from T^T = W11 L21^T, then W12 = X21^T.
int32_t inverse_blocks(tpe_ctx* ctx, const double* L, int32_t n, double* X, double* W,
                       double* Tt, int32_t b0, int32_t nblk, int64_t* launches) {
    if (nblk <= 1) return TPE_OK;
    const int32_t h = nblk / 2;
    TPE_TRY(inverse_blocks(ctx, L, n, X, W, Tt, b0, h, launches));
    TPE_TRY(inverse_blocks(ctx, L, n, X, W, Tt, b0 + h, nblk - h, launches));
    const int32_t r1 = b0 * NB, m1 = h * NB, r2 = r1 + m1;
    const int32_t m2 = min(n, (b0 + nblk) * NB) - r2;
    DGemmArgs t;  // T^T (m1 x m2) = W11 L21^T
    t.A = W + (int64_t)r1 * n + r1;
    t.lda = n;
    t.B = L + (int64_t)r2 * n + r1;
    t.ldb = n;
    t.C = Tt;
    t.ldc = m2;
    t.M = m1;
    t.N = m2;
    t.K = m1;
    t.mode = kDAUpper;
    TPE_TRY(dgemm_nt(ctx, t, ctx->stream));
    DGemmArgs u;  // X21 (m2 x m1) = -X22 T
    u.A = X + (int64_t)r2 * n + r2;
    u.lda = n;
    u.B = Tt;
    u.ldb = m2;
    u.C = X + (int64_t)r2 * n + r1;
    u.ldc = n;
    u.M = m2;
    u.N = m1;
    u.K = m2;
    u.alpha = -1.0;
    u.mode = kDALower;
    TPE_TRY(dgemm_nt(ctx, u, ctx->stream));
    transpose_fp64_kernel<<<dim3((m1 + 31) / 32, (m2 + 31) / 32), dim3(32, 8), 0, ctx->stream>>>(
        X + (int64_t)r2 * n + r1, n, m2, m1, W + (int64_t)r1 * n + r2, n);
    TPE_CUDA_TRY(cudaGetLastError());
    *launches += 3;
    return TPE_OK;
}
}  // namespace

int32_t lower_inverse_fp64(tpe_ctx* ctx, const double* d_L, const double* d_Linv, int32_t n,
                           double* X, double* W, double* Tt) {
    const int32_t nb = (n + NB - 1) / NB;
    int64_t launches = 0;
    KernelScope ks(ctx, TPE_KGROUP_TRSV, 1 + 3 * (int64_t)(nb - 1));
    TPE_CUDA_TRY(cudaMemsetAsync(X, 0, sizeof(double) * (size_t)n * n, ctx->stream));
    TPE_CUDA_TRY(cudaMemsetAsync(W, 0, sizeof(double) * (size_t)n * n, ctx->stream));
    diag_inverse_kernel<<<nb, 256, 0, ctx->stream>>>(d_Linv, n, X, W);
    TPE_CUDA_TRY(cudaGetLastError());
    return inverse_blocks(ctx, d_L, n, X, W, Tt, 0, nb, &launches);
}

int32_t transpose_fp64(tpe_ctx* ctx, const double* src, int64_t lds, int32_t m, int32_t c,
                       double* dst, int64_t ldd) {
    KernelScope ks(ctx, TPE_KGROUP_TRSV, 1);
    transpose_fp64_kernel<<<dim3((c + 31) / 32, (m + 31) / 32), dim3(32, 8), 0, ctx->stream>>>(
        src, lds, m, c, dst, ldd);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t mirror_lower(tpe_ctx* ctx, double* M, int32_t n) {
    KernelScope ks(ctx, TPE_KGROUP_TRSV, 1);
    const unsigned nt = (unsigned)((n + 31) / 32);
    mirror_lower_kernel<<<dim3(nt, nt), dim3(32, 8), 0, ctx->stream>>>(M, n);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t spd_inverse_fp64(tpe_ctx* ctx, const double* d_L, const double* d_Linv, int32_t n,
                         double* X, double* W, double* Tt, double* out) {
    TPE_TRY(lower_inverse_fp64(ctx, d_L, d_Linv, n, X, W, Tt));
    KernelScope ks(ctx, TPE_KGROUP_TRSV, 2);
    DGemmArgs g;  // out = X^T X = W W^T (lower tiles; W[i][k] = 0 for k < i)
    g.A = W;
    g.lda = n;
    g.B = W;
    g.ldb = n;
    g.C = out;
    g.ldc = n;
    g.M = g.N = g.K = n;
    g.mode = kDLowerTiles | kDAUpper;
    TPE_TRY(dgemm_nt(ctx, g, ctx->stream));
    const unsigned nt = (unsigned)((n + 31) / 32);
    mirror_lower_kernel<<<dim3(nt, nt), dim3(32, 8), 0, ctx->stream>>>(out, n);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

}  // namespace tpe
