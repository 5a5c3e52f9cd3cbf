// Mixed-precision saddle solve: the factorization of A_rho runs on the tensor
// cores in FP32, the solution is made FP64-accurate by preconditioned CG.
//
// The FP64 path factors A_rho = A + (rho/V) 1 1^T (dense.cu) and back-substitutes.
// Here the same SPD matrix is
//   1. Jacobi-scaled, S = D A_rho D with D = diag(A_rho)^(-1/2), and rounded
//      to FP32 (padded to Vp, the next multiple of 128, with an identity block);
//   2. factored S ~ L L^T in FP32: 128 x 128 diagonal blocks in one CTA
//      (potrf128_kernel, which also inverts them), the panel solve and the
//      trailing update as 3xTF32 tcgen05 GEMMs (tc_gemm.cu);
//   3. inverted, Z = L^{-1}, by the recursive block formula
//      Z21 = -Z22 L21 Z11: the rows split into a first part of 128 * 2^k rows
//      (the largest such part below Vp) and the rest, recursively; inside a
//      part of 128 * 2^k rows level by level, all blocks of a level batched
//      into one tcgen05 GEMM; W = Z^T is kept beside Z so every product is an
//      A * B^T of row-major operands;
//   4. used as the preconditioner M = Z^T Z = (L L^T)^{-1} of a block CG on
//      S y = D b in FP64, x = D y. Z and W are copied once to plain FP32
//      (hi + lo is exact in FP32) and every product of the CG -- S p with the
//      FP64 A, Z r and W u with the FP32 copies -- runs in FP64 arithmetic on
//      the FP64 tensor cores (mrhs_dmma_kernel).
// At V=8192 (kappa(A_rho) ~ 1e10, kappa(S) ~ 1e8) plain iterative refinement
// with an FP32 factor diverges (kappa(S) * u32 > 1); CG with it reaches a 1e-13
// relative residual in about 7 iterations. The FP64 path remains the fallback
// whenever the FP32 factorization breaks down or CG does not converge.
#include <math.h>

#include <algorithm>

#include "tc.h"
#include "tpe_internal.h"

namespace tpe {
namespace {

constexpr int kT = 128;       // diagonal block = GEMM tile
constexpr int kMaxRhs = 16;   // right-hand sides per CG pass

__host__ __device__ __forceinline__ void split32(float x, float& hi, float& lo) {
    union {
        float f;
        uint32_t u;
    } v;
    v.f = x;
    v.u = (v.u + 0x1000u) & 0xFFFFE000u;
    hi = v.f;
    lo = x - hi;
}

// d_i = 1 / sqrt(A_ii + shift) and dinv_i = 1 / d_i for real rows, 1 on the pad.
__global__ void jacobi_kernel(const double* __restrict__ A, int32_t V, int32_t Vp, double shift,
                              double* __restrict__ d, double* __restrict__ dinv) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Vp) return;
    const double s = i < V ? sqrt(A[(size_t)i * V + i] + shift) : 1.0;
    d[i] = 1.0 / s;
    dinv[i] = s;
}

// S (Vp x Vp, FP32, ld Vp) = D (A + shift) D, identity on the pad.
// S[i][j] = d_i (A_ij + shift) d_j rounded to FP32 for i, j < V, the identity on
// the pad. Four consecutive columns per thread (two 16-byte loads of A when V is
// even, one 16-byte store of S); grid (ceil(Vp / 1024), rows), rows strided.
__global__ void __launch_bounds__(256) scale_to_f32_kernel(const double* __restrict__ A, int32_t V,
                                                           int32_t Vp, double shift,
                                                           const double* __restrict__ d,
                                                           float* __restrict__ S) {
    const int32_t j = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (j >= Vp) return;
    for (int32_t i = blockIdx.y; i < Vp; i += gridDim.y) {
        float o[4];
        if (i < V && j + 3 < V && (V & 1) == 0) {
            const double di = d[i];
            const double2 a0 = *reinterpret_cast<const double2*>(A + (size_t)i * V + j);
            const double2 a1 = *reinterpret_cast<const double2*>(A + (size_t)i * V + j + 2);
            const double2 d0 = *reinterpret_cast<const double2*>(d + j);
            const double2 d1 = *reinterpret_cast<const double2*>(d + j + 2);
            o[0] = (float)(di * (a0.x + shift) * d0.x);
            o[1] = (float)(di * (a0.y + shift) * d0.y);
            o[2] = (float)(di * (a1.x + shift) * d1.x);
            o[3] = (float)(di * (a1.y + shift) * d1.y);
        } else {
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int32_t jj = j + c;
                o[c] = (i < V && jj < V) ? (float)(d[i] * (A[(size_t)i * V + jj] + shift) * d[jj])
                                         : (i == jj ? 1.0f : 0.0f);
            }
        }
        *reinterpret_cast<float4*>(S + (size_t)i * Vp + j) = make_float4(o[0], o[1], o[2], o[3]);
    }
}

// L[r0+i][c0+j] = split(S[r0+i][c0+j]) for i < rows, j < 128 (ld shared).
__global__ void split_copy_kernel(const float* __restrict__ S, int32_t ld, int32_t r0, int32_t c0,
                                  int32_t rows, float* __restrict__ hi, float* __restrict__ lo) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)rows * kT) return;
    const size_t o = (size_t)(r0 + t / kT) * ld + c0 + (t % kT);
    float h, l;
    split32(S[o], h, l);
    hi[o] = h;
    lo[o] = l;
}

constexpr int kLd3 = 132;   // row stride of a and z (16-byte aligned rows)
constexpr int kP3 = 100;    // row stride of plT (the panel, transposed)
constexpr int kS3 = 36;     // row stride of the 32 x 32 scratch blocks
constexpr int kTs3 = 36;    // row stride of the off-diagonal T scratch
constexpr int kPw3 = 32;

// shared-memory offsets (floats)
constexpr int kOffA = 0;
constexpr int kOffZ = kOffA + kT * kLd3;
constexpr int kOffP = kOffZ + kT * kLd3;               // plT: 32 x kP3, also the final T scratch
constexpr int kPSize = 3 * 32 * kTs3 > 32 * kP3 ? 3 * 32 * kTs3 : 32 * kP3;
constexpr int kOffTsc = kOffP + kPSize;               // 2 x 32 x kTs3
constexpr int kOffRd = kOffTsc + 2 * 32 * kTs3;       // 128
constexpr int kOffZdT = kOffRd + kT;                  // 32 x kS3: Z_dd^T of the current panel
constexpr int kOffLt = kOffZdT + 32 * kS3;            // 32 x kS3: L_dd^T (wf32 scratch)
constexpr int kSmem3Floats = kOffLt + 32 * kS3;
static_assert(kOffZ % 4 == 0 && kOffP % 4 == 0 && kOffTsc % 4 == 0 && kOffZdT % 4 == 0 &&
              kOffLt % 4 == 0, "float4 alignment");

__device__ __forceinline__ void tri_decode(int e, int& ti, int& tj) {
    int t = (int)((sqrtf(8.0f * (float)e + 1.0f) - 1.0f) * 0.5f);
    while ((t + 1) * (t + 2) / 2 <= e) t++;
    while (t * (t + 1) / 2 > e) t--;
    ti = t;
    tj = e - t * (t + 1) / 2;
}

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float f4(const float4& v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// One warp factors the 32 x 32 diagonal part at (c0, c0) of a (lane = row) and
// inverts it: one rank-1 update per column by shuffles, with each column's
// pivot formed ahead on its own lane. The inverse (lane = column of Z) reads L
// column-wise from a transposed copy. Writes L to a, Z (lower) to z, Z^T to zdt, 1/L_ii to rd.
__device__ __noinline__ void warp_factor32(float* sm, int c0, int lane, int32_t* bad) {
    float* a = sm + kOffA;
    float* z = sm + kOffZ;
    float* rd = sm + kOffRd;
    float* zdt = sm + kOffZdT;
    float* lt = sm + kOffLt;
    float v[32];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const float4 x = ld4(a + (c0 + lane) * kLd3 + c0 + 4 * q);
        v[4 * q] = (4 * q <= lane) ? x.x : 0.0f;
        v[4 * q + 1] = (4 * q + 1 <= lane) ? x.y : 0.0f;
        v[4 * q + 2] = (4 * q + 2 <= lane) ? x.z : 0.0f;
        v[4 * q + 3] = (4 * q + 3 <= lane) ? x.w : 0.0f;
    }
    bool brk = false;
    float myrs = 1.0f;
    // The pivot of column K + 1 is formed on its own lane right after column K
    // (dn = v[K+1] - L[K+1][K]^2: the last update of that diagonal entry uses
    // the lane's own value) and broadcast before column K's other updates, so
    // the pivot chain holds one shuffle per column; the updates themselves run
    // in the same order as one rank-1 update per column.
    float piv = __shfl_sync(0xffffffffu, v[0], 0);
#pragma unroll
    for (int K = 0; K < 32; K++) {
        if (!(piv > 0.0f) || !isfinite(piv)) {
            brk = true;
            piv = 1.0f;
        }
        const float rs = rsqrtf(piv);
        const float lk = (lane == K) ? piv * rs : v[K] * rs;  // L[lane][K] (lanes >= K)
        if (lane >= K) v[K] = lk;
        if (lane == K) myrs = rs;
        float pnext = 0.0f;
        if (K + 1 < 32) pnext = __shfl_sync(0xffffffffu, fmaf(-lk, lk, v[K + 1]), K + 1);
#pragma unroll
        for (int m = K + 1; m < 32; m++) {
            const float lmk = __shfl_sync(0xffffffffu, lk, m);
            if (lane >= m) v[m] = fmaf(-lk, lmk, v[m]);
        }
        piv = pnext;
    }
    if (brk && lane == 0) atomicExch(bad, 1);
    // L back to a (rows, 16-byte stores), L^T to lt (lt[k][lane] = L[lane][k]), 1/L_ii
#pragma unroll
    for (int q = 0; q < 8; q++)
        st4(a + (c0 + lane) * kLd3 + c0 + 4 * q, make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]));
#pragma unroll
    for (int k = 0; k < 32; k++) lt[k * kS3 + lane] = v[k];
    rd[c0 + lane] = myrs;
    __syncwarp();
    // inverse, lane = column j: x[i] = Z[i][j]
    float x[32];
#pragma unroll
    for (int i = 0; i < 32; i++) x[i] = (i == lane) ? 1.0f : 0.0f;
    float rdv[32];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const float4 r4 = ld4(rd + c0 + 4 * q);
        rdv[4 * q] = r4.x;
        rdv[4 * q + 1] = r4.y;
        rdv[4 * q + 2] = r4.z;
        rdv[4 * q + 3] = r4.w;
    }
#pragma unroll
    for (int k = 0; k < 32; k++) {
        x[k] *= rdv[k];
#pragma unroll
        for (int q = (k + 1) / 4; q < 8; q++) {
            const float4 l4 = ld4(lt + k * kS3 + 4 * q);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int i = 4 * q + u;
                if (i > k) x[i] = fmaf(-f4(l4, u), x[k], x[i]);
            }
        }
    }
    // Z rows to z (column lane), Z^T rows to zdt (row lane)
#pragma unroll
    for (int i = 0; i < 32; i++) z[(c0 + i) * kLd3 + c0 + lane] = (i >= lane) ? x[i] : 0.0f;
#pragma unroll
    for (int q = 0; q < 8; q++)
        st4(zdt + lane * kS3 + 4 * q,
            make_float4(4 * q >= lane ? x[4 * q] : 0.0f, 4 * q + 1 >= lane ? x[4 * q + 1] : 0.0f,
                        4 * q + 2 >= lane ? x[4 * q + 2] : 0.0f, 4 * q + 3 >= lane ? x[4 * q + 3] : 0.0f));
    __syncwarp();
}

// a[R..R+3][C..C+3] -= P rows (4ti..) P rows (4tj..)^T over the 32 panel columns
// (P transposed in plT).
__device__ __forceinline__ void update_tile(float* a, const float* plt, int ti, int tj, int base) {
    float acc[4][4];
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y] = 0.0f;
#pragma unroll 8
    for (int k = 0; k < kPw3; k++) {
        const float4 pr = ld4(plt + k * kP3 + 4 * ti);
        const float4 pc = ld4(plt + k * kP3 + 4 * tj);
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
            for (int y = 0; y < 4; y++) acc[x][y] += f4(pr, x) * f4(pc, y);
    }
    const int R = base + 4 * ti, Cc = base + 4 * tj;
#pragma unroll
    for (int x = 0; x < 4; x++) {
        float* p = a + (R + x) * kLd3 + Cc;
        float4 o = ld4(p);
        o.x -= acc[x][0];
        o.y -= acc[x][1];
        o.z -= acc[x][2];
        o.w -= acc[x][3];
        st4(p, o);
    }
}

__device__ __forceinline__ void group_sync(int bar, int nthr) {
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nthr) : "memory");
}

// Off-diagonal 32 x 32 blocks of Z inside the block: for each listed pair
// (bi, bj), bj < bi, T = sum_{c=bj}^{bi-1} L_{bi,c} Z_{c,bj}, then
// Z_{bi,bj} = -Z_{bi,bi} T. 64 threads per pair (8 x 8 threads of 4 x 4 outputs).
__device__ void offdiag_blocks(const float* __restrict__ a, float* __restrict__ z,
                                float* __restrict__ tsc, const int* pa, const int* pb, int npairs,
                                int t, int nthr, int bar) {
    const int slot = t >> 6;
    const bool act = slot < npairs;
    const int tr = (t >> 3) & 7, tc = t & 7;
    const int bi = act ? pa[slot] : 0, bj = act ? pb[slot] : 0;
    float acc[4][4];
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y] = 0.0f;
    if (act) {
        for (int k4 = bj * kPw3; k4 < bi * kPw3; k4 += 4) {
            float4 lr[4], zc[4];
#pragma unroll
            for (int x = 0; x < 4; x++) lr[x] = ld4(a + (bi * kPw3 + 4 * tr + x) * kLd3 + k4);
#pragma unroll
            for (int u = 0; u < 4; u++) zc[u] = ld4(z + (k4 + u) * kLd3 + bj * kPw3 + 4 * tc);
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int y = 0; y < 4; y++) acc[x][y] += f4(lr[x], u) * f4(zc[u], y);
        }
#pragma unroll
        for (int x = 0; x < 4; x++)
            st4(tsc + (slot * kPw3 + 4 * tr + x) * kTs3 + 4 * tc,
                make_float4(acc[x][0], acc[x][1], acc[x][2], acc[x][3]));
    }
    group_sync(bar, nthr);
    if (act) {
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
            for (int y = 0; y < 4; y++) acc[x][y] = 0.0f;
        const int qmax = 4 * tr + 4;  // Z_aa is lower: columns q <= row
        for (int q4 = 0; q4 < qmax; q4 += 4) {
            float4 zr[4], tq[4];
#pragma unroll
            for (int x = 0; x < 4; x++) zr[x] = ld4(z + (bi * kPw3 + 4 * tr + x) * kLd3 + bi * kPw3 + q4);
#pragma unroll
            for (int u = 0; u < 4; u++) tq[u] = ld4(tsc + (slot * kPw3 + q4 + u) * kTs3 + 4 * tc);
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int y = 0; y < 4; y++) acc[x][y] += f4(zr[x], u) * f4(tq[u], y);
        }
#pragma unroll
        for (int x = 0; x < 4; x++)
            st4(z + (bi * kPw3 + 4 * tr + x) * kLd3 + bj * kPw3 + 4 * tc,
                make_float4(-acc[x][0], -acc[x][1], -acc[x][2], -acc[x][3]));
    }
    group_sync(bar, nthr);
}

// One CTA factors the 128 x 128 diagonal block at (j0, j0) of S (its lower
// triangle) and writes Z_jj = L_jj^{-1} (split, zero above the diagonal) to Z.
// L_jj itself is not needed outside (the panel solve uses Z_jj, the inverse
// uses only the blocks below the diagonal), and W_jj = Z_jj^T is written by
// diag_transpose_kernel once the whole factorization is done.
//
// Blocked right-looking over four 32-column panels with an in-CTA look-ahead:
// warp 0 factors a panel's 32 x 32 diagonal part in registers and inverts it
// (warp_factor32); all eight warps solve the rows below against that inverse
// (warp = 4 columns, lane = row, the panel stored transposed); then warps 0
// and 1 apply the rank-32 update to the next panel's diagonal part and warp 0
// factors it, while warps 1-7 update the rest of the trailing triangle (4 x 4
// register tiles from 16-byte loads) and form the off-diagonal 32 x 32 blocks
// of the inverse, Z_ab = -Z_aa sum_{b<=c<a} L_ac Z_cb, one block distance at a
// time. Reciprocal square roots are the fast approximate ones: the factor is a
// preconditioner, CG restores FP64 accuracy. *bad = 1 when a pivot is not
// positive and finite. Rows of a and z are 132 floats apart (16-byte aligned),
// so every shared-memory access of the inner loops is a 16-byte one.
__global__ void __launch_bounds__(256, 1)
potrf128_kernel(const float* __restrict__ S, int32_t ld, int32_t j0, float* __restrict__ Zhi,
            float* __restrict__ Zlo, int32_t* __restrict__ bad) {
    extern __shared__ __align__(16) float sm[];
    float* a = sm + kOffA;
    float* z = sm + kOffZ;
    float* plt = sm + kOffP;
    float* zdt = sm + kOffZdT;
    float* tsc = sm + kOffTsc;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        float4 buf[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int e = tid + 256 * q;  // float4 index
            const int r = e >> 5, c = (e & 31) * 4;
            buf[q] = *reinterpret_cast<const float4*>(S + (size_t)(j0 + r) * ld + j0 + c);
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int e = tid + 256 * q;
            const int r = e >> 5, c = (e & 31) * 4;
            st4(a + r * kLd3 + c, buf[q]);
        }
    }
    __syncthreads();
    if (warp == 0) warp_factor32(sm, 0, lane, bad);
    __syncthreads();
    for (int p = 0; p < kT / kPw3 - 1; p++) {
        const int c0 = p * kPw3;
        const int nr = kT - c0 - kPw3;
        // panel rows below: plT[m][r] = sum_k A[c0+32+r][c0+k] * Zd[m][k]
        {
            const int m0 = 4 * warp;
            for (int r0 = 0; r0 < nr; r0 += 32) {
                const int r = r0 + lane;
                const float* arow = a + (c0 + kPw3 + r) * kLd3 + c0;
                float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                for (int k4 = 0; k4 < kPw3; k4 += 4) {
                    const float4 ak = ld4(arow + k4);
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const float4 zk = ld4(zdt + (k4 + u) * kS3 + m0);
                        const float av = f4(ak, u);
                        acc[0] += av * zk.x;
                        acc[1] += av * zk.y;
                        acc[2] += av * zk.z;
                        acc[3] += av * zk.w;
                    }
                }
#pragma unroll
                for (int t = 0; t < 4; t++) plt[(m0 + t) * kP3 + r] = acc[t];
            }
        }
        __syncthreads();
            const int base = c0 + kPw3;
        const int nt = nr / 4;
        const int ntiles = nt * (nt + 1) / 2;
        constexpr int kNext = 36;  // 4 x 4 tiles of the next 32 x 32 diagonal part (packed first)
        if (warp < 2) {
            // warps 0 and 1: the next diagonal part, then warp 0 factors it
            const int e = warp * 18 + lane;
            if (lane < 18) {
                int ti, tj;
                tri_decode(e, ti, tj);
                update_tile(a, plt, ti, tj, base);
            }
            group_sync(3, 64);
        }
        if (warp == 0) {
            warp_factor32(sm, base, lane, bad);
        } else {
            for (int e = kNext + tid - 32; e < ntiles; e += 224) {
                int ti, tj;
                tri_decode(e, ti, tj);
                update_tile(a, plt, ti, tj, base);
            }
            // the panel rows become final L
            for (int e = tid - 32; e < nr * kPw3; e += 224) {
                const int r = e >> 5, m = e & 31;
                a[(base + r) * kLd3 + c0 + m] = plt[m * kP3 + r];
            }
            // while warp 0 factors the next panel: the off-diagonal Z blocks of
            // block row p (inputs final: L columns < 32 p, Z blocks of rows <= p)
            if (p > 0) {
                int pa[2], pb[2];
                for (int q = 0; q < p; q++) {
                    pa[q] = p;
                    pb[q] = p - 1 - q;
                }
                offdiag_blocks(a, z, tsc, pa, pb, p, tid - 32, 224, 1);
            }
        }
        __syncthreads();
        }
    // the last block row of Z: its three off-diagonal blocks at once
    {
        const int pa[3] = {3, 3, 3}, pb[3] = {2, 1, 0};
        offdiag_blocks(a, z, plt, pa, pb, 3, tid, 256, 2);
    }
    // Z_jj (split), four columns per thread step, zero above the diagonal
    for (int e = tid; e < kT * kT / 4; e += 256) {
        const int r = e >> 5, c = (e & 31) * 4;
        const float4 zz = ld4(z + r * kLd3 + c);
        float4 h, l;
        split32(c <= r ? zz.x : 0.0f, h.x, l.x);
        split32(c + 1 <= r ? zz.y : 0.0f, h.y, l.y);
        split32(c + 2 <= r ? zz.z : 0.0f, h.z, l.z);
        split32(c + 3 <= r ? zz.w : 0.0f, h.w, l.w);
        const size_t o = (size_t)(j0 + r) * ld + j0 + c;
        *reinterpret_cast<float4*>(Zhi + o) = h;
        *reinterpret_cast<float4*>(Zlo + o) = l;
    }
    __syncthreads();
}

// W_jj = Z_jj^T for the diagonal blocks b0 + blockIdx.z, split.
__global__ void diag_transpose_kernel(const float* __restrict__ zhi, const float* __restrict__ zlo,
                                      float* __restrict__ whi, float* __restrict__ wlo, int32_t ld,
                                      int32_t b0) {
    __shared__ float th[32][33], tl[32][33];
    const int32_t j0 = (b0 + (int32_t)blockIdx.z) * kT;
    const int32_t r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const size_t o = (size_t)(j0 + r0 + yy) * ld + j0 + c0 + threadIdx.x;
        th[yy][threadIdx.x] = zhi[o];
        tl[yy][threadIdx.x] = zlo[o];
    }
    __syncthreads();
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const size_t o = (size_t)(j0 + c0 + yy) * ld + j0 + r0 + threadIdx.x;
        whi[o] = th[threadIdx.x][yy];
        wlo[o] = tl[threadIdx.x][yy];
    }
}

// W[s + c][s + m + r] = Z[s + m + r][s + c] (r, c < m), s = base + blockIdx.z * 2m.
__global__ void transpose_block_kernel(const float* __restrict__ zhi, const float* __restrict__ zlo,
                                       float* __restrict__ whi, float* __restrict__ wlo,
                                       int32_t ld, int32_t m, int32_t base) {
    __shared__ float th[32][33], tl[32][33];
    const int32_t s = base + (int32_t)blockIdx.z * 2 * m;
    const int32_t r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const size_t o = (size_t)(s + m + r0 + yy) * ld + s + c0 + threadIdx.x;
        th[yy][threadIdx.x] = zhi[o];
        tl[yy][threadIdx.x] = zlo[o];
    }
    __syncthreads();
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const size_t o = (size_t)(s + c0 + yy) * ld + s + m + r0 + threadIdx.x;
        whi[o] = th[threadIdx.x][yy];
        wlo[o] = tl[threadIdx.x][yy];
    }
}

// W[c0 + c][r0 + r] = Z[r0 + r][c0 + c] (r < 32 gridDim.y, c < 32 gridDim.x),
// split: the W12 = Z21^T of an uneven split of the inverse.
__global__ void transpose_rect_kernel(const float* __restrict__ zhi, const float* __restrict__ zlo,
                                      float* __restrict__ whi, float* __restrict__ wlo,
                                      int32_t ld, int32_t r0, int32_t c0) {
    __shared__ float th[32][33], tl[32][33];
    const int32_t rb = r0 + blockIdx.y * 32, cb = c0 + blockIdx.x * 32;
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const size_t o = (size_t)(rb + yy) * ld + cb + threadIdx.x;
        th[yy][threadIdx.x] = zhi[o];
        tl[yy][threadIdx.x] = zlo[o];
    }
    __syncthreads();
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const size_t o = (size_t)(cb + yy) * ld + rb + threadIdx.x;
        whi[o] = th[threadIdx.x][yy];
        wlo[o] = tl[threadIdx.x][yy];
    }
}

// ---- block CG kernels (vectors are [nr][Vp] FP64, pad entries stay 0) ------


// UT[j][c] = d_j P[c][j] for j < V, c < nr (0 elsewhere, up to Vp rows of 16),
// and the column sums of each 256-row block into spart[block][c] (summed in a
// fixed order by mrhs_t_reduce_kernel): the matvec's scaling and the sums its
// rank-one shift needs, in right-hand-side-major form.
__global__ void __launch_bounds__(256) cg_prep_t_kernel(const double* __restrict__ P,
                                                       const double* __restrict__ d, int32_t V,
                                                       int32_t Vp, int32_t nr,
                                                       double* __restrict__ UT,
                                                       double* __restrict__ spart) {
    __shared__ double red[8][kMaxRhs];
    const int32_t j = blockIdx.x * 256 + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double dj = j < V ? d[j] : 0.0;
    double u[kMaxRhs];
#pragma unroll
    for (int c = 0; c < kMaxRhs; c++) u[c] = (c < nr && j < V) ? dj * P[(size_t)c * Vp + j] : 0.0;
    if (j < Vp) {
        double2* row = reinterpret_cast<double2*>(UT + (size_t)j * kMaxRhs);
#pragma unroll
        for (int c = 0; c < kMaxRhs; c += 2) row[c / 2] = make_double2(u[c], u[c + 1]);
    }
#pragma unroll
    for (int c = 0; c < kMaxRhs; c++) {
        double v = u[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < kMaxRhs) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += red[w][threadIdx.x];
        spart[(size_t)blockIdx.x * kMaxRhs + threadIdx.x] = t;
    }
}

// ---- multi-right-hand-side products on the FP64 tensor cores ----------------
//
// part[z][c][i] = sum_{j in range z of row block} M[i][j] X[c][j] for c < 16:
// mma.sync m8n8k4 (FP64), 64 rows per CTA (8 per warp), the row block's column
// range split into gridDim.y equal parts (split K, summed in a fixed order by
// mrhs_reduce_kernel). TRI = 0: all columns; 1: j < r0 + 64 (lower-triangular
// M); 2: j >= r0 (upper). The K order inside a 16-column group is permuted
// (MMA step s takes columns 4m + s, m = 0..3) so each lane's four consecutive
// columns of M feed four MMAs without shuffles; X is staged transposed in
// shared memory with rows padded to 17 doubles (conflict-free fragment loads).
constexpr int kMvRows = 64;
constexpr int kMvChunk = 256;
constexpr int kXs = kMaxRhs + 1;

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <int TRI, typename MT>
__global__ void __launch_bounds__(256)
mrhs_dmma_kernel(const MT* __restrict__ M, int32_t ldm, int32_t n,
                 const double* __restrict__ X, int32_t ldx, int32_t nr,
                 double* __restrict__ part) {
    __shared__ double xs[kMvChunk * kXs];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int32_t r0 = blockIdx.x * kMvRows;
    int32_t lo = 0, hi = n;
    if (TRI == 1) hi = min(n, r0 + kMvRows);
    if (TRI == 2) lo = r0;
    const int32_t per = (((hi - lo) + (int32_t)gridDim.y - 1) / (int32_t)gridDim.y + 15) / 16 * 16;
    const int32_t ks = lo + (int32_t)blockIdx.y * per;
    const int32_t ke = min(hi, ks + per);
    const int32_t row = r0 + warp * 8 + (lane >> 2);
    const bool rin = row < n;
    const MT* mrow = M + (size_t)(rin ? row : 0) * ldm;
    const int m4 = (lane & 3) * 4;
    const int gq = lane >> 2;
    const bool vec = sizeof(MT) == 8 ? (ldm & 1) == 0 : (ldm & 3) == 0;
    double c0a = 0.0, c0b = 0.0, c1a = 0.0, c1b = 0.0;
    for (int32_t kc = ks; kc < ke; kc += kMvChunk) {
        const int32_t kn = min(kMvChunk, ke - kc);
        __syncthreads();
        for (int e = threadIdx.x; e < kMaxRhs * kMvChunk; e += 256) {
            const int c = e / kMvChunk, jj = e % kMvChunk;
            xs[jj * kXs + c] = (c < nr && jj < kn) ? X[(size_t)c * ldx + kc + jj] : 0.0;
        }
        __syncthreads();
        // kUG 16-column groups per pass (the same bytes in flight per thread for
        // FP32 and FP64 M): their loads of M are all issued before the first MMA
        // (the MMA order, and so the sums, are those of one group at a time)
        constexpr int kUG = sizeof(MT) == 8 ? 4 : 8;
        for (int g0 = 0; g0 < kn; g0 += 16 * kUG) {
            MT a[kUG][4];
#pragma unroll
            for (int u = 0; u < kUG; u++) {
                const int32_t col = kc + g0 + 16 * u + m4;
                if (g0 + 16 * u < kn && rin && vec && col + 3 < ke) {
                    if constexpr (sizeof(MT) == 8) {
                        const double2 p0 = *reinterpret_cast<const double2*>(mrow + col);
                        const double2 p1 = *reinterpret_cast<const double2*>(mrow + col + 2);
                        a[u][0] = p0.x;
                        a[u][1] = p0.y;
                        a[u][2] = p1.x;
                        a[u][3] = p1.y;
                    } else {
                        const float4 p0 = *reinterpret_cast<const float4*>(mrow + col);
                        a[u][0] = p0.x;
                        a[u][1] = p0.y;
                        a[u][2] = p0.z;
                        a[u][3] = p0.w;
                    }
                } else {
#pragma unroll
                    for (int t = 0; t < 4; t++)
                        a[u][t] = (g0 + 16 * u < kn && rin && col + t < ke) ? mrow[col + t] : (MT)0;
                }
            }
#pragma unroll
            for (int u = 0; u < kUG; u++) {
                const int g = g0 + 16 * u;
                if (g >= kn) break;
#pragma unroll
                for (int s4 = 0; s4 < 4; s4++) {
                    const double* xr = xs + (g + m4 + s4) * kXs;
                    dmma884(c0a, c0b, (double)a[u][s4], xr[gq]);
                    dmma884(c1a, c1b, (double)a[u][s4], xr[8 + gq]);
                }
            }
        }
    }
    if (rin) {
        double* P = part + (size_t)blockIdx.y * kMaxRhs * ldx;
        const int cb = 2 * (lane & 3);
        P[(size_t)cb * ldx + row] = c0a;
        P[(size_t)(cb + 1) * ldx + row] = c0b;
        P[(size_t)(8 + cb) * ldx + row] = c1a;
        P[(size_t)(9 + cb) * ldx + row] = c1b;
    }
}

// ---- the CG's multi-RHS products, right-hand-side-major form ------------------
//
// Y = M X for up to 16 right-hand sides with the vectors held right-hand-side
// major (XT[j][c], 16 doubles per row j): every DMMA B fragment is then eight
// consecutive doubles of four rows (256 bytes in 8 sectors) read straight from
// L2, with no shared-memory staging and no block barriers. A warp owns 32 rows
// (four m8 fragments sharing each B fragment), a CTA 128 rows (one 128-row tile
// of the FP32 factor copies, whose lower or upper tiles alone are defined), and
// the columns split into chunks of kKChunk (grid.x) whose partial sums go to
// part[chunk][c][row] for a fixed-order reduction.
constexpr int kKChunk = 512;
constexpr int kTRows = 128;   // rows per CTA (four warps of 32)

// XT[j][c] = X[c][j] (j < n, c < nr), 0 elsewhere; nout rows of 16.
__global__ void rhs_major_kernel(const double* __restrict__ X, int32_t ldx, int32_t nr, int32_t n,
                                 int32_t nout, double* __restrict__ XT) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nout * kMaxRhs) return;
    const int32_t j = (int32_t)(t / kMaxRhs);
    const int c = (int)(t % kMaxRhs);
    XT[t] = (c < nr && j < n) ? X[(size_t)c * ldx + j] : 0.0;
}

// Columns [lo, hi) of chunk ch for the 128-row tile at rb0 (empty when lo >= hi).
__host__ __device__ __forceinline__ void mrhs_t_range(int tri, int32_t n, int32_t ch, int32_t rb0,
                                                      int32_t& lo, int32_t& hi) {
    lo = ch * kKChunk;
    hi = min(n, lo + kKChunk);
    if (tri == 1) hi = min(hi, rb0 + kTRows);  // lower tiles: k < tile end
    if (tri == 2) lo = max(lo, rb0);           // upper tiles: k >= tile start
}

// part[ch][c][row] = sum_{k in chunk ch} M[row][k] X[c][k], TRI as in mrhs_t_range.
// MT float: two 16-column groups per pass (A loads of both issued first).
template <int TRI, typename MT>
__global__ void __launch_bounds__(128, 4)
mrhs_t_kernel(const MT* __restrict__ M, int32_t ldm, int32_t n, const double* __restrict__ XT,
              double* __restrict__ part, int32_t ldp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int32_t ch = blockIdx.x, rb0 = blockIdx.y * kTRows;
    int32_t lo, hi;
    mrhs_t_range(TRI, n, ch, rb0, lo, hi);
    if (lo >= hi) return;  // the reduction skips this chunk for these rows
    const int q = lane & 3, gq = lane >> 2;
    constexpr int kF = 4;                       // m8 fragments per warp
    constexpr int kG = sizeof(MT) == 4 ? 2 : 1; // 16-column groups per pass
    const MT* mrow[kF];
    bool rin[kF];
#pragma unroll
    for (int f = 0; f < kF; f++) {
        const int32_t row = rb0 + warp * 32 + 8 * f + gq;
        rin[f] = row < n;
        mrow[f] = M + (size_t)(rin[f] ? row : 0) * ldm;
    }
    const bool vec = sizeof(MT) == 8 ? (ldm & 1) == 0 : (ldm & 3) == 0;
    double acc[kF][4];
#pragma unroll
    for (int f = 0; f < kF; f++) acc[f][0] = acc[f][1] = acc[f][2] = acc[f][3] = 0.0;
    for (int32_t g0 = lo; g0 < hi; g0 += 16 * kG) {
        MT a[kG][kF][4];
        double b0[kG][4], b1[kG][4];
#pragma unroll
        for (int u = 0; u < kG; u++) {
            const int32_t g = g0 + 16 * u;
            const int32_t col = g + 4 * q;
#pragma unroll
            for (int f = 0; f < kF; f++) {
                if (g < hi && rin[f] && vec && col + 3 < hi) {
                    if constexpr (sizeof(MT) == 8) {
                        const double2 p0 = *reinterpret_cast<const double2*>(mrow[f] + col);
                        const double2 p1 = *reinterpret_cast<const double2*>(mrow[f] + col + 2);
                        a[u][f][0] = p0.x;
                        a[u][f][1] = p0.y;
                        a[u][f][2] = p1.x;
                        a[u][f][3] = p1.y;
                    } else {
                        const float4 p0 = *reinterpret_cast<const float4*>(mrow[f] + col);
                        a[u][f][0] = p0.x;
                        a[u][f][1] = p0.y;
                        a[u][f][2] = p0.z;
                        a[u][f][3] = p0.w;
                    }
                } else {
#pragma unroll
                    for (int t = 0; t < 4; t++)
                        a[u][f][t] = (g < hi && rin[f] && col + t < hi) ? mrow[f][col + t] : (MT)0;
                }
            }
            // B: slot q <-> column g + 4 q + s4; rows past n are zero in XT
#pragma unroll
            for (int s4 = 0; s4 < 4; s4++) {
                const double* xr = XT + (size_t)(g < hi ? col + s4 : 0) * kMaxRhs;
                b0[u][s4] = g < hi ? xr[gq] : 0.0;
                b1[u][s4] = g < hi ? xr[8 + gq] : 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < kG; u++) {
#pragma unroll
            for (int s4 = 0; s4 < 4; s4++) {
#pragma unroll
                for (int f = 0; f < kF; f++) {
                    dmma884(acc[f][0], acc[f][1], (double)a[u][f][s4], b0[u][s4]);
                    dmma884(acc[f][2], acc[f][3], (double)a[u][f][s4], b1[u][s4]);
                }
            }
        }
    }
    const int cb = 2 * q;
    double* P = part + (size_t)ch * kMaxRhs * ldp;
#pragma unroll
    for (int f = 0; f < kF; f++) {
        if (!rin[f]) continue;
        const int32_t row = rb0 + warp * 32 + 8 * f + gq;
        P[(size_t)cb * ldp + row] = acc[f][0];
        P[(size_t)(cb + 1) * ldp + row] = acc[f][1];
        P[(size_t)(8 + cb) * ldp + row] = acc[f][2];
        P[(size_t)(9 + cb) * ldp + row] = acc[f][3];
    }
}

// Y[c][i] = scale_i (sum over the row's non-empty chunks of part[ch][c][i] +
// shift sum_z spart[z][c]) for i < n, c < nr (scale, spart optional); also
// YT[i][c] when YT is given (its columns c >= nr stay as they are: zero).
__global__ void mrhs_t_reduce_kernel(const double* __restrict__ part, int32_t ldp, int tri,
                                     int32_t n, int32_t nr, const double* __restrict__ scale,
                                     double shift, const double* __restrict__ spart, int32_t nz,
                                     double* __restrict__ Y, int32_t ldy, double* __restrict__ YT) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nr * n) return;
    const int c = (int)(t / n);
    const int32_t i = (int32_t)(t % n);
    const int32_t rb0 = i / kTRows * kTRows;
    const int32_t nch = (n + kKChunk - 1) / kKChunk;
    double acc = 0.0;
    for (int32_t ch = 0; ch < nch; ch++) {
        int32_t lo, hi;
        mrhs_t_range(tri, n, ch, rb0, lo, hi);
        if (lo < hi) acc += part[((size_t)ch * kMaxRhs + c) * ldp + i];
    }
    if (spart) {
        double sc = 0.0;
        for (int32_t z = 0; z < nz; z++) sc += spart[(size_t)z * kMaxRhs + c];
        acc += shift * sc;
    }
    if (scale) acc *= scale[i];
    if (Y) Y[(size_t)c * ldy + i] = acc;
    if (YT) YT[(size_t)i * kMaxRhs + c] = acc;
}

// Y[c][i] = scale_i (sum_z part[z][c][i] + shift s[c]) for i < n (scale, s optional).
__global__ void mrhs_reduce_kernel(const double* __restrict__ part, int32_t nsplit, int32_t n,
                                   int32_t ldx, int32_t nr, const double* __restrict__ scale,
                                   double shift, const double* __restrict__ s,
                                   double* __restrict__ Y) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nr * n) return;
    const int c = (int)(t / n);
    const int32_t i = (int32_t)(t % n);
    double acc = 0.0;
    for (int z = 0; z < nsplit; z++) acc += part[((size_t)z * kMaxRhs + c) * ldx + i];
    if (s) acc += shift * s[c];
    if (scale) acc *= scale[i];
    Y[(size_t)c * ldx + i] = acc;
}

// Plain FP32 copies of the inverse factor (hi + lo is exact in FP32): Zf = Z on
// lower tiles (diagonal tiles included, their upper parts are zero), Wf = W
// on upper tiles. The CG applies them with FP64 arithmetic.
// Restricted to the diagonal block [r0, r0 + n)^2 (the top level's
// off-diagonal blocks are written in FP32 directly).
__global__ void factor_to_f32_kernel(const float* __restrict__ zhi, const float* __restrict__ zlo,
                                     const float* __restrict__ whi, const float* __restrict__ wlo,
                                     int32_t Vp, int32_t r0, int32_t n, float* __restrict__ zf,
                                     float* __restrict__ wf) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * n) return;
    const int32_t i = r0 + (int32_t)(e / n), j = r0 + (int32_t)(e % n);
    const int64_t t = (int64_t)i * Vp + j;
    const int ti = i / kT, tj = j / kT;
    if (ti >= tj) zf[t] = zhi[t] + zlo[t];
    if (ti <= tj) wf[t] = whi[t] + wlo[t];
}

// Wf[c][base + r] = Zf[base + r][c] (r < 32 gridDim.y, c < 32 gridDim.x): the top
// level's W12 = Z21^T in FP32.
__global__ void transpose_f32_kernel(const float* __restrict__ zf, float* __restrict__ wf,
                                     int32_t ld, int32_t base) {
    __shared__ float t[32][33];
    const int32_t r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y)
        t[yy][threadIdx.x] = zf[(size_t)(base + r0 + yy) * ld + c0 + threadIdx.x];
    __syncthreads();
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y)
        wf[(size_t)(c0 + yy) * ld + base + r0 + threadIdx.x] = t[threadIdx.x][yy];
}

constexpr int kDotChunks = 32;

// part[c][z] = sum over chunk z of a[c][i] b[c][i] w_i^2 (w null -> 1).
__global__ void col_dots_part_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                     const double* __restrict__ w, int32_t Vp,
                                     double* __restrict__ part) {
    __shared__ double red[8];
    const int c = blockIdx.y, z = blockIdx.x;
    const int32_t len = (Vp + kDotChunks - 1) / kDotChunks;
    const int32_t i0 = z * len, i1 = min(Vp, i0 + len);
    double acc = 0.0;
    for (int32_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        double t = a[(size_t)c * Vp + i] * b[(size_t)c * Vp + i];
        if (w) t *= w[i] * w[i];
        acc += t;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int ww = 0; ww < (int)(blockDim.x >> 5); ww++) t += red[ww];
        part[c * kDotChunks + z] = t;
    }
}

// out[c] = sum_z part[c][z] in a fixed order.
__global__ void col_dots_final_kernel(const double* __restrict__ part, int32_t n,
                                      double* __restrict__ out) {
    const int c = threadIdx.x;
    if (c >= n) return;
    double t = 0.0;
    for (int z = 0; z < kDotChunks; z++) t += part[c * kDotChunks + z];
    out[c] = t;
}

// alpha_c = rz[c] / pq[c]; X += alpha P; R -= alpha Q
__global__ void cg_update_xr_kernel(double* __restrict__ X, double* __restrict__ R,
                                    const double* __restrict__ P, const double* __restrict__ Q,
                                    const double* __restrict__ rz, const double* __restrict__ pq,
                                    int32_t Vp, int32_t nr) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nr * Vp) return;
    const int c = (int)(t / Vp);
    const double al = pq[c] != 0.0 ? rz[c] / pq[c] : 0.0;
    X[t] += al * P[t];
    R[t] -= al * Q[t];
}

// P = Z + beta P with beta_c = rz_new[c] / rz_old[c]
__global__ void cg_update_p_kernel(double* __restrict__ P, const double* __restrict__ Zv,
                                   const double* __restrict__ rz_new,
                                   const double* __restrict__ rz_old, int32_t Vp, int32_t nr) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nr * Vp) return;
    const int c = (int)(t / Vp);
    const double be = rz_old[c] != 0.0 ? rz_new[c] / rz_old[c] : 0.0;
    P[t] = Zv[t] + be * P[t];
}

// R = D B (scaled right-hand sides, pad 0); X = 0
__global__ void cg_init_kernel(const double* __restrict__ B, const double* __restrict__ d,
                               int32_t V, int32_t Vp, int32_t nr, double* __restrict__ R,
                               double* __restrict__ X) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nr * Vp) return;
    const int c = (int)(t / Vp), i = (int)(t % Vp);
    R[t] = i < V ? d[i] * B[(size_t)c * V + i] : 0.0;
    X[t] = 0.0;
}

// B[c][i] = d_i X[c][i] for i < V (unscale)
__global__ void cg_final_kernel(const double* __restrict__ X, const double* __restrict__ d,
                                int32_t V, int32_t Vp, int32_t nr, double* __restrict__ B) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nr * V) return;
    const int c = (int)(t / V), i = (int)(t % V);
    B[t] = d[i] * X[(size_t)c * Vp + i];
}

inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

int32_t make_split(tpe_ctx* ctx, DevBuf& hi, DevBuf& lo, int32_t rows, int32_t cols,
                   tc::SplitMat& m) {
    const size_t bytes = sizeof(float) * (size_t)rows * cols;
    TPE_TRY(ensure(ctx, hi, bytes));
    TPE_TRY(ensure(ctx, lo, bytes));
    if (m.hi != hi.as<float>() || m.lo != lo.as<float>() || m.rows != rows || m.cols != cols ||
        m.ld != cols) {
        m.hi = hi.as<float>();
        m.lo = lo.as<float>();
        m.rows = rows;
        m.cols = cols;
        m.ld = cols;
        if (!tc::make_maps(m)) {
            m.hi = m.lo = nullptr;
            set_error(ctx, TPE_ERR_CUDA, "cuTensorMapEncodeTiled failed for the FP32 factor");
            return TPE_ERR_CUDA;
        }
    }
    return TPE_OK;
}

#define TC_TRY(expr) TPE_CUDA_TRY(expr)

}  // namespace

int32_t mixed_padded_size(int32_t V) { return V <= kT ? kT : (V + kT - 1) / kT * kT; }

namespace {
// Rows of the first part of an uneven split of n rows (n a multiple of 128, at
// least 256): the largest 128 * 2^k below n, so the first part's levels batch.
int32_t first_part(int32_t n) {
    int32_t h = kT;
    while (2 * h < n) h *= 2;
    return h;
}
bool pow2_blocks(int32_t n) { return n >= kT && ((n / kT) & (n / kT - 1)) == 0; }
}  // namespace

// FP32 factorization and inverse of the scaled A_rho (steps 1-3 above).
// *ok = false when the FP32 factorization broke down.
namespace {
// The diagonal transposes and the recursive-halving levels m = 128 .. hs/2 of
// Z = L^{-1} on the rows [base, base + hs) (hs a power of two times 128), on
// stream s. The level of width m pairs its blocks two by two: T^T = W11 L21^T
// (into T rows base/2 + ...), Z21 = -Z22 T, W12 = Z21^T. ctr: two zeroed tile
// counters per level.
int32_t inverse_half(tpe_ctx* ctx, int32_t base, int32_t hs, cudaStream_t s, int32_t* d_err,
                     int32_t* ctr) {
    MixedFactor& mf = ctx->mf;
    const int32_t Vp = mf.Vp;
    diag_transpose_kernel<<<dim3(kT / 32, kT / 32, hs / kT), dim3(32, 8), 0, s>>>(
        mf.Z.hi, mf.Z.lo, mf.W.hi, mf.W.lo, Vp, base / kT);
    TPE_CUDA_TRY(cudaGetLastError());
    int li = 0;
    for (int32_t m = kT; m < hs; m *= 2, li++) {
        const int32_t npairs = hs / (2 * m);
        const bool pers = m >= 1024 && s == ctx->stream;  // beside the factorization: one tile per CTA
        tc::GemmArgs t;  // T^T = W11 L21^T
        t.a_r0 = t.a_c0 = base;
        t.a_zr = t.a_zc = 2 * m;
        t.b_r0 = base + m;
        t.b_c0 = base;
        t.b_zr = t.b_zc = 2 * m;
        t.c_r0 = base / 2;
        t.c_zr = m;
        t.M = t.N = t.K = m;
        t.mode = tc::kAUpper;
        t.nbatch = npairs;
        TPE_CUDA_TRY(tc::gemm_nt(mf.W, mf.L, mf.T, t, d_err, s, pers ? ctx->num_sms : 0, ctr + 2 * li));
        tc::GemmArgs u;  // Z21 = -Z22 T
        u.a_r0 = u.a_c0 = base + m;
        u.a_zr = u.a_zc = 2 * m;
        u.b_r0 = base / 2;
        u.b_zr = m;
        u.c_r0 = base + m;
        u.c_c0 = base;
        u.c_zr = u.c_zc = 2 * m;
        u.M = u.N = u.K = m;
        u.mode = tc::kALower;
        u.alpha = -1.0f;
        u.nbatch = npairs;
        TPE_CUDA_TRY(tc::gemm_nt(mf.Z, mf.T, mf.Z, u, d_err, s, pers ? ctx->num_sms : 0,
                                 ctr + 2 * li + 1));
        transpose_block_kernel<<<dim3(m / 32, m / 32, npairs), dim3(32, 8), 0, s>>>(
            mf.Z.hi, mf.Z.lo, mf.W.hi, mf.W.lo, Vp, m, base);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    return TPE_OK;
}

// Launches inverse_half issues for hs rows.
int64_t inverse_half_launches(int32_t hs) {
    int64_t n = 1;
    for (int32_t m = kT; m < hs; m *= 2) n += 3;
    return n;
}

// Launches inverse_rec issues for n rows.
int64_t inverse_rec_launches(int32_t n) {
    if (pow2_blocks(n)) return inverse_half_launches(n);
    const int32_t a = first_part(n);
    return inverse_half_launches(a) + inverse_rec_launches(n - a) + 3;
}

// Z = L^{-1} (and W = Z^T) on the rows [base, base + n), n any multiple of 128,
// on stream s: a first part of 128 * 2^k rows by inverse_half, the rest
// recursively, then the cross block Z21 = -Z22 (L21 Z11) through
// T^T = W11 L21^T (T rows from base, free by then: every earlier use of T on
// this stream inside [base, base + n) has finished, and the first part of the
// top level, on another stream, uses only rows below base / 2).
int32_t inverse_rec(tpe_ctx* ctx, int32_t base, int32_t n, cudaStream_t s, int32_t* d_err,
                    int32_t* ctr) {
    if (pow2_blocks(n)) return inverse_half(ctx, base, n, s, d_err, ctr);
    MixedFactor& mf = ctx->mf;
    const int32_t a = first_part(n), b = n - a;
    // each inverse_half takes its own tile counters (two per level, at most 16)
    TPE_TRY(inverse_half(ctx, base, a, s, d_err, ctr));
    TPE_TRY(inverse_rec(ctx, base + a, b, s, d_err, ctr + 16));
    tc::GemmArgs t;  // T^T (a x b) = W11 L21^T, W11 upper
    t.a_r0 = t.a_c0 = base;
    t.b_r0 = base + a;
    t.b_c0 = base;
    t.c_r0 = base;
    t.M = a;
    t.N = b;
    t.K = a;
    t.mode = tc::kAUpper;
    TPE_CUDA_TRY(tc::gemm_nt(mf.W, mf.L, mf.T, t, d_err, s));
    tc::GemmArgs u;  // Z21 (b x a) = -Z22 T, Z22 lower
    u.a_r0 = u.a_c0 = base + a;
    u.b_r0 = base;
    u.c_r0 = base + a;
    u.c_c0 = base;
    u.M = b;
    u.N = a;
    u.K = b;
    u.mode = tc::kALower;
    u.alpha = -1.0f;
    TPE_CUDA_TRY(tc::gemm_nt(mf.Z, mf.T, mf.Z, u, d_err, s));
    transpose_rect_kernel<<<dim3(a / 32, b / 32, 1), dim3(32, 8), 0, s>>>(
        mf.Z.hi, mf.Z.lo, mf.W.hi, mf.W.lo, mf.Vp, base + a, base);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}
}  // namespace

int32_t mixed_factor(tpe_ctx* ctx, const double* d_A, int32_t V, double rho, bool* ok) {
    MixedFactor& mf = ctx->mf;
    *ok = false;
    mf.valid = false;
    const int32_t Vp = mixed_padded_size(V);
    const cudaStream_t st = ctx->stream;
    mf.V = V;
    mf.Vp = Vp;
    mf.rho = rho;
    const double shift = rho / V;
    TPE_TRY(ensure(ctx, ctx->mx_d, sizeof(double) * Vp));
    TPE_TRY(ensure(ctx, ctx->mx_dinv, sizeof(double) * Vp));
    TPE_TRY(ensure(ctx, ctx->mx_S, sizeof(float) * (size_t)Vp * Vp));
    TPE_TRY(make_split(ctx, ctx->mx_Lhi, ctx->mx_Llo, Vp, Vp, mf.L));
    TPE_TRY(make_split(ctx, ctx->mx_Zhi, ctx->mx_Zlo, Vp, Vp, mf.Z));
    TPE_TRY(make_split(ctx, ctx->mx_Whi, ctx->mx_Wlo, Vp, Vp, mf.W));
    // the top level's split: H1 = 128 * 2^k rows, the largest below Vp, then H2
    const int32_t H1 = Vp > kT ? first_part(Vp) : Vp, H2 = Vp - H1;
    if (Vp > kT) {
        // T: level scratch (inverse_half: rows base/2 ..) and the cross blocks of
        // uneven splits (rows base ..); T2: the top level's T^T (H1 x H2)
        TPE_TRY(make_split(ctx, ctx->mx_Thi, ctx->mx_Tlo, Vp, Vp / 2, mf.T));
        TPE_TRY(make_split(ctx, ctx->mx_T2hi, ctx->mx_T2lo, H1, H2, mf.T2));
    }
    TPE_TRY(ensure(ctx, ctx->mx_Zd, sizeof(float) * (size_t)Vp * Vp));
    TPE_TRY(ensure(ctx, ctx->mx_Wd, sizeof(float) * (size_t)Vp * Vp));
    tc::SplitMat& Zf = mf.Zf;  // the CG's FP32 copy of Z, as a plain GEMM output
    if (Zf.hi != ctx->mx_Zd.as<float>() || Zf.rows != Vp) {
        Zf.hi = ctx->mx_Zd.as<float>();
        Zf.lo = nullptr;
        Zf.rows = Zf.cols = Zf.ld = Vp;
        if (!tc::make_maps(Zf)) {
            Zf.hi = nullptr;
            set_error(ctx, TPE_ERR_CUDA, "cuTensorMapEncodeTiled failed for the FP32 inverse factor");
            return TPE_ERR_CUDA;
        }
    }
    TPE_TRY(ensure(ctx, ctx->status, sizeof(int32_t) * 4));
    int32_t* d_bad = ctx->status.as<int32_t>() + 2;
    TPE_CUDA_TRY(cudaMemsetAsync(d_bad, 0, 2 * sizeof(int32_t), st));
    // tile counters of the persistent GEMMs: one per panel's trailing update,
    // then two per inverse level
    // (nb for the trailing updates; 16 for the first part of the inverse, 16 per
    // recursion depth of the rest, one for the top level)
    const size_t nctr = (size_t)(Vp / kT) + 256;
    TPE_TRY(ensure(ctx, ctx->mx_ctr, sizeof(int32_t) * nctr));
    int32_t* d_ctr = ctx->mx_ctr.as<int32_t>();
    TPE_CUDA_TRY(cudaMemsetAsync(d_ctr, 0, sizeof(int32_t) * nctr, st));
    int32_t* d_err = d_bad + 1;
    double* d = ctx->mx_d.as<double>();
    float* S = ctx->mx_S.as<float>();
    tc::SplitMat& Sm = mf.S;  // the trailing matrix as a plain FP32 GEMM output
    if (Sm.hi != S || Sm.rows != Vp) {
        Sm.hi = S;
        Sm.lo = nullptr;
        Sm.rows = Sm.cols = Sm.ld = Vp;
        if (!tc::make_maps(Sm)) {
            Sm.hi = nullptr;
            set_error(ctx, TPE_ERR_CUDA, "cuTensorMapEncodeTiled failed for the FP32 trailing matrix");
            return TPE_ERR_CUDA;
        }
    }
    const int nb = Vp / kT;
    const size_t potrf_smem = sizeof(float) * kSmem3Floats;
    TPE_CUDA_TRY(cudaFuncSetAttribute(potrf128_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)potrf_smem));
    // Critical path on the main stream, per block j: potrf, then one CTA that
    // solves the panel's first row tile (L_{j+1,j}) from the FP32 matrix and
    // updates the next diagonal block by it; then potrf j+1. Beside it, on
    // stream5 (high priority), the split copy and solve of the rest of the panel,
    // the update of the rest of block column j+1 and of diagonal block j+2 (which
    // the next step's one-CTA kernel waits for), and on stream2 (low priority)
    // the rest of the trailing update, which only stream5's next column update
    // waits for (look-ahead of one block).
    // Every tile receives its updates in the order of the one-stream schedule
    // (rests of earlier panels first), so the results do not depend on it.
    while ((int32_t)ctx->fac_events.size() < 4 * nb + 3) {
        cudaEvent_t e;
        TPE_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->fac_events.push_back(e);
    }
    cudaEvent_t* ev_t1 = ctx->fac_events.data();          // first row tile of panel j solved
    cudaEvent_t* ev_tr = ctx->fac_events.data() + nb;     // whole panel j solved
    cudaEvent_t* ev_s = ctx->fac_events.data() + 2 * nb;  // block column j+1 final below block j+1
    cudaEvent_t* ev_r = ctx->fac_events.data() + 3 * nb;  // trailing update of panel j done
    cudaEvent_t ev_mid = ctx->fac_events[4 * nb];         // panels 0 .. nb/2-1 done
    cudaEvent_t ev_half = ctx->fac_events[4 * nb + 1];    // first half of the inverse done
    cudaEvent_t ev_side = ctx->fac_events[4 * nb + 2];    // side streams drained
    const cudaStream_t st2 = ctx->stream2, st5 = ctx->stream5;
    // The trailing updates run persistent (one CTA per SM walking its tiles) on
    // the SMs left by the concurrent gradient, minus a few kept free so that the
    // chain's launches never wait for a whole update.
    const int32_t rest_ctas = std::max(16, ctx->num_sms - ctx->grad_sms - ctx->free_sms);
    {
        const int64_t nrest = nb > 2 ? nb - 2 : 0;
        KernelScope ks(ctx, TPE_KGROUP_CHOLESKY, 2 + (int64_t)nb + (int64_t)(nb - 1) + 4 * nrest + (nrest > 0 ? nrest - 1 : 0) +
                                                     (nb > 1 ? 1 + inverse_half_launches(H1) : 0));
        jacobi_kernel<<<nblk(Vp, 256), 256, 0, st>>>(d_A, V, Vp, shift, d, ctx->mx_dinv.as<double>());
        scale_to_f32_kernel<<<dim3((unsigned)((Vp + 1023) / 1024), (unsigned)std::min(Vp, 65535)), 256, 0,
                              st>>>(d_A, V, Vp, shift, d, S);
        TPE_CUDA_TRY(cudaGetLastError());
        for (int j = 0; j < nb; j++) {
            const int32_t j0 = j * kT;
            potrf128_kernel<<<1, 256, potrf_smem, st>>>(S, Vp, j0, mf.Z.hi, mf.Z.lo, d_bad);
            TPE_CUDA_TRY(cudaGetLastError());
            if (j + 1 == nb) break;
            const int32_t rows = Vp - j0 - kT;
            const bool more = rows > kT;  // rows below block j+1 (then also a trailing update)
            // L_{j+1,j} = S_{j+1,j} Z_jj^T and the next diagonal block's update by it,
            // one CTA. Block column j below its diagonal and diagonal block j+1 are
            // final once the previous step's stream5 work has run: the column
            // update and the diagonal tile of the trailing update, both after the
            // trailing update before that. The previous trailing update itself
            // (the rest) is not waited for: it has a whole step to finish.
            if (j > 0) TPE_CUDA_TRY(cudaStreamWaitEvent(st, ev_s[j - 1], 0));
            TC_TRY(tc::chain_tile(mf.L, mf.Z, Sm, j0, d_err, st));
            TPE_CUDA_TRY(cudaEventRecord(ev_t1[j], st));
            tc::GemmArgs t;  // the panel below block j+1: L = S Z_jj^T (in place in L)
            t.a_c0 = j0;
            t.b_r0 = j0;
            t.b_c0 = j0;
            t.c_c0 = j0;
            t.N = kT;
            t.K = kT;
            if (more) {
                // the rest of the panel (rows j0+256 ..): its split copy follows the
                // previous column update on this stream, its solve needs Z_jj. Both
                // start after the one-CTA kernel, so that its CTA never waits for
                // an SM behind theirs.
                TPE_CUDA_TRY(cudaStreamWaitEvent(st5, ev_t1[j], 0));
                split_copy_kernel<<<nblk((int64_t)(rows - kT) * kT, 256), 256, 0, st5>>>(
                    S, Vp, j0 + 2 * kT, j0, rows - kT, mf.L.hi, mf.L.lo);
                TPE_CUDA_TRY(cudaGetLastError());
                tc::GemmArgs t2 = t;
                t2.a_r0 = t2.c_r0 = j0 + 2 * kT;
                t2.M = rows - kT;
                TC_TRY(tc::gemm_nt(mf.L, mf.Z, mf.L, t2, d_err, st5));
                TPE_CUDA_TRY(cudaEventRecord(ev_tr[j], st5));
                // trailing update (low priority): S[j0+256.., j0+256..] -= L21 L21^T,
                // lower tiles but the first (diagonal block j+2: stream5, below)
                TPE_CUDA_TRY(cudaStreamWaitEvent(st2, ev_tr[j], 0));
                tc::GemmArgs u;
                u.a_r0 = u.b_r0 = j0 + 2 * kT;
                u.a_c0 = u.b_c0 = j0;
                u.c_r0 = u.c_c0 = j0 + 2 * kT;
                u.M = u.N = rows - kT;
                u.K = kT;
                u.mode = tc::kLowerTiles;
                u.alpha = -1.0f;
                u.beta = 1.0f;
                u.tile_skip = 1;
                // block column j+1 below block j+1: after the previous trailing
                // update, with L_{j+1,j} from the main stream
                if (j > 0) TPE_CUDA_TRY(cudaStreamWaitEvent(st5, ev_r[j - 1], 0));
                tc::GemmArgs v;  // S[j0+256.., block j+1] -= L_{rows,j} L_{j+1,j}^T
                v.a_r0 = j0 + 2 * kT;
                v.a_c0 = j0;
                v.b_r0 = j0 + kT;
                v.b_c0 = j0;
                v.c_r0 = j0 + 2 * kT;
                v.c_c0 = j0 + kT;
                v.M = rows - kT;
                v.N = kT;
                v.K = kT;
                v.alpha = -1.0f;
                v.beta = 1.0f;
                TC_TRY(tc::gemm_nt(mf.L, mf.L, Sm, v, d_err, st5));
                tc::GemmArgs dg = u;  // diagonal block j+2 -= L_{j+2,j} L_{j+2,j}^T
                dg.M = dg.N = kT;
                dg.mode = 0;
                dg.tile_skip = 0;
                TC_TRY(tc::gemm_nt(mf.L, mf.L, Sm, dg, d_err, st5));
                TPE_CUDA_TRY(cudaEventRecord(ev_s[j], st5));
                if (rows - kT > kT)
                    TC_TRY(tc::gemm_nt(mf.L, mf.L, Sm, u, d_err, st2, rest_ctas, d_ctr + j));
                TPE_CUDA_TRY(cudaEventRecord(ev_r[j], st2));
            }
            if (nb > 1 && j == H1 / kT - 1) {
                // panels 0 .. H1/128-1 are final: the first part of the inverse and
                // the top level's T^T = W11 L21^T go to stream4 (low priority)
                TPE_CUDA_TRY(cudaEventRecord(ev_mid, more ? st5 : st));
                TPE_CUDA_TRY(cudaStreamWaitEvent(ctx->stream4, ev_mid, 0));
                TPE_TRY(inverse_half(ctx, 0, H1, ctx->stream4, d_err, d_ctr + Vp / kT));
                tc::GemmArgs t2;  // T^T (H1 x H2) = W11 L21^T
                t2.b_r0 = H1;
                t2.M = t2.K = H1;
                t2.N = H2;
                t2.mode = tc::kAUpper;
                TC_TRY(tc::gemm_nt(mf.W, mf.L, mf.T2, t2, d_err, ctx->stream4));
                TPE_CUDA_TRY(cudaEventRecord(ev_half, ctx->stream4));
            }
        }
        // the whole factor (every panel solved, every update applied) before the inverse
        TPE_CUDA_TRY(cudaEventRecord(ev_side, st5));
        TPE_CUDA_TRY(cudaStreamWaitEvent(st, ev_side, 0));
        TPE_CUDA_TRY(cudaEventRecord(ev_side, st2));
        TPE_CUDA_TRY(cudaStreamWaitEvent(st, ev_side, 0));
    }
    {
        // Z = L^{-1} (W = Z^T alongside) by the recursive block formula. The
        // first part (rows < H1: its diagonal transposes, its levels and the top
        // level's T^T = W11 L21^T) depends only on panels 0 .. H1/128-1, so it
        // already ran on stream4 beside the rest of the factorization; the rest
        // (rows H1 ..) and the top level's Z21 = -Z22 T follow here.
        if (Vp == kT) {
            KernelScope ks(ctx, TPE_KGROUP_TRSV, 1);
            diag_transpose_kernel<<<dim3(kT / 32, kT / 32, 1), dim3(32, 8), 0, st>>>(
                mf.Z.hi, mf.Z.lo, mf.W.hi, mf.W.lo, Vp, 0);
            TPE_CUDA_TRY(cudaGetLastError());
        } else {
            KernelScope ks(ctx, TPE_KGROUP_TRSV, inverse_rec_launches(H2) + 2);
            TPE_TRY(inverse_rec(ctx, H1, H2, st, d_err, d_ctr + Vp / kT + 32));
            TPE_CUDA_TRY(cudaStreamWaitEvent(st, ev_half, 0));
            tc::GemmArgs u;  // top level: Z21 (H2 x H1) = -Z22 T
            u.a_r0 = u.a_c0 = H1;
            u.c_r0 = H1;
            u.M = u.K = H2;
            u.N = H1;
            u.mode = tc::kALower;
            u.alpha = -1.0f;
            // no later product reads it split: written straight into the CG's FP32 copy
            TC_TRY(tc::gemm_nt(mf.Z, mf.T2, mf.Zf, u, d_err, st, H1 >= 1024 ? ctx->num_sms : 0,
                               d_ctr + Vp / kT + 255));
            transpose_f32_kernel<<<dim3(H1 / 32, H2 / 32, 1), dim3(32, 8), 0, st>>>(
                ctx->mx_Zd.as<float>(), ctx->mx_Wd.as<float>(), Vp, H1);
            TPE_CUDA_TRY(cudaGetLastError());
        }
    }
    {
        // the diagonal parts (the whole matrix when it is one block)
        KernelScope ks(ctx, TPE_KGROUP_TRSV, Vp > kT ? 2 : 1);
        if (Vp > kT) {
            factor_to_f32_kernel<<<nblk((int64_t)H1 * H1, 256), 256, 0, st>>>(
                mf.Z.hi, mf.Z.lo, mf.W.hi, mf.W.lo, Vp, 0, H1, ctx->mx_Zd.as<float>(),
                ctx->mx_Wd.as<float>());
            factor_to_f32_kernel<<<nblk((int64_t)H2 * H2, 256), 256, 0, st>>>(
                mf.Z.hi, mf.Z.lo, mf.W.hi, mf.W.lo, Vp, H1, H2, ctx->mx_Zd.as<float>(),
                ctx->mx_Wd.as<float>());
        } else {
            factor_to_f32_kernel<<<nblk((int64_t)Vp * Vp, 256), 256, 0, st>>>(
                mf.Z.hi, mf.Z.lo, mf.W.hi, mf.W.lo, Vp, 0, Vp, ctx->mx_Zd.as<float>(),
                ctx->mx_Wd.as<float>());
        }
        TPE_CUDA_TRY(cudaGetLastError());
    }
    int32_t flags[2] = {0, 0};
    TPE_CUDA_TRY(cudaMemcpyAsync(flags, d_bad, sizeof(flags), cudaMemcpyDeviceToHost, st));
    TPE_CUDA_TRY(cudaStreamSynchronize(st));
    if (flags[1]) {
        set_error(ctx, TPE_ERR_DEVICE_TIMEOUT, "tensor-core pipeline wait timed out");
        return TPE_ERR_DEVICE_TIMEOUT;
    }
    *ok = flags[0] == 0;
    mf.valid = *ok;
    return TPE_OK;
}

int32_t mrhs_fp64(tpe_ctx* ctx, const double* M, int32_t n, const double* X, int32_t ldx,
                  int32_t nr, double* Y) {
    if (nr <= 0 || n <= 0) return TPE_OK;
    if (nr > kMaxRhs || ldx < n) {
        set_error(ctx, TPE_ERR_TOO_LARGE, "mrhs_fp64: at most 16 right-hand sides, ldx >= n");
        return TPE_ERR_TOO_LARGE;
    }
    constexpr int kSplit = 8;
    TPE_TRY(ensure(ctx, ctx->mx_part, sizeof(double) * (size_t)kSplit * kMaxRhs * ldx));
    double* part = ctx->mx_part.as<double>();
    KernelScope ks(ctx, TPE_KGROUP_OTHER, 2);
    mrhs_dmma_kernel<0, double><<<dim3((unsigned)((n + kMvRows - 1) / kMvRows), kSplit), 256, 0,
                                  ctx->stream>>>(M, n, n, X, ldx, nr, part);
    mrhs_reduce_kernel<<<nblk((int64_t)nr * n, 256), 256, 0, ctx->stream>>>(
        part, kSplit, n, ldx, nr, nullptr, 0.0, nullptr, Y);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

// Solves A_rho X = B for nr right-hand sides (B, X: [nr][V] FP64 device; may
// alias) by CG on the scaled system preconditioned with the FP32 inverse factor.
// *iters = iterations of the last pass; *converged = every column reached
// ||B - A_rho X|| <= tol ||B||.
constexpr int kPredictFrom = 30;  // CG iterations always allowed before a predicted stop
constexpr int kRateSpan = 10;     // iterations the residual rate is measured over

int32_t mixed_solve(tpe_ctx* ctx, const double* d_A, const double* d_B, double* d_X, int32_t nr,
                    int32_t maxit, double tol, int32_t* iters, bool* converged) {
    const MixedFactor& mf = ctx->mf;
    const int32_t V = mf.V, Vp = mf.Vp;
    const double shift = mf.rho / V;
    const cudaStream_t st = ctx->stream;
    *converged = true;
    *iters = 0;
    const size_t vec = (size_t)kMaxRhs * Vp;
    const int32_t nz = (Vp + 255) / 256;  // 256-row blocks of the matvec's column sums
    TPE_TRY(ensure(ctx, ctx->mx_vec, sizeof(double) * (8 * vec + 8 * kMaxRhs + kMaxRhs * kDotChunks +
                                                       (size_t)nz * kMaxRhs)));
    // split-K partial sums of the right-hand-side-major products: one slot per
    // column chunk
    const int32_t nch = (Vp + kKChunk - 1) / kKChunk;
    TPE_TRY(ensure(ctx, ctx->mx_part, sizeof(double) * (size_t)nch * kMaxRhs * Vp));
    double* X = ctx->mx_vec.as<double>();
    double* R = X + vec;
    double* P = R + vec;
    double* Q = P + vec;
    double* Zv = Q + vec;
    double* U = Zv + vec;
    double* XT = U + vec;   // a product's input, right-hand-side major (Vp x 16)
    double* UT = XT + vec;  // the preconditioner's middle vector, the same way
    double* sc = UT + vec;  // 8 arrays of kMaxRhs scalars
    double* pq = sc + kMaxRhs;
    double* rz[2] = {sc + 2 * kMaxRhs, sc + 3 * kMaxRhs};
    double* res2 = sc + 4 * kMaxRhs;
    double* bn2 = sc + 5 * kMaxRhs;
    double* dpart = sc + 8 * kMaxRhs;  // kMaxRhs x kDotChunks partial dot products
    double* spart = dpart + kMaxRhs * kDotChunks;  // nz x kMaxRhs column sums of the matvec
    double* part = ctx->mx_part.as<double>();
    const double* d = ctx->mx_d.as<double>();
    const float* Zf = ctx->mx_Zd.as<float>();
    const float* Wf = ctx->mx_Wd.as<float>();
    std::vector<double> hres(kMaxRhs), hbn(kMaxRhs);
    // squared residual norms of the last kRateSpan + 1 iterations (a ring), for
    // the predicted stop below
    std::vector<double> hist((size_t)(kRateSpan + 1) * kMaxRhs);
    int32_t max_iters = 0;
    const dim3 grid_p((unsigned)nch, (unsigned)(Vp / kTRows));
    const dim3 grid_a((unsigned)((V + kKChunk - 1) / kKChunk), (unsigned)((V + kTRows - 1) / kTRows));
    for (int32_t c0 = 0; c0 < nr; c0 += kMaxRhs) {
        const int32_t n = nr - c0 < kMaxRhs ? nr - c0 : kMaxRhs;
        const int64_t tot = (int64_t)n * Vp;
        // UT's columns n .. 15 stay zero through the pass (the reductions write
        // columns < n only)
        TPE_CUDA_TRY(cudaMemsetAsync(UT, 0, sizeof(double) * vec, st));
        // out = W (Z in): the preconditioner (L L^T)^{-1} of the scaled system
        auto precond = [&](const double* in, double* out) -> int32_t {
            KernelScope ks(ctx, TPE_KGROUP_TRSV, 5);
            rhs_major_kernel<<<nblk(vec, 256), 256, 0, st>>>(in, Vp, n, Vp, Vp, XT);
            mrhs_t_kernel<1, float><<<grid_p, 128, 0, st>>>(Zf, Vp, Vp, XT, part, Vp);
            mrhs_t_reduce_kernel<<<nblk(tot, 256), 256, 0, st>>>(part, Vp, 1, Vp, n, nullptr, 0.0,
                                                                  nullptr, 0, nullptr, Vp, UT);
            mrhs_t_kernel<2, float><<<grid_p, 128, 0, st>>>(Wf, Vp, Vp, UT, part, Vp);
            mrhs_t_reduce_kernel<<<nblk(tot, 256), 256, 0, st>>>(part, Vp, 2, Vp, n, nullptr, 0.0,
                                                                  nullptr, 0, out, Vp, nullptr);
            TPE_CUDA_TRY(cudaGetLastError());
            return TPE_OK;
        };
        // out = S in = D (A + shift 1 1^T) D in, rows < V
        auto matvec = [&](const double* in, double* out) -> int32_t {
            KernelScope ks(ctx, TPE_KGROUP_OTHER, 3);
            cg_prep_t_kernel<<<nz, 256, 0, st>>>(in, d, V, Vp, n, XT, spart);
            mrhs_t_kernel<0, double><<<grid_a, 128, 0, st>>>(d_A, V, V, XT, part, Vp);
            mrhs_t_reduce_kernel<<<nblk((int64_t)n * V, 256), 256, 0, st>>>(part, Vp, 0, V, n, d, shift,
                                                                             spart, nz, out, Vp, nullptr);
            TPE_CUDA_TRY(cudaGetLastError());
            return TPE_OK;
        };
        auto dots = [&](const double* a, const double* b, const double* w, double* out) -> int32_t {
            KernelScope ks(ctx, TPE_KGROUP_OTHER, 2);
            col_dots_part_kernel<<<dim3(kDotChunks, n), 256, 0, st>>>(a, b, w, Vp, dpart);
            col_dots_final_kernel<<<1, 32, 0, st>>>(dpart, n, out);
            TPE_CUDA_TRY(cudaGetLastError());
            return TPE_OK;
        };
        {
            KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
            cg_init_kernel<<<nblk(tot, 256), 256, 0, st>>>(d_B + (size_t)c0 * V, d, V, Vp, n, R, X);
            TPE_CUDA_TRY(cudaGetLastError());
        }
        // the matrix-vector kernel writes rows < V only: the pad of Q stays 0
        TPE_CUDA_TRY(cudaMemsetAsync(Q, 0, sizeof(double) * tot, st));
        // residual norms of the unscaled system: ||D^{-1} R||
        const double* di = ctx->mx_dinv.as<double>();
        TPE_TRY(dots(R, R, di, bn2));
        TPE_CUDA_TRY(cudaMemcpyAsync(hbn.data(), bn2, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        TPE_TRY(precond(R, Zv));
        TPE_CUDA_TRY(cudaMemcpyAsync(P, Zv, sizeof(double) * tot, cudaMemcpyDeviceToDevice, st));
        TPE_TRY(dots(R, Zv, nullptr, rz[0]));
        int it = 0;
        bool done = false;
        for (it = 1; it <= maxit; it++) {
            TPE_TRY(matvec(P, Q));
            TPE_TRY(dots(P, Q, nullptr, pq));
            {
                KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
                cg_update_xr_kernel<<<nblk(tot, 256), 256, 0, st>>>(X, R, P, Q, rz[(it - 1) & 1], pq, Vp, n);
                TPE_CUDA_TRY(cudaGetLastError());
            }
            TPE_TRY(dots(R, R, di, res2));
            TPE_TRY(download_on(ctx, st, hres.data(), res2, sizeof(double) * n));
            done = true;
            for (int c = 0; c < n; c++)
                if (!(hres[c] <= tol * tol * hbn[c])) done = false;
            if (done) break;
            // From iteration kPredictFrom on, stop (not converged: the caller falls
            // back to the FP64 factorization) once a column's residual rate over
            // the last kRateSpan iterations predicts it reaches tol only after maxit.
            std::copy(hres.begin(), hres.begin() + n,
                      hist.begin() + (size_t)(it % (kRateSpan + 1)) * kMaxRhs);
            if (it >= kPredictFrom && it >= kRateSpan) {
                bool hopeless = false;
                for (int c = 0; c < n && !hopeless; c++) {
                    const double target = tol * tol * hbn[c];
                    if (hres[c] <= target) continue;
                    const double now = hres[c],
                                 old = hist[(size_t)((it - kRateSpan) % (kRateSpan + 1)) * kMaxRhs + c];
                    if (!(now < old) || !(now > 0.0)) {
                        hopeless = true;
                    } else {
                        const double rate = log(now / old) / kRateSpan;  // < 0
                        hopeless = it + log(target / now) / rate > maxit;
                    }
                }
                if (hopeless) break;
            }
            TPE_TRY(precond(R, Zv));
            TPE_TRY(dots(R, Zv, nullptr, rz[it & 1]));
            {
                KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
                cg_update_p_kernel<<<nblk(tot, 256), 256, 0, st>>>(P, Zv, rz[it & 1], rz[(it - 1) & 1], Vp, n);
                TPE_CUDA_TRY(cudaGetLastError());
            }
        }
        if (!done) *converged = false;
        if (it > max_iters) max_iters = it > maxit ? maxit : it;
        {
            KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
            cg_final_kernel<<<nblk((int64_t)n * V, 256), 256, 0, st>>>(X, d, V, Vp, n, d_X + (size_t)c0 * V);
            TPE_CUDA_TRY(cudaGetLastError());
        }
    }
    *iters = max_iters;
    return TPE_OK;
}

}  // namespace tpe
