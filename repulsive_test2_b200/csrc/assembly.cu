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


// (|d|+eps)^(-(2 sigma + 1)) from dn = |d|+eps and its reciprocal idn;
// MODE 1: alpha = 3, beta = 6 -> exponent 7/3.
template <int MODE>
__device__ __forceinline__ double inv_dist_pow(double dn, double idn, double distExp) {
    if (MODE == 1) return rcbrt(dn) * (idn * idn);
    return 1.0 / pow(dn, distExp);
}

// |d| and 1/(|d| + eps) for x = |d|^2 from one reciprocal square root r:
// 1/(|d| + eps) = r / (1 + t), t = eps r, summed as r (1 - t + t^2) when
// t < 2^-20 (the first term left out is below 2^-60 relative); otherwise the
// square root and the division themselves.
__device__ __forceinline__ void dist_inv(double x, double eps, double& s, double& inv_se) {
    const double r = rsqrt(x);
    const double t = eps * r;
    if (t < 9.5367431640625e-07) {
        s = x * r;
        inv_se = fma(-r, t * (1.0 - t), r);
    } else {
        s = sqrt(x);
        inv_se = 1.0 / (s + eps);
    }
}

// sqrt(x) for x >= 0 from a reciprocal square root (0 at x = 0).
__device__ __forceinline__ double sqrt_r(double x) { return x > 0.0 ? x * rsqrt(x) : sqrt(x); }

constexpr int kT = 32;  // pair tile: 32 edges I x 32 edges J

struct EdgeRec {
    double4 p1;  // endpoint 1, l^eps
    double4 p2;  // endpoint 2
    double4 T;   // unit tangent (0 below 1e-14), raw length
    int2 ij;
};

__device__ __forceinline__ void load_edge(const double4* __restrict__ ea,
                                          const double4* __restrict__ eb,
                                          const int2* __restrict__ edges, int32_t E, int32_t I,
                                          EdgeRec& r) {
    if (I >= E) {
        r.p1 = make_double4(0, 0, 0, 1);
        r.p2 = make_double4(0, 0, 0, 1);
        r.T = make_double4(0, 0, 0, 0);
        r.ij = make_int2(-1, -1);
        return;
    }
    r.p1 = ea[I];
    r.p2 = eb[I];
    r.ij = edges[I];
    const double ex = r.p2.x - r.p1.x, ey = r.p2.y - r.p1.y, ez = r.p2.z - r.p1.z;
    const double len = sqrt(ex * ex + ey * ey + ez * ez);
    if (len < 1e-14) {
        r.T = make_double4(0, 0, 0, len);
    } else {
        const double inv = 1.0 / len;
        r.T = make_double4(ex * inv, ey * inv, ez * inv, len);
    }
}

// Symmetric pair weights of one unordered pair: (w_IJ + w_JI, q_IJ + q_JI).
template <int MODE>
__device__ __forceinline__ double2 pair_weight(const EdgeRec& a, const EdgeRec& b, double distExp,
                                               double eps) {
    double sumDist = 0.0, sumLowIJ = 0.0, sumLowJI = 0.0;
#pragma unroll
    for (int s = 0; s < 4; s++) {
        const int ai = s >> 1, bj = s & 1;
        const double dx = (ai ? a.p2.x : a.p1.x) - (bj ? b.p2.x : b.p1.x);
        const double dy = (ai ? a.p2.y : a.p1.y) - (bj ? b.p2.y : b.p1.y);
        const double dz = (ai ? a.p2.z : a.p1.z) - (bj ? b.p2.z : b.p1.z);
        double dlen, idn;
        dist_inv(dx * dx + dy * dy + dz * dz, eps, dlen, idn);
        const double dn = dlen + eps;
        const double kd = inv_dist_pow<MODE>(dn, idn, distExp);
        sumDist += kd;
        const double idn2 = idn * idn;
        const double kq = kd * (idn2 * idn2);
        double cx = a.T.y * dz - a.T.z * dy, cy = a.T.z * dx - a.T.x * dz,
               cz = a.T.x * dy - a.T.y * dx;
        double cn = sqrt_r(cx * cx + cy * cy + cz * cz) + eps;
        sumLowIJ += cn * cn * kq;
        cx = b.T.y * dz - b.T.z * dy;
        cy = b.T.z * dx - b.T.x * dz;
        cz = b.T.x * dy - b.T.y * dx;
        cn = sqrt_r(cx * cx + cy * cy + cz * cz) + eps;
        sumLowJI += cn * cn * kq;
    }
    const double ll = a.p1.w * b.p1.w;
    return make_double2(0.5 * ll * sumDist, 0.0625 * ll * (sumLowIJ + sumLowJI));
}

// One block per upper-triangular 32x32 tile (it <= jt) of the E x E pair
// matrix; 256 threads = 32 J lanes x 8 row groups of 4 I rows. Writes
// M[I][J] = (-(w_IJ+w_JI) T_I.T_J / (l_I l_J), -(q_IJ+q_JI)) coalesced along J,
// and its mirror M[J][I] through a shared-memory transpose. Row sums of the
// weights go to rowpart[slot][row] (slot = the other tile index), each slot
// written once, for the diagonal pass.
template <int MODE>
__global__ void __launch_bounds__(256)
pair_weights_kernel(const double4* __restrict__ ea, const double4* __restrict__ eb,
                    const int2* __restrict__ edges, int32_t E, double distExp, double eps,
                    double2* __restrict__ M, double2* __restrict__ rowpart) {
    __shared__ EdgeRec sI[kT], sJ[kT];
    __shared__ double2 tile[kT][kT + 1];
    __shared__ double2 colred[8][kT];
    const int64_t t = blockIdx.x;
    int32_t it = (int32_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((int64_t)it * (it + 1) / 2 > t) it--;
    while ((int64_t)(it + 1) * (it + 2) / 2 <= t) it++;
    const int32_t jt_rel = (int32_t)(t - (int64_t)it * (it + 1) / 2);
    // map the lower-triangle enumeration (it >= jt_rel) to the upper tile (row jt_rel, col it)
    const int32_t ti = jt_rel, tj = it;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    if (threadIdx.x < kT) load_edge(ea, eb, edges, E, ti * kT + threadIdx.x, sI[threadIdx.x]);
    else if (threadIdx.x < 2 * kT)
        load_edge(ea, eb, edges, E, tj * kT + threadIdx.x - kT, sJ[threadIdx.x - kT]);
    __syncthreads();
    const int32_t J = tj * kT + tx;
    const EdgeRec& b = sJ[tx];
    double2 colsum = make_double2(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int li = ty + 8 * r;
        const int32_t I = ti * kT + li;
        const EdgeRec& a = sI[li];
        double2 out = make_double2(0.0, 0.0);
        double2 w = make_double2(0.0, 0.0);
        const bool ok = I < E && J < E && I != J && a.ij.x != b.ij.x && a.ij.x != b.ij.y &&
                        a.ij.y != b.ij.x && a.ij.y != b.ij.y;
        if (ok) {
            w = pair_weight<MODE>(a, b, distExp, eps);
            const double dotT = a.T.x * b.T.x + a.T.y * b.T.y + a.T.z * b.T.z;
            out = make_double2(-w.x * dotT / (a.p1.w * b.p1.w), -w.y);
        }
        if (I < E && J < E) M[(int64_t)I * E + J] = out;
        tile[li][tx] = out;
        colsum.x += w.x;
        colsum.y += w.y;
        // row sum over this tile's J (warp = one row group)
        double2 rs = w;
        for (int o = 16; o > 0; o >>= 1) {
            rs.x += __shfl_down_sync(0xffffffffu, rs.x, o);
            rs.y += __shfl_down_sync(0xffffffffu, rs.y, o);
        }
        if (tx == 0 && I < E) rowpart[(int64_t)tj * E + I] = rs;
    }
    if (ti == tj) return;  // diagonal tile: every (I, J) was computed directly
    colred[ty][tx] = colsum;
    __syncthreads();
    // mirror: M[J][I] for I in tile ti, written along I
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

// Diagonal of the pair matrix: (d_I, d0_I) from the per-tile row sums.
__global__ void pair_diag_kernel(const double4* __restrict__ ea, int32_t E, int32_t nt,
                                 const double2* __restrict__ rowpart, double2* __restrict__ M) {
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= E) return;
    double sx = 0.0, sy = 0.0;
    for (int32_t s = 0; s < nt; s++) {
        const double2 p = rowpart[(int64_t)s * E + I];
        sx += p.x;
        sy += p.y;
    }
    const double ell = ea[I].w;
    M[(int64_t)I * E + I] = make_double2(sx / (ell * ell), sy);
}

// A[v][u] = sum_{(I,a) in inc(v)} sum_{(J,b) in inc(u)} (s_a s_b Mb'[I][J] + M0'[I][J]),
// s_0 = +1 (v is the edge's first vertex), s_1 = -1. Lower-triangle tiles only;
// each entry is written with its mirror.
__global__ void __launch_bounds__(1024, 2)
gather_A_kernel(const double2* __restrict__ M, int32_t E, const int32_t* __restrict__ inc_off,
                const int32_t* __restrict__ inc, int32_t V, int32_t tiles, double* __restrict__ A,
                double* __restrict__ B, double* __restrict__ B0) {
    // blockIdx.x enumerates lower-triangular 32x32 tiles (ti >= tj); the tile is
    // written along rows, and its mirror (tj, ti) through a shared-memory
    // transpose, so both stores are coalesced.
    __shared__ double ta[32][33], tb[32][33], t0[32][33];
    // the incidence lists of the tile's 32 rows and 32 columns, staged once
    // (vertices of degree <= kDeg; a tile with a larger degree reads them from
    // global memory as it goes)
    constexpr int kDeg = 4;
    __shared__ int32_t inc_r[32][kDeg], inc_c[32][kDeg];
    __shared__ int32_t deg_r[32], deg_c[32];
    __shared__ int big;
    const int32_t t = blockIdx.x;
    int32_t ti = (int32_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((int64_t)ti * (ti + 1) / 2 > t) ti--;
    while ((int64_t)(ti + 1) * (ti + 2) / 2 <= t) ti++;
    const int32_t tj = t - ti * (ti + 1) / 2;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int32_t v = ti * 32 + ty;
    const int32_t u = tj * 32 + tx;
    (void)tiles;
    const bool ok = v < V && u < V && u <= v;
    const int tid = ty * 32 + tx;
    if (tid == 0) big = 0;
    __syncthreads();
    if (tid < 64) {
        const int k = tid & 31;
        const bool isrow = tid < 32;
        const int32_t w = (isrow ? ti : tj) * 32 + k;
        int32_t n = 0;
        if (w < V) {
            const int32_t b = inc_off[w];
            n = inc_off[w + 1] - b;
            if (n > kDeg) big = 1;
            for (int q = 0; q < n && q < kDeg; q++) (isrow ? inc_r : inc_c)[k][q] = inc[b + q];
        }
        (isrow ? deg_r : deg_c)[k] = n;
    }
    __syncthreads();
    double sb = 0.0, s0 = 0.0;
    if (ok && !big) {
        // same sums, same order as below
        for (int p = 0; p < deg_r[ty]; p++) {
            const int32_t ip = inc_r[ty][p];
            const int32_t I = ip >> 1;
            const double sa = (ip & 1) ? -1.0 : 1.0;
            const double2* row = M + (int64_t)I * E;
            for (int q = 0; q < deg_c[tx]; q++) {
                const int32_t iq = inc_c[tx][q];
                const int32_t J = iq >> 1;
                const double sgn = (iq & 1) ? -sa : sa;
                const double2 m = row[J];
                sb += sgn * m.x;
                s0 += m.y;
            }
        }
    } else if (ok) {
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
    }
    ta[ty][tx] = sb + s0;
    tb[ty][tx] = sb;
    t0[ty][tx] = s0;
    __syncthreads();
    if (ok) {
        A[(int64_t)v * V + u] = ta[ty][tx];
        if (B) B[(int64_t)v * V + u] = tb[ty][tx];
        if (B0) B0[(int64_t)v * V + u] = t0[ty][tx];
    }
    // mirror: entry (row tj*32 + ty, column ti*32 + tx) = value (ti*32 + tx, tj*32 + ty)
    const int32_t mr = tj * 32 + ty, mc = ti * 32 + tx;
    if (mc < V && mr < V && mr < mc) {
        A[(int64_t)mr * V + mc] = ta[tx][ty];
        if (B) B[(int64_t)mr * V + mc] = tb[tx][ty];
        if (B0) B0[(int64_t)mr * V + mc] = t0[tx][ty];
    }
}

// ---- closed single loop: A straight from the pair weights -------------------
//
// When the curve is one closed loop with edge I = (I, I+1 mod V) (E = V), vertex
// v is the second vertex of edge v-1 and the first of edge v, so
//   A[v][u] = sum_{I in {v-1, v}} sum_{J in {u-1, u}} s_vI s_uJ Mb'[I][J] + M0'[I][J]
// (s = +1 for the first vertex, -1 for the second): a 2 x 2 stencil on the pair
// matrix. One block per lower-triangular 32 x 32 vertex tile computes the
// 33 x 33 pair weights of its edges and the one edge before (shared memory) and
// writes A's tile and its mirror once each; nothing of size E^2 is stored. The
// pair matrix's diagonal (the row sums) is added to A's cyclic band afterwards
// (loop_band_kernel), from the same per-tile row sums as the general path.
constexpr int kLT = 32;       // vertex tile
constexpr int kLH = kLT + 1;  // edges per side: the tile's own and the one before

template <int MODE>
__global__ void __launch_bounds__(256)
assemble_loop_kernel(const double4* __restrict__ ea, const double4* __restrict__ eb,
                     const int2* __restrict__ edges, int32_t V, double distExp, double eps,
                     double* __restrict__ A, double2* __restrict__ rowpart) {
    __shared__ EdgeRec sI[kLH], sJ[kLH];
    __shared__ double2 W[kLH][kLH + 1];  // (Mb', M0') of edge pair (k, l)
    // the symmetric weights w of the same pairs, then (after the row sums) the
    // A tile staged for its mirror
    __shared__ double2 wr_raw[kLH * (kLH + 1)];
    double2(*Wr)[kLH + 1] = reinterpret_cast<double2(*)[kLH + 1]>(wr_raw);
    double(*ta)[kLT + 1] = reinterpret_cast<double(*)[kLT + 1]>(wr_raw);
    static_assert(sizeof(double) * kLT * (kLT + 1) <= sizeof(double2) * kLH * (kLH + 1),
                  "the staged A tile fits in the weights' space");
    const int32_t t = blockIdx.x;
    int32_t ti = (int32_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((int64_t)ti * (ti + 1) / 2 > t) ti--;
    while ((int64_t)(ti + 1) * (ti + 2) / 2 <= t) ti++;
    const int32_t tj = t - ti * (ti + 1) / 2;
    const int32_t v0 = ti * kLT, u0 = tj * kLT;
    const int tid = threadIdx.x;
    // edge index of row k: k = 0 is the edge before the tile, k >= 1 edge v0 + k - 1
    auto edge_of = [&](int32_t w0, int k) -> int32_t {
        if (k == 0) return w0 == 0 ? V - 1 : w0 - 1;
        const int32_t I = w0 + k - 1;
        return I < V ? I : -1;
    };
    if (tid < kLH) {
        const int32_t I = edge_of(v0, tid);
        load_edge(ea, eb, edges, V, I < 0 ? V : I, sI[tid]);  // I = V: an empty record
    } else if (tid < 2 * kLH) {
        const int32_t J = edge_of(u0, tid - kLH);
        load_edge(ea, eb, edges, V, J < 0 ? V : J, sJ[tid - kLH]);
    }
    __syncthreads();
    for (int e = tid; e < kLH * kLH; e += blockDim.x) {
        const int k = e / kLH, l = e % kLH;
        const EdgeRec& a = sI[k];
        const EdgeRec& b = sJ[l];
        const int32_t I = edge_of(v0, k), J = edge_of(u0, l);
        double2 out = make_double2(0.0, 0.0), w = out;
        const bool ok = I >= 0 && J >= 0 && I != J && a.ij.x != b.ij.x && a.ij.x != b.ij.y &&
                        a.ij.y != b.ij.x && a.ij.y != b.ij.y;
        if (ok) {
            w = pair_weight<MODE>(a, b, distExp, eps);
            const double dotT = a.T.x * b.T.x + a.T.y * b.T.y + a.T.z * b.T.z;
            out = make_double2(-w.x * dotT / (a.p1.w * b.p1.w), -w.y);
        }
        W[k][l] = out;
        Wr[k][l] = w;
    }
    __syncthreads();
    // row sums of the tile's own edges (k, l >= 1): row I over tile tj's edges,
    // and (off-diagonal tiles) row J over tile ti's edges
    if (tid < kLT) {
        const int32_t I = v0 + tid;
        if (I < V) {
            double2 rs = make_double2(0.0, 0.0);
            for (int l = 1; l < kLH; l++) {
                rs.x += Wr[tid + 1][l].x;
                rs.y += Wr[tid + 1][l].y;
            }
            rowpart[(int64_t)tj * V + I] = rs;
        }
    } else if (tid < 2 * kLT && ti != tj) {
        const int c = tid - kLT;
        const int32_t J = u0 + c;
        if (J < V) {
            double2 cs = make_double2(0.0, 0.0);
            for (int k = 1; k < kLH; k++) {
                cs.x += Wr[k][c + 1].x;
                cs.y += Wr[k][c + 1].y;
            }
            rowpart[(int64_t)ti * V + J] = cs;
        }
    }
    __syncthreads();  // the row sums have read Wr; ta takes its place
    // A[v][u] for the tile (rows v0 + r, columns u0 + c, u <= v), the incident
    // edges of each vertex in ascending edge order
    for (int e = tid; e < kLT * kLT; e += blockDim.x) {
        const int r = e / kLT, c = e % kLT;
        const int32_t v = v0 + r, u = u0 + c;
        double sb = 0.0, s0 = 0.0;
        if (v < V && u < V && u <= v) {
            // (row index in W, sign): v's edges v-1 (second vertex, -1) and v (+1)
            int kp[2], lq[2];
            double sp[2], sq[2];
            if (v == 0) { kp[0] = 1; sp[0] = 1.0; kp[1] = 0; sp[1] = -1.0; }
            else { kp[0] = r; sp[0] = -1.0; kp[1] = r + 1; sp[1] = 1.0; }
            if (u == 0) { lq[0] = 1; sq[0] = 1.0; lq[1] = 0; sq[1] = -1.0; }
            else { lq[0] = c; sq[0] = -1.0; lq[1] = c + 1; sq[1] = 1.0; }
#pragma unroll
            for (int p = 0; p < 2; p++)
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const double2 m = W[kp[p]][lq[q]];
                    sb += sp[p] * sq[q] * m.x;
                    s0 += m.y;
                }
        }
        ta[r][c] = sb + s0;
    }
    __syncthreads();
    for (int e = tid; e < kLT * kLT; e += blockDim.x) {
        const int r = e / kLT, c = e % kLT;
        const int32_t v = v0 + r, u = u0 + c;
        if (v < V && u < V && u <= v) A[(int64_t)v * V + u] = ta[r][c];
        // mirror: entry (u0 + r, v0 + c) = value (v0 + c, u0 + r)
        const int32_t mr = u0 + r, mc = v0 + c;
        if (mc < V && mr < V && mr < mc) A[(int64_t)mr * V + mc] = ta[c][r];
    }
}

// The pair matrix's diagonal on A's cyclic band: for each vertex v, the terms
// with I = J of the stencil: A[v][v] += Mb'_{v-1} + Mb'_v + M0'_{v-1} + M0'_v,
// A[v][v+1] = A[v+1][v] += -Mb'_v + M0'_v, with (Mb'_I, M0'_I) = (d_I / l_I^2, d0_I)
// summed from the per-tile row sums in tile order. Each block forms the
// diagonal entries of its 256 vertices and of the vertex before them once, in
// shared memory.
__global__ void __launch_bounds__(256) loop_band_kernel(const double4* __restrict__ ea, int32_t V,
                                                        int32_t nt, const double2* __restrict__ rowpart,
                                                        double* __restrict__ A) {
    __shared__ double2 dg[257];
    const int32_t b0 = blockIdx.x * 256;
    auto diag = [&](int32_t I) -> double2 {
        double sx = 0.0, sy = 0.0;
#pragma unroll 8
        for (int32_t s = 0; s < nt; s++) {
            const double2 p = rowpart[(int64_t)s * V + I];
            sx += p.x;
            sy += p.y;
        }
        const double ell = ea[I].w;
        return make_double2(sx / (ell * ell), sy);
    };
    const int32_t v = b0 + threadIdx.x;
    if (v < V) dg[threadIdx.x + 1] = diag(v);
    if (threadIdx.x == 0) dg[0] = diag(b0 == 0 ? V - 1 : b0 - 1);
    __syncthreads();
    if (v >= V) return;
    const double2 dv = dg[threadIdx.x + 1], dp = dg[threadIdx.x];
    A[(int64_t)v * V + v] += (dp.x + dv.x) + (dp.y + dv.y);
    const int32_t u = v + 1 == V ? 0 : v + 1;
    const double off = -dv.x + dv.y;
    A[(int64_t)v * V + u] += off;
    A[(int64_t)u * V + v] += off;
}

}  // namespace

int32_t gather_A_launch(tpe_ctx* ctx, double* d_A, double* d_B, double* d_B0) {
    const int32_t V = ctx->V, E = ctx->E;
    const int32_t nt = (V + 31) / 32;
    const int32_t tiles = nt * (nt + 1) / 2;
    KernelScope ks(ctx, TPE_KGROUP_GATHER_A, 1);
    gather_A_kernel<<<tiles, dim3(32, 32), 0, ctx->stream>>>(
        ctx->pairM.as<double2>(), E, ctx->d_inc_off.as<int32_t>(), ctx->d_inc.as<int32_t>(), V,
        tiles, d_A, d_B, d_B0);
    TPE_CUDA_TRY(cudaGetLastError());
    return TPE_OK;
}

int32_t assemble_fp64(tpe_ctx* ctx, double alpha, double beta, double eps, double* d_A,
                      double* d_B, double* d_B0) {
    const int32_t E = ctx->E;
    if (ctx->closed_loop && !d_B && !d_B0) {
        // one closed loop: A straight from the pair weights (no E x E matrix)
        const int32_t V = ctx->V;
        const double s = (beta - 1.0) / alpha;
        const double distExp = 2.0 * (s - 1.0) + 1.0;
        const int32_t nt = (V + kLT - 1) / kLT;
        const int64_t tiles = (int64_t)nt * (nt + 1) / 2;
        TPE_TRY(ensure(ctx, ctx->tmp, sizeof(double2) * (size_t)nt * V));
        {
            KernelScope ks(ctx, TPE_KGROUP_PAIR_WEIGHTS, 1);
            if (alpha == 3.0 && beta == 6.0)
                assemble_loop_kernel<1><<<(unsigned)tiles, 256, 0, ctx->stream>>>(
                    ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), V,
                    distExp, eps, d_A, ctx->tmp.as<double2>());
            else
                assemble_loop_kernel<0><<<(unsigned)tiles, 256, 0, ctx->stream>>>(
                    ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), V,
                    distExp, eps, d_A, ctx->tmp.as<double2>());
            TPE_CUDA_TRY(cudaGetLastError());
        }
        KernelScope ks(ctx, TPE_KGROUP_GATHER_A, 1);
        loop_band_kernel<<<(V + 255) / 256, 256, 0, ctx->stream>>>(ctx->edge_a.as<double4>(), V, nt,
                                                                 ctx->tmp.as<double2>(), d_A);
        TPE_CUDA_TRY(cudaGetLastError());
        return TPE_OK;
    }
    TPE_TRY(ensure(ctx, ctx->pairM, sizeof(double2) * (size_t)E * E));
    const double s = (beta - 1.0) / alpha;
    const double sigma = s - 1.0;
    const double distExp = 2.0 * sigma + 1.0;
    const int mode = (alpha == 3.0 && beta == 6.0) ? 1 : 0;
    const int32_t ntp = (E + kT - 1) / kT;
    TPE_TRY(ensure(ctx, ctx->tmp, sizeof(double2) * (size_t)ntp * E));
    {
        KernelScope ks(ctx, TPE_KGROUP_PAIR_WEIGHTS, 2);
        const int64_t tiles = (int64_t)ntp * (ntp + 1) / 2;
        if (mode == 1)
            pair_weights_kernel<1><<<(unsigned)tiles, 256, 0, ctx->stream>>>(
                ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E,
                distExp, eps, ctx->pairM.as<double2>(), ctx->tmp.as<double2>());
        else
            pair_weights_kernel<0><<<(unsigned)tiles, 256, 0, ctx->stream>>>(
                ctx->edge_a.as<double4>(), ctx->edge_b.as<double4>(), ctx->d_edges.as<int2>(), E,
                distExp, eps, ctx->pairM.as<double2>(), ctx->tmp.as<double2>());
        pair_diag_kernel<<<(E + 255) / 256, 256, 0, ctx->stream>>>(
            ctx->edge_a.as<double4>(), E, ntp, ctx->tmp.as<double2>(), ctx->pairM.as<double2>());
        TPE_CUDA_TRY(cudaGetLastError());
    }
    return gather_A_launch(ctx, d_A, d_B, d_B0);
}

}  // namespace tpe
