/*
 * tpe_oracle.c — TEST INFRASTRUCTURE ONLY: the CPU checker for libtpe.
 *
 * A scalar FP64 restatement of the reference's TypeScript hot path, written
 * from the reference's behaviour (file:line cited per function) and keeping
 * its operation order: x->y->z sums, epsilon added after each norm, the pre-
 * epsilon 1e-14 guards, the final /2, the `|| 0` coercion of gradient
 * increments, dsytf2-style Bunch-Kaufman pivoting, and the check-before-
 * correct projection loop. Compiled with -ffp-contract=off (JavaScript has no
 * fused multiply-add). Exponentiation follows JavaScriptCore's Math.pow
 * (tpeo_js_pow), which is what the reference's bit-exact goldens were made with.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load this
 * library; nothing in the product links against it.
 */
#include "tpe_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* JavaScript number semantics                                               */
/* ------------------------------------------------------------------------- */

/* JavaScriptCore evaluates Math.pow(x, y) (and x ** y) by exponentiation by
 * squaring when y is an integer in [0, 1000], otherwise by the C library pow. */
double tpeo_js_pow(double x, double y) {
    if (isnan(y)) return NAN;
    if (isinf(y) && fabs(x) == 1.0) return NAN;
    if (y >= 0.0 && y <= 1000.0 && y == (double)(int32_t)y) {
        int32_t n = (int32_t)y;
        double result = 1.0;
        while (n) {
            if (n & 1) result *= x;
            x *= x;
            n >>= 1;
        }
        return result;
    }
    return pow(x, y);
}

/* Math.max: NaN if any argument is NaN. */
static double js_max2(double a, double b) {
    if (isnan(a) || isnan(b)) return NAN;
    if (a == 0.0 && b == 0.0) return signbit(a) ? b : a;
    return a > b ? a : b;
}

/* `x || 0`: NaN, +0 and -0 all become +0 (tangentPointEnergy.ts:152-156). */
static inline double or0(double x) { return (x != x || x == 0.0) ? 0.0 : x; }

static inline int disjoint(const int32_t* ed, int32_t I, int32_t J) {
    if (I == J) return 0;
    const int32_t a1 = ed[2 * I], a2 = ed[2 * I + 1], b1 = ed[2 * J], b2 = ed[2 * J + 1];
    return a1 != b1 && a1 != b2 && a2 != b1 && a2 != b2;
}

#define P(v, c) xyz[3 * (v) + (c)]

/* ------------------------------------------------------------------------- */
/* Pair kernels (src/core/tangentPointEnergy.ts)                            */
/* ------------------------------------------------------------------------- */

/* calculateDisjointPairs, tangentPointEnergy.ts:33-47. */
int64_t tpeo_disjoint_pairs(const int32_t* edges, int32_t E, int32_t* offsets,
                            int32_t* partners, int64_t cap) {
    int64_t count = 0;
    for (int32_t i = 0; i < E; i++) {
        if (offsets) offsets[i] = (int32_t)count;
        for (int32_t j = 0; j < E; j++) {
            if (!disjoint(edges, i, j)) continue;
            if (partners && count < cap) partners[count] = j;
            count++;
        }
    }
    if (offsets) offsets[E] = (int32_t)count;
    return count;
}

/* calculateEnergy, tangentPointEnergy.ts:50-111. The J loop visits the ordered
 * disjoint partners of I in ascending order, as calculateDisjointPairs lists them. */
double tpeo_energy_rows(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                        double alpha, double beta, double eps, int32_t I0, int32_t I1) {
    (void)V;
    double total = 0.0;
    for (int32_t I = I0; I < I1; I++) {
        const int32_t i1 = ed[2 * I], i2 = ed[2 * I + 1];
        const double eIx = P(i2, 0) - P(i1, 0);
        const double eIy = P(i2, 1) - P(i1, 1);
        const double eIz = P(i2, 2) - P(i1, 2);
        const double ell_I = sqrt(eIx * eIx + eIy * eIy + eIz * eIz) + eps;
        for (int32_t J = 0; J < E; J++) {
            if (!disjoint(ed, I, J)) continue;
            const int32_t j1 = ed[2 * J], j2 = ed[2 * J + 1];
            const double eJx = P(j2, 0) - P(j1, 0);
            const double eJy = P(j2, 1) - P(j1, 1);
            const double eJz = P(j2, 2) - P(j1, 2);
            const double ell_J = sqrt(eJx * eJx + eJy * eJy + eJz * eJz) + eps;
            const int32_t iv[2] = {i1, i2}, jv[2] = {j1, j2};
            double sumK = 0.0;
            for (int a = 0; a < 2; a++) {
                for (int b = 0; b < 2; b++) {
                    const int32_t i = iv[a], j = jv[b];
                    const double dx = P(i, 0) - P(j, 0);
                    const double dy = P(i, 1) - P(j, 1);
                    const double dz = P(i, 2) - P(j, 2);
                    const double d_norm = sqrt(dx * dx + dy * dy + dz * dz) + eps;
                    const double cx = eIy * dz - eIz * dy;
                    const double cy = eIz * dx - eIx * dz;
                    const double cz = eIx * dy - eIy * dx;
                    const double c_norm = sqrt(cx * cx + cy * cy + cz * cz) + eps;
                    sumK += tpeo_js_pow(c_norm, alpha) / tpeo_js_pow(d_norm, beta);
                }
            }
            total += 0.25 * tpeo_js_pow(ell_I, 1.0 - alpha) * ell_J * sumK;
        }
    }
    return total / 2.0;
}

double tpeo_energy(const double* xyz, int32_t V, const int32_t* ed, int32_t E, double alpha,
                   double beta, double eps) {
    return tpeo_energy_rows(xyz, V, ed, E, alpha, beta, eps, 0, E);
}

typedef struct {
    double f, dd[3], de[3];
} kderivs;

/* kernelDerivs, tangentPointEnergy.ts:165-244: f = (|e x d|+eps)^a / (|d|+eps)^b
 * and its derivatives with respect to d and e. */
static kderivs kernel_derivs(double ex, double ey, double ez, double dx, double dy, double dz,
                             double alpha, double beta, double eps) {
    kderivs k;
    const double rd = sqrt(dx * dx + dy * dy + dz * dz);
    double hx = 0, hy = 0, hz = 0;
    if (!(rd < 1e-14)) {
        const double inv = 1.0 / rd;
        hx = inv * dx;
        hy = inv * dy;
        hz = inv * dz;
    }
    const double d_eps = rd + eps;
    const double cx = ey * dz - ez * dy;
    const double cy = ez * dx - ex * dz;
    const double cz = ex * dy - ey * dx;
    const double rc = sqrt(cx * cx + cy * cy + cz * cz);
    const double c_eps = rc + eps;
    const double cPowA = tpeo_js_pow(c_eps, alpha);
    const double dPowB = tpeo_js_pow(d_eps, beta);
    k.f = cPowA / dPowB;
    double ddx = 0, ddy = 0, ddz = 0, dex = 0, dey = 0, dez = 0;
    if (rc >= 1e-14) {
        const double invRc = 1.0 / rc;
        const double ccex = cy * ez - cz * ey;
        const double ccey = cz * ex - cx * ez;
        const double ccez = cx * ey - cy * ex;
        ddx = invRc * ccex;
        ddy = invRc * ccey;
        ddz = invRc * ccez;
        const double dccx = dy * cz - dz * cy;
        const double dccy = dz * cx - dx * cz;
        const double dccz = dx * cy - dy * cx;
        dex = invRc * dccx;
        dey = invRc * dccy;
        dez = invRc * dccz;
    }
    const double coeff_c = (alpha * tpeo_js_pow(c_eps, alpha - 1.0)) / dPowB;
    const double coeff_d = (-beta * cPowA) / tpeo_js_pow(d_eps, beta + 1.0);
    k.dd[0] = coeff_c * ddx + coeff_d * hx;
    k.dd[1] = coeff_c * ddy + coeff_d * hy;
    k.dd[2] = coeff_c * ddz + coeff_d * hz;
    k.de[0] = coeff_c * dex;
    k.de[1] = coeff_c * dey;
    k.de[2] = coeff_c * dez;
    return k;
}

static inline void add_grad(double* g, int32_t idx, double x, double y, double z) {
    g[3 * idx + 0] += or0(x);
    g[3 * idx + 1] += or0(y);
    g[3 * idx + 2] += or0(z);
}

/* gradientAnalytical, tangentPointEnergy.ts:139-392 (rows [I0, I1), then *0.5). */
void tpeo_gradient_rows(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                        double alpha, double beta, double eps, int32_t I0, int32_t I1,
                        double* g) {
    memset(g, 0, sizeof(double) * 3 * (size_t)V);
    for (int32_t I = I0; I < I1; I++) {
        const int32_t i1 = ed[2 * I], i2 = ed[2 * I + 1];
        const double eIx = P(i2, 0) - P(i1, 0);
        const double eIy = P(i2, 1) - P(i1, 1);
        const double eIz = P(i2, 2) - P(i1, 2);
        const double reI = sqrt(eIx * eIx + eIy * eIy + eIz * eIz);
        double ehx = 0, ehy = 0, ehz = 0;
        if (!(reI < 1e-14)) {
            const double inv = 1.0 / reI;
            ehx = inv * eIx;
            ehy = inv * eIy;
            ehz = inv * eIz;
        }
        const double ell_I = reI + eps;
        const double ell_I_pow = tpeo_js_pow(ell_I, 1.0 - alpha);
        const double dPowCoeff = (1.0 - alpha) * tpeo_js_pow(ell_I, -alpha);
        const double p1x = dPowCoeff * (-1.0 * ehx), p1y = dPowCoeff * (-1.0 * ehy),
                     p1z = dPowCoeff * (-1.0 * ehz);
        const double p2x = dPowCoeff * ehx, p2y = dPowCoeff * ehy, p2z = dPowCoeff * ehz;
        for (int32_t J = 0; J < E; J++) {
            if (!disjoint(ed, I, J)) continue;
            const int32_t j1 = ed[2 * J], j2 = ed[2 * J + 1];
            const double eJx = P(j2, 0) - P(j1, 0);
            const double eJy = P(j2, 1) - P(j1, 1);
            const double eJz = P(j2, 2) - P(j1, 2);
            const double reJ = sqrt(eJx * eJx + eJy * eJy + eJz * eJz);
            double jhx = 0, jhy = 0, jhz = 0;
            if (!(reJ < 1e-14)) {
                const double inv = 1.0 / reJ;
                jhx = inv * eJx;
                jhy = inv * eJy;
                jhz = inv * eJz;
            }
            const double ell_J = reJ + eps;
            const double q1x = -1.0 * jhx, q1y = -1.0 * jhy, q1z = -1.0 * jhz;
            const int32_t ti[4] = {i1, i1, i2, i2}, tj[4] = {j1, j2, j1, j2};
            kderivs k[4];
            double sumF = 0.0;
            for (int t = 0; t < 4; t++) {
                const double dx = P(ti[t], 0) - P(tj[t], 0);
                const double dy = P(ti[t], 1) - P(tj[t], 1);
                const double dz = P(ti[t], 2) - P(tj[t], 2);
                k[t] = kernel_derivs(eIx, eIy, eIz, dx, dy, dz, alpha, beta, eps);
                sumF += k[t].f;
            }
            const double sI = 0.25 * ell_J * sumF;
            add_grad(g, i1, sI * p1x, sI * p1y, sI * p1z);
            add_grad(g, i2, sI * p2x, sI * p2y, sI * p2z);
            const double sJ = 0.25 * ell_I_pow * sumF;
            add_grad(g, j1, sJ * q1x, sJ * q1y, sJ * q1z);
            add_grad(g, j2, sJ * jhx, sJ * jhy, sJ * jhz);
            const double base = 0.25 * ell_I_pow * ell_J;
            const double nbase = -base;
            for (int t = 0; t < 4; t++) {
                add_grad(g, ti[t], base * k[t].dd[0], base * k[t].dd[1], base * k[t].dd[2]);
                add_grad(g, tj[t], nbase * k[t].dd[0], nbase * k[t].dd[1], nbase * k[t].dd[2]);
                add_grad(g, i1, nbase * k[t].de[0], nbase * k[t].de[1], nbase * k[t].de[2]);
                add_grad(g, i2, base * k[t].de[0], base * k[t].de[1], base * k[t].de[2]);
            }
        }
    }
    for (int32_t v = 0; v < V; v++) {
        g[3 * v + 0] *= 0.5;
        g[3 * v + 1] *= 0.5;
        g[3 * v + 2] *= 0.5;
    }
}

void tpeo_gradient(const double* xyz, int32_t V, const int32_t* ed, int32_t E, double alpha,
                   double beta, double eps, double* g) {
    tpeo_gradient_rows(xyz, V, ed, E, alpha, beta, eps, 0, E, g);
}

/* gradientFiniteDiff, tangentPointEnergy.ts:114-136 (forward differences). */
void tpeo_gradient_fd(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                      double alpha, double beta, double eps, double h, double* g) {
    const double E0 = tpeo_energy(xyz, V, ed, E, alpha, beta, eps);
    double* pert = (double*)malloc(sizeof(double) * 3 * (size_t)V);
    for (int32_t v = 0; v < V; v++) {
        for (int d = 0; d < 3; d++) {
            memcpy(pert, xyz, sizeof(double) * 3 * (size_t)V);
            pert[3 * v + d] += h;
            const double E1 = tpeo_energy(pert, V, ed, E, alpha, beta, eps);
            g[3 * v + d] = (E1 - E0) / h;
        }
    }
    free(pert);
}

/* ------------------------------------------------------------------------- */
/* Gram assembly (src/core/sobolev/innerProduct.ts)                          */
/* ------------------------------------------------------------------------- */

static void edge_geometry_eps(const double* xyz, const int32_t* ed, int32_t E, double eps,
                              double* ell, double* T) {
    for (int32_t I = 0; I < E; I++) {
        const int32_t i1 = ed[2 * I], i2 = ed[2 * I + 1];
        const double ex = P(i2, 0) - P(i1, 0);
        const double ey = P(i2, 1) - P(i1, 1);
        const double ez = P(i2, 2) - P(i1, 2);
        const double r = sqrt(ex * ex + ey * ey + ez * ez);
        ell[I] = r + eps;
        if (r < 1e-14) {
            T[3 * I] = T[3 * I + 1] = T[3 * I + 2] = 0.0;
        } else {
            const double inv = 1.0 / r;
            T[3 * I] = ex * inv;
            T[3 * I + 1] = ey * inv;
            T[3 * I + 2] = ez * inv;
        }
    }
}

static void symmetrize(double* B, int32_t n) {
    for (int32_t i = 0; i < n; i++)
        for (int32_t j = i + 1; j < n; j++) {
            const double avg = 0.5 * (B[(size_t)i * n + j] + B[(size_t)j * n + i]);
            B[(size_t)i * n + j] = avg;
            B[(size_t)j * n + i] = avg;
        }
}

/* High-order pair accumulation of assembleBHighFlat (innerProduct.ts:79-126). */
static void bhigh_rows(const double* xyz, int32_t n, const int32_t* ed, int32_t E,
                       double alpha, double beta, double eps, const double* ell,
                       const double* T, int32_t I0, int32_t I1, double* B) {
    const double s = (beta - 1.0) / alpha;
    const double sigma = s - 1.0;
    const double distExp = 2.0 * sigma + 1.0;
    for (int32_t I = I0; I < I1; I++) {
        const int32_t idxI[2] = {ed[2 * I], ed[2 * I + 1]};
        const double ellI = ell[I];
        const double* TI = T + 3 * I;
        for (int32_t J = 0; J < E; J++) {
            if (!disjoint(ed, I, J)) continue;
            const int32_t idxJ[2] = {ed[2 * J], ed[2 * J + 1]};
            const double ellJ = ell[J];
            const double* TJ = T + 3 * J;
            double sumDist = 0.0;
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    const int32_t ia = idxI[a], jb = idxJ[b];
                    const double dx = P(ia, 0) - P(jb, 0);
                    const double dy = P(ia, 1) - P(jb, 1);
                    const double dz = P(ia, 2) - P(jb, 2);
                    const double dNorm = sqrt(dx * dx + dy * dy + dz * dz) + eps;
                    sumDist += 1.0 / tpeo_js_pow(dNorm, distExp);
                }
            const double w = 0.25 * ellI * ellJ * sumDist;
            const double dotT = TI[0] * TJ[0] + TI[1] * TJ[1] + TI[2] * TJ[2];
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    const double sign = ((a + b) % 2 == 0) ? 1.0 : -1.0;
                    const size_t ia = (size_t)idxI[a], ib = (size_t)idxI[b];
                    const size_t ja = (size_t)idxJ[a], jb = (size_t)idxJ[b];
                    B[ia * n + ib] += (sign * w) / (ellI * ellI);
                    B[ia * n + jb] -= (sign * w * dotT) / (ellI * ellJ);
                    B[ja * n + jb] += (sign * w) / (ellJ * ellJ);
                    B[ja * n + ib] -= (sign * w * dotT) / (ellI * ellJ);
                }
        }
    }
}

/* Low-order pair accumulation of assembleBLowFlat (innerProduct.ts:217-272). */
static void blow_rows(const double* xyz, int32_t n, const int32_t* ed, int32_t E,
                      double alpha, double beta, double eps, const double* ell, const double* T,
                      int32_t I0, int32_t I1, double* B0) {
    const double s = (beta - 1.0) / alpha;
    const double sigma = s - 1.0;
    const double distExp = 2.0 * sigma + 1.0;
    for (int32_t I = I0; I < I1; I++) {
        const int32_t idxI[2] = {ed[2 * I], ed[2 * I + 1]};
        const double ellI = ell[I];
        const double* TI = T + 3 * I;
        for (int32_t J = 0; J < E; J++) {
            if (!disjoint(ed, I, J)) continue;
            const int32_t idxJ[2] = {ed[2 * J], ed[2 * J + 1]};
            const double ellJ = ell[J];
            double sumLow = 0.0;
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    const int32_t ia = idxI[a], jb = idxJ[b];
                    const double dx = P(ia, 0) - P(jb, 0);
                    const double dy = P(ia, 1) - P(jb, 1);
                    const double dz = P(ia, 2) - P(jb, 2);
                    const double dNorm = sqrt(dx * dx + dy * dy + dz * dz) + eps;
                    const double cx = TI[1] * dz - TI[2] * dy;
                    const double cy = TI[2] * dx - TI[0] * dz;
                    const double cz = TI[0] * dy - TI[1] * dx;
                    const double crossNorm = sqrt(cx * cx + cy * cy + cz * cz) + eps;
                    const double k24 =
                        (crossNorm * crossNorm) / (dNorm * dNorm * dNorm * dNorm);
                    sumLow += k24 / tpeo_js_pow(dNorm, distExp);
                }
            const double wLow = 0.25 * ellI * ellJ * sumLow;
            const double q = 0.25 * wLow;
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    const size_t ia = (size_t)idxI[a], ib = (size_t)idxI[b];
                    const size_t ja = (size_t)idxJ[a], jb = (size_t)idxJ[b];
                    B0[ia * n + ib] += q;
                    B0[ia * n + jb] -= q;
                    B0[ja * n + ib] -= q;
                    B0[ja * n + jb] += q;
                }
        }
    }
}

void tpeo_assemble_bhigh(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                         double alpha, double beta, double eps, double* B) {
    double* ell = (double*)malloc(sizeof(double) * (size_t)E);
    double* T = (double*)malloc(sizeof(double) * 3 * (size_t)E);
    edge_geometry_eps(xyz, ed, E, eps, ell, T);
    memset(B, 0, sizeof(double) * (size_t)V * V);
    bhigh_rows(xyz, V, ed, E, alpha, beta, eps, ell, T, 0, E, B);
    symmetrize(B, V);
    free(ell);
    free(T);
}

void tpeo_assemble_blow(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                        double alpha, double beta, double eps, double* B0) {
    double* ell = (double*)malloc(sizeof(double) * (size_t)E);
    double* T = (double*)malloc(sizeof(double) * 3 * (size_t)E);
    edge_geometry_eps(xyz, ed, E, eps, ell, T);
    memset(B0, 0, sizeof(double) * (size_t)V * V);
    blow_rows(xyz, V, ed, E, alpha, beta, eps, ell, T, 0, E, B0);
    symmetrize(B0, V);
    free(ell);
    free(T);
}

/* assembleAFlat, innerProduct.ts:325-350: A = B + B0 elementwise. */
void tpeo_assemble_a(const double* xyz, int32_t V, const int32_t* ed, int32_t E, double alpha,
                     double beta, double eps, double* A) {
    const size_t nn = (size_t)V * V;
    double* B = (double*)malloc(sizeof(double) * nn);
    tpeo_assemble_bhigh(xyz, V, ed, E, alpha, beta, eps, B);
    tpeo_assemble_blow(xyz, V, ed, E, alpha, beta, eps, A);
    for (size_t i = 0; i < nn; i++) A[i] = B[i] + A[i];
    free(B);
}

void tpeo_assemble_a_rows(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                          double alpha, double beta, double eps, int32_t I0, int32_t I1,
                          double* A) {
    double* ell = (double*)malloc(sizeof(double) * (size_t)E);
    double* T = (double*)malloc(sizeof(double) * 3 * (size_t)E);
    edge_geometry_eps(xyz, ed, E, eps, ell, T);
    bhigh_rows(xyz, V, ed, E, alpha, beta, eps, ell, T, I0, I1, A);
    blow_rows(xyz, V, ed, E, alpha, beta, eps, ell, T, I0, I1, A);
    free(ell);
    free(T);
}

/* ------------------------------------------------------------------------- */
/* Constraints (constraints.ts, constraintSet.ts) and norms (lineSearch.ts)  */
/* ------------------------------------------------------------------------- */

/* Raw length and the safe unit tangent e*(1/len) used by the constraint rows. */
static inline double raw_edge(const double* xyz, const int32_t* ed, int32_t I, double* T) {
    const int32_t i1 = ed[2 * I], i2 = ed[2 * I + 1];
    const double ex = P(i2, 0) - P(i1, 0);
    const double ey = P(i2, 1) - P(i1, 1);
    const double ez = P(i2, 2) - P(i1, 2);
    const double ell = sqrt(ex * ex + ey * ey + ez * ez);
    if (ell < 1e-14) {
        T[0] = T[1] = T[2] = 0.0;
    } else {
        const double inv = 1.0 / ell;
        T[0] = ex * inv;
        T[1] = ey * inv;
        T[2] = ez * inv;
    }
    return ell;
}

/* barycenterTarget, constraints.ts:23-52. */
void tpeo_barycenter_target(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                            double* x0) {
    double total = 0.0, acc[3] = {0, 0, 0};
    for (int32_t I = 0; I < E; I++) {
        const int32_t i1 = ed[2 * I], i2 = ed[2 * I + 1];
        const double ex = P(i2, 0) - P(i1, 0);
        const double ey = P(i2, 1) - P(i1, 1);
        const double ez = P(i2, 2) - P(i1, 2);
        const double ell = sqrt(ex * ex + ey * ey + ez * ez);
        total += ell;
        for (int c = 0; c < 3; c++) acc[c] += ell * 0.5 * (P(i1, c) + P(i2, c));
    }
    if (total < 1e-14) {
        double mean[3] = {0, 0, 0};
        for (int32_t v = 0; v < V; v++)
            for (int c = 0; c < 3; c++) mean[c] += P(v, c) / (double)V;
        for (int c = 0; c < 3; c++) x0[c] = mean[c];
        return;
    }
    for (int c = 0; c < 3; c++) x0[c] = acc[c] / total;
}

/* totalLength, constraintSet.ts:64-75. */
double tpeo_total_length(const double* xyz, const int32_t* ed, int32_t E) {
    double L = 0.0;
    for (int32_t I = 0; I < E; I++) {
        const int32_t i1 = ed[2 * I], i2 = ed[2 * I + 1];
        const double ex = P(i2, 0) - P(i1, 0);
        const double ey = P(i2, 1) - P(i1, 1);
        const double ez = P(i2, 2) - P(i1, 2);
        L += sqrt(ex * ex + ey * ey + ez * ez);
    }
    return L;
}

/* edgeLengths, constraintSet.ts:172-181. */
void tpeo_edge_lengths(const double* xyz, const int32_t* ed, int32_t E, double* ell) {
    for (int32_t I = 0; I < E; I++) {
        const int32_t i1 = ed[2 * I], i2 = ed[2 * I + 1];
        const double ex = P(i2, 0) - P(i1, 0);
        const double ey = P(i2, 1) - P(i1, 1);
        const double ez = P(i2, 2) - P(i1, 2);
        ell[I] = sqrt(ex * ex + ey * ey + ez * ez);
    }
}

/* l2CurveNorm, lineSearch.ts:53-75 (values is V x 3 interleaved). */
double tpeo_l2_curve_norm(const double* values, const double* xyz, const int32_t* ed,
                          int32_t E) {
    double total = 0.0;
    for (int32_t I = 0; I < E; I++) {
        const int32_t i1 = ed[2 * I], i2 = ed[2 * I + 1];
        const double ex = P(i2, 0) - P(i1, 0);
        const double ey = P(i2, 1) - P(i1, 1);
        const double ez = P(i2, 2) - P(i1, 2);
        const double ell = sqrt(ex * ex + ey * ey + ez * ez);
        const double* v1 = values + 3 * i1;
        const double* v2 = values + 3 * i2;
        total += 0.5 * ell *
                 (v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2] +
                  (v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2]));
    }
    return sqrt(js_max2(0.0, total));
}

/* barycenterScale, lineSearch.ts:86-109. */
static double barycenter_scale(const double* xyz, const int32_t* ed, int32_t E,
                               const double* x0) {
    double L = 0.0, R = 0.0;
    for (int32_t I = 0; I < E; I++) {
        const int32_t i1 = ed[2 * I], i2 = ed[2 * I + 1];
        const double ex = P(i2, 0) - P(i1, 0);
        const double ey = P(i2, 1) - P(i1, 1);
        const double ez = P(i2, 2) - P(i1, 2);
        L += sqrt(ex * ex + ey * ey + ez * ez);
        const double d1x = P(i1, 0) - x0[0], d1y = P(i1, 1) - x0[1], d1z = P(i1, 2) - x0[2];
        const double d2x = P(i2, 0) - x0[0], d2y = P(i2, 1) - x0[1], d2z = P(i2, 2) - x0[2];
        R = js_max2(js_max2(R, sqrt(d1x * d1x + d1y * d1y + d1z * d1z)),
                    sqrt(d2x * d2x + d2y * d2y + d2z * d2z));
    }
    return js_max2(1.0, L * js_max2(1.0, R));
}

static int32_t block_rows(const tpe_constraint* b, int32_t E) {
    switch (b->kind) {
        case TPE_BLOCK_BARYCENTER: return 3;
        case TPE_BLOCK_TOTAL_LENGTH: return 1;
        case TPE_BLOCK_EDGE_LENGTHS: return E;
        case TPE_BLOCK_POINT: return 3;
        default: return -1;
    }
}

int32_t tpeo_constraint_rows(const tpe_constraint* set, int32_t nblocks, int32_t E) {
    int32_t k = 0;
    for (int32_t b = 0; b < nblocks; b++) {
        const int32_t r = block_rows(&set[b], E);
        if (r < 0) return -1;
        k += r;
    }
    return k;
}

/* One block's Phi rows and dense C rows (row stride 3V). */
static void evaluate_block(const tpe_constraint* b, const double* xyz, int32_t n,
                           const int32_t* ed, int32_t E, double* phi, double* C) {
    const size_t m = 3 * (size_t)n;
    const int32_t rows = block_rows(b, E);
    if (C) memset(C, 0, sizeof(double) * m * (size_t)rows);
    double T[3];
    switch (b->kind) {
        case TPE_BLOCK_BARYCENTER: { /* barycenterPhiAndC, constraints.ts:67-120 */
            const double* x0 = b->target;
            phi[0] = phi[1] = phi[2] = 0.0;
            for (int32_t I = 0; I < E; I++) {
                const int32_t i1 = ed[2 * I], i2 = ed[2 * I + 1];
                const double ell = raw_edge(xyz, ed, I, T);
                double rvec[3];
                for (int r = 0; r < 3; r++) rvec[r] = 0.5 * (P(i1, r) + P(i2, r)) - x0[r];
                phi[0] += ell * rvec[0];
                phi[1] += ell * rvec[1];
                phi[2] += ell * rvec[2];
                if (!C) continue;
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) {
                        const double delta = (r == c) ? 1.0 : 0.0;
                        C[r * m + (size_t)c * n + i1] += -T[c] * rvec[r] + 0.5 * ell * delta;
                        C[r * m + (size_t)c * n + i2] += T[c] * rvec[r] + 0.5 * ell * delta;
                    }
            }
            break;
        }
        case TPE_BLOCK_TOTAL_LENGTH: { /* constraintSet.ts:119-162 */
            double L = 0.0;
            for (int32_t I = 0; I < E; I++) {
                const int32_t i1 = ed[2 * I], i2 = ed[2 * I + 1];
                const double ell = raw_edge(xyz, ed, I, T);
                L += ell;
                if (!C) continue;
                for (int c = 0; c < 3; c++) {
                    C[(size_t)c * n + i1] += T[c];
                    C[(size_t)c * n + i2] += -T[c];
                }
            }
            phi[0] = b->L0 - L;
            break;
        }
        case TPE_BLOCK_EDGE_LENGTHS: { /* constraintSet.ts:206-250 */
            for (int32_t r = 0; r < E; r++) {
                const int32_t i1 = ed[2 * r], i2 = ed[2 * r + 1];
                const double ell = raw_edge(xyz, ed, r, T);
                const double target = (b->ell0 && r < b->n_ell0) ? b->ell0[r] : NAN;
                phi[r] = target - ell;
                if (!C) continue;
                for (int c = 0; c < 3; c++) {
                    C[(size_t)r * m + (size_t)c * n + i1] += T[c];
                    C[(size_t)r * m + (size_t)c * n + i2] += -T[c];
                }
            }
            break;
        }
        case TPE_BLOCK_POINT: { /* constraintSet.ts:271-301 */
            const int32_t v = b->vertex;
            if (v < 0 || v >= n) {
                phi[0] = phi[1] = phi[2] = NAN;
                break;
            }
            for (int r = 0; r < 3; r++) {
                if (C) C[(size_t)r * m + (size_t)r * n + v] = 1.0;
                phi[r] = P(v, r) - b->target[r];
            }
            break;
        }
        default: break;
    }
}

void tpeo_evaluate_constraint_set(const tpe_constraint* set, int32_t nblocks,
                                  const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                                  double* phi, double* C) {
    int32_t row = 0;
    for (int32_t b = 0; b < nblocks; b++) {
        evaluate_block(&set[b], xyz, V, ed, E, phi + row,
                       C ? C + (size_t)row * 3 * V : NULL);
        row += block_rows(&set[b], E);
    }
}

/* ConstraintBlock.scale for each catalog block (lineSearch.ts:86-109,
 * constraintSet.ts:154-160, 242-248, 287-299). */
double tpeo_block_scale(const tpe_constraint* b, const double* xyz, int32_t V,
                        const int32_t* ed, int32_t E) {
    switch (b->kind) {
        case TPE_BLOCK_BARYCENTER: return barycenter_scale(xyz, ed, E, b->target);
        case TPE_BLOCK_TOTAL_LENGTH:
        case TPE_BLOCK_EDGE_LENGTHS: return js_max2(1.0, tpeo_total_length(xyz, ed, E));
        case TPE_BLOCK_POINT: {
            double R = 0.0;
            for (int32_t v = 0; v < V; v++) {
                const double dx = P(v, 0) - b->target[0];
                const double dy = P(v, 1) - b->target[1];
                const double dz = P(v, 2) - b->target[2];
                R = js_max2(R, sqrt(dx * dx + dy * dy + dz * dz));
            }
            return js_max2(1.0, R);
        }
        default: return NAN;
    }
}

/* ------------------------------------------------------------------------- */
/* Dense solvers (src/core/sobolev/linsolve.ts)                              */
/* ------------------------------------------------------------------------- */

static int all_finite(const double* a, size_t n) {
    for (size_t i = 0; i < n; i++)
        if (!isfinite(a[i])) return 0;
    return 1;
}

/* luFactor, linsolve.ts:243-316. */
int32_t tpeo_lu_factor(double* k, int32_t n, int32_t* piv) {
    if (!all_finite(k, (size_t)n * n)) return TPE_ERR_SINGULAR;
    for (int32_t i = 0; i < n; i++) piv[i] = i;
    for (int32_t col = 0; col < n; col++) {
        int32_t pivotRow = col;
        double maxAbs = fabs(k[(size_t)col * n + col]);
        for (int32_t r = col + 1; r < n; r++) {
            const double a = fabs(k[(size_t)r * n + col]);
            if (a > maxAbs) {
                maxAbs = a;
                pivotRow = r;
            }
        }
        if (!(maxAbs > 0)) return TPE_ERR_SINGULAR;
        if (pivotRow != col) {
            double* ra = k + (size_t)col * n;
            double* rb = k + (size_t)pivotRow * n;
            for (int32_t c = 0; c < n; c++) {
                const double t = ra[c];
                ra[c] = rb[c];
                rb[c] = t;
            }
            const int32_t tp = piv[col];
            piv[col] = piv[pivotRow];
            piv[pivotRow] = tp;
        }
        const double* rowc = k + (size_t)col * n;
        const double pivotVal = rowc[col];
        for (int32_t r = col + 1; r < n; r++) {
            double* rowr = k + (size_t)r * n;
            const double mult = rowr[col] / pivotVal;
            rowr[col] = mult;
            for (int32_t c = col + 1; c < n; c++) rowr[c] -= mult * rowc[c];
        }
    }
    return TPE_OK;
}

/* luSolveFactored, linsolve.ts:326-360. */
int32_t tpeo_lu_solve(const double* m, int32_t n, const int32_t* piv, const double* rhs,
                      double* x) {
    if (!all_finite(rhs, (size_t)n)) return TPE_ERR_NONFINITE_INPUT;
    double* y = (double*)malloc(sizeof(double) * (size_t)n);
    for (int32_t i = 0; i < n; i++) {
        double s = rhs[piv[i]];
        const double* row = m + (size_t)i * n;
        for (int32_t j = 0; j < i; j++) s -= row[j] * y[j];
        y[i] = s;
    }
    for (int32_t i = n - 1; i >= 0; i--) {
        double s = y[i];
        const double* row = m + (size_t)i * n;
        for (int32_t j = i + 1; j < n; j++) s -= row[j] * x[j];
        x[i] = s / row[i];
    }
    free(y);
    return TPE_OK;
}

/* ldltFactor, linsolve.ts:431-589: Bunch-Kaufman (LAPACK dsytf2, UPLO='L')
 * on the lower triangle of a row-major buffer, with the trailing updates
 * visited row-wise and LAPACK's 1-based ipiv encoding. */
int32_t tpeo_ldlt_factor(double* k, int32_t n, int32_t* ipiv) {
    if (!all_finite(k, (size_t)n * n)) return TPE_ERR_SINGULAR;
    const double ALPHA = (1.0 + sqrt(17.0)) / 8.0;
    double* w1 = (double*)calloc((size_t)n, sizeof(double));
    double* w2 = (double*)calloc((size_t)n, sizeof(double));
#define K(i, j) k[(size_t)(i) * n + (j)]
    int32_t col = 0;
    while (col < n) {
        const double absakk = fabs(K(col, col));
        int32_t imax = col;
        double colmax = 0.0;
        for (int32_t r = col + 1; r < n; r++) {
            const double a = fabs(K(r, col));
            if (a > colmax) {
                colmax = a;
                imax = r;
            }
        }
        if (!(js_max2(absakk, colmax) > 0)) {
            free(w1);
            free(w2);
            return TPE_ERR_SINGULAR;
        }
        int32_t kstep = 1, kp = col;
        if (absakk >= ALPHA * colmax) {
            kp = col;
        } else {
            double rowmax = 0.0;
            for (int32_t j = col; j < imax; j++) rowmax = js_max2(rowmax, fabs(K(imax, j)));
            for (int32_t r = imax + 1; r < n; r++) rowmax = js_max2(rowmax, fabs(K(r, imax)));
            if (absakk >= ALPHA * colmax * (colmax / rowmax)) {
                kp = col;
            } else if (fabs(K(imax, imax)) >= ALPHA * rowmax) {
                kp = imax;
            } else {
                kp = imax;
                kstep = 2;
            }
        }
        const int32_t kk = col + kstep - 1;
        if (kp != kk) {
            for (int32_t r = kp + 1; r < n; r++) {
                const double t = K(r, kk);
                K(r, kk) = K(r, kp);
                K(r, kp) = t;
            }
            for (int32_t j = kk + 1; j < kp; j++) {
                const double t = K(j, kk);
                K(j, kk) = K(kp, j);
                K(kp, j) = t;
            }
            const double td = K(kk, kk);
            K(kk, kk) = K(kp, kp);
            K(kp, kp) = td;
            if (kstep == 2) {
                const double t = K(col + 1, col);
                K(col + 1, col) = K(kp, col);
                K(kp, col) = t;
            }
        }
        if (kstep == 1) {
            if (col < n - 1) {
                const double d11 = 1.0 / K(col, col);
                for (int32_t j = col + 1; j < n; j++) w1[j] = d11 * K(j, col);
                for (int32_t i = col + 1; i < n; i++) {
                    const double aik = K(i, col);
                    double* rowi = k + (size_t)i * n;
                    for (int32_t j = col + 1; j <= i; j++) rowi[j] -= aik * w1[j];
                }
                for (int32_t r = col + 1; r < n; r++) K(r, col) *= d11;
            }
        } else {
            if (col < n - 2) {
                const double d21 = K(col + 1, col);
                const double d11 = K(col + 1, col + 1) / d21;
                const double d22 = K(col, col) / d21;
                const double t = 1.0 / (d11 * d22 - 1.0);
                const double d21t = t / d21;
                for (int32_t j = col + 2; j < n; j++) {
                    const double ajk = K(j, col);
                    const double ajk1 = K(j, col + 1);
                    w1[j] = d21t * (d11 * ajk - ajk1);
                    w2[j] = d21t * (d22 * ajk1 - ajk);
                }
                for (int32_t i = col + 2; i < n; i++) {
                    const double aik = K(i, col);
                    const double aik1 = K(i, col + 1);
                    double* rowi = k + (size_t)i * n;
                    for (int32_t j = col + 2; j <= i; j++)
                        rowi[j] = rowi[j] - aik * w1[j] - aik1 * w2[j];
                }
                for (int32_t j = col + 2; j < n; j++) {
                    K(j, col) = w1[j];
                    K(j, col + 1) = w2[j];
                }
            }
        }
        if (kstep == 1) {
            ipiv[col] = kp + 1;
        } else {
            ipiv[col] = -(kp + 1);
            ipiv[col + 1] = -(kp + 1);
        }
        col += kstep;
    }
    free(w1);
    free(w2);
    return TPE_OK;
}

/* ldltSolveFactored, linsolve.ts:603-691 (LAPACK dsytrs, UPLO='L'). */
int32_t tpeo_ldlt_solve(const double* m, int32_t n, const int32_t* ipiv, const double* rhs,
                        double* b) {
    if (!all_finite(rhs, (size_t)n)) return TPE_ERR_NONFINITE_INPUT;
    memcpy(b, rhs, sizeof(double) * (size_t)n);
#define M(i, j) m[(size_t)(i) * n + (j)]
    int32_t i = 0;
    while (i < n) {
        if (ipiv[i] > 0) {
            const int32_t kp = ipiv[i] - 1;
            if (kp != i) {
                const double t = b[i];
                b[i] = b[kp];
                b[kp] = t;
            }
            for (int32_t r = i + 1; r < n; r++) b[r] -= M(r, i) * b[i];
            b[i] /= M(i, i);
            i += 1;
        } else {
            const int32_t kp = -ipiv[i] - 1;
            if (kp != i + 1) {
                const double t = b[i + 1];
                b[i + 1] = b[kp];
                b[kp] = t;
            }
            for (int32_t r = i + 2; r < n; r++) b[r] = b[r] - M(r, i) * b[i] - M(r, i + 1) * b[i + 1];
            const double akm1k = M(i + 1, i);
            const double akm1 = M(i, i) / akm1k;
            const double ak = M(i + 1, i + 1) / akm1k;
            const double denom = akm1 * ak - 1.0;
            const double bkm1 = b[i] / akm1k;
            const double bk = b[i + 1] / akm1k;
            b[i] = (ak * bkm1 - bk) / denom;
            b[i + 1] = (akm1 * bk - bkm1) / denom;
            i += 2;
        }
    }
    i = n - 1;
    while (i >= 0) {
        if (ipiv[i] > 0) {
            double s = b[i];
            for (int32_t r = i + 1; r < n; r++) s -= M(r, i) * b[r];
            b[i] = s;
            const int32_t kp = ipiv[i] - 1;
            if (kp != i) {
                const double t = b[i];
                b[i] = b[kp];
                b[kp] = t;
            }
            i -= 1;
        } else {
            double s = b[i];
            for (int32_t r = i + 1; r < n; r++) s -= M(r, i) * b[r];
            b[i] = s;
            double s1 = b[i - 1];
            for (int32_t r = i + 1; r < n; r++) s1 -= M(r, i - 1) * b[r];
            b[i - 1] = s1;
            const int32_t kp = -ipiv[i] - 1;
            if (kp != i) {
                const double t = b[i];
                b[i] = b[kp];
                b[kp] = t;
            }
            i -= 2;
        }
    }
    return TPE_OK;
}

/* structuredSaddleResidual, linsolve.ts:810-849. */
static double structured_residual(const double* a, int32_t n, const double* C, int32_t k,
                                  const double* z, const double* rhs) {
    const size_t m = 3 * (size_t)n;
    double resNormSq = 0.0, rhsNormSq = 0.0;
    for (int b = 0; b < 3; b++) {
        const size_t off = (size_t)b * n;
        for (int32_t i = 0; i < n; i++) {
            double s = 0.0;
            const double* row = a + (size_t)i * n;
            for (int32_t j = 0; j < n; j++) s += row[j] * z[off + j];
            const size_t r0 = off + i;
            for (int32_t r = 0; r < k; r++) s += C[(size_t)r * m + r0] * z[m + r];
            const double d = s - rhs[r0];
            resNormSq += d * d;
            rhsNormSq += rhs[r0] * rhs[r0];
        }
    }
    for (int32_t r = 0; r < k; r++) {
        double s = 0.0;
        const double* Cr = C + (size_t)r * m;
        for (size_t j = 0; j < m; j++) s += Cr[j] * z[j];
        const double d = s - rhs[m + r];
        resNormSq += d * d;
        rhsNormSq += rhs[m + r] * rhs[m + r];
    }
    return sqrt(resNormSq) / js_max2(1.0, sqrt(rhsNormSq));
}

/* A frozen saddle operator (linsolve.ts:865-870): the unfactored a and C plus
 * the packed factorization of K. */
typedef struct {
    const double* a;
    int32_t n;
    const double* C;
    int32_t k;
    double* fac;
    int32_t* piv;
    int32_t factor_mode;
} saddle_op;

static void build_saddle(const double* a, int32_t n, const double* C, int32_t k, double* K) {
    const size_t m = 3 * (size_t)n, size = m + (size_t)k;
    memset(K, 0, sizeof(double) * size * size);
    for (int b = 0; b < 3; b++) {
        const size_t off = (size_t)b * n;
        for (int32_t i = 0; i < n; i++)
            memcpy(K + (off + i) * size + off, a + (size_t)i * n, sizeof(double) * (size_t)n);
    }
    for (int32_t r = 0; r < k; r++) {
        const double* Cr = C + (size_t)r * m;
        for (size_t j = 0; j < m; j++) {
            K[(m + r) * size + j] = Cr[j];
            K[j * size + (m + r)] = Cr[j];
        }
    }
}

static int32_t op_factor(saddle_op* op) {
    const size_t size = 3 * (size_t)op->n + (size_t)op->k;
    op->fac = (double*)malloc(sizeof(double) * size * size);
    op->piv = (int32_t*)malloc(sizeof(int32_t) * (size + 1));
    if (!op->fac || !op->piv) return TPE_ERR_OUT_OF_MEMORY;
    build_saddle(op->a, op->n, op->C, op->k, op->fac);
    return op->factor_mode == TPE_FACTOR_LU ? tpeo_lu_factor(op->fac, (int32_t)size, op->piv)
                                            : tpeo_ldlt_factor(op->fac, (int32_t)size, op->piv);
}

static int32_t op_solve(const saddle_op* op, const double* rhs, double* z, double* residual) {
    const int32_t size = 3 * op->n + op->k;
    const int32_t st = op->factor_mode == TPE_FACTOR_LU
                           ? tpeo_lu_solve(op->fac, size, op->piv, rhs, z)
                           : tpeo_ldlt_solve(op->fac, size, op->piv, rhs, z);
    if (st != TPE_OK) return st;
    if (residual) *residual = structured_residual(op->a, op->n, op->C, op->k, z, rhs);
    return TPE_OK;
}

static void op_free(saddle_op* op) {
    free(op->fac);
    free(op->piv);
    op->fac = NULL;
    op->piv = NULL;
}

/* solveSaddleFromA, linsolve.ts:742-803. */
int32_t tpeo_solve_saddle_from_a(const double* A, int32_t n, const double* C, int32_t k,
                                 const double* rhs_top, const double* rhs_bottom,
                                 int32_t factor_mode, double* x, double* lambda,
                                 double* residual) {
    const size_t m = 3 * (size_t)n, size = m + (size_t)k;
    saddle_op op = {A, n, C, k, NULL, NULL, factor_mode};
    int32_t st = op_factor(&op);
    if (st != TPE_OK) {
        op_free(&op);
        return st;
    }
    double* rhs = (double*)malloc(sizeof(double) * size);
    double* z = (double*)malloc(sizeof(double) * size);
    memcpy(rhs, rhs_top, sizeof(double) * m);
    for (int32_t r = 0; r < k; r++) rhs[m + r] = rhs_bottom ? rhs_bottom[r] : 0.0;
    double res = 0.0;
    st = op_solve(&op, rhs, z, &res);
    if (st == TPE_OK) {
        memcpy(x, z, sizeof(double) * m);
        if (lambda) memcpy(lambda, z + m, sizeof(double) * (size_t)k);
        if (residual) *residual = res;
    }
    free(rhs);
    free(z);
    op_free(&op);
    return st;
}

/* ------------------------------------------------------------------------- */
/* Penalties (src/core/sobolev/penalties.ts)                                 */
/* ------------------------------------------------------------------------- */

typedef struct {
    double wLength, wDiff, wField, X[3];
} resolved_pen;

/* resolve, penalties.ts:60-77. */
static resolved_pen resolve_pen(const tpe_penalties* c) {
    resolved_pen r = {c->total_length, c->length_diff, c->field_weight, {0, 0, 0}};
    if (r.wField != 0.0) {
        const double x = c->field_X[0], y = c->field_X[1], z = c->field_X[2];
        const double n = sqrt(x * x + y * y + z * z);
        if (n < 1e-14) {
            r.wField = 0.0;
        } else {
            r.X[0] = x / n;
            r.X[1] = y / n;
            r.X[2] = z / n;
        }
    }
    return r;
}

/* penaltiesActive, penalties.ts:86-90. */
int32_t tpeo_penalties_active(const tpe_penalties* c) {
    if (!c) return 0;
    const resolved_pen r = resolve_pen(c);
    return r.wLength != 0.0 || r.wDiff != 0.0 || r.wField != 0.0;
}

/* edgeGeometry, penalties.ts:95-110 (tangent by division e/len). */
static void pen_geometry(const double* xyz, const int32_t* ed, int32_t E, double* ell, double* T) {
    for (int32_t r = 0; r < E; r++) {
        const int32_t i1 = ed[2 * r], i2 = ed[2 * r + 1];
        const double ex = P(i2, 0) - P(i1, 0);
        const double ey = P(i2, 1) - P(i1, 1);
        const double ez = P(i2, 2) - P(i1, 2);
        const double len = sqrt(ex * ex + ey * ey + ez * ez);
        ell[r] = len;
        if (len < 1e-14) {
            T[3 * r] = T[3 * r + 1] = T[3 * r + 2] = 0.0;
        } else {
            T[3 * r] = ex / len;
            T[3 * r + 1] = ey / len;
            T[3 * r + 2] = ez / len;
        }
    }
}

/* interiorVertices, penalties.ts:116-127: (v, I_v, J_v) for degree-2 vertices,
 * incident edges in ascending edge order. Returns the count; out has 3 ints each. */
static int32_t interior_vertices(int32_t n, const int32_t* ed, int32_t E, int32_t* out) {
    int32_t* deg = (int32_t*)calloc((size_t)n, sizeof(int32_t));
    int32_t* first = (int32_t*)malloc(sizeof(int32_t) * (size_t)n * 2);
    for (int32_t r = 0; r < E; r++) {
        for (int s = 0; s < 2; s++) {
            const int32_t v = ed[2 * r + s];
            if (deg[v] < 2) first[2 * v + deg[v]] = r;
            deg[v]++;
        }
    }
    int32_t cnt = 0;
    for (int32_t v = 0; v < n; v++)
        if (deg[v] == 2) {
            out[3 * cnt] = v;
            out[3 * cnt + 1] = first[2 * v];
            out[3 * cnt + 2] = first[2 * v + 1];
            cnt++;
        }
    free(deg);
    free(first);
    return cnt;
}

/* penaltyEnergy, penalties.ts:139-168. */
double tpeo_penalty_energy(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                           const tpe_penalties* c) {
    const resolved_pen r = resolve_pen(c);
    double* ell = (double*)malloc(sizeof(double) * (size_t)E);
    double* T = (double*)malloc(sizeof(double) * 3 * (size_t)E);
    pen_geometry(xyz, ed, E, ell, T);
    double total = 0.0;
    if (r.wLength != 0.0) {
        double acc = 0.0;
        for (int32_t e = 0; e < E; e++) acc += ell[e];
        total += r.wLength * acc;
    }
    if (r.wDiff != 0.0) {
        int32_t* iv = (int32_t*)malloc(sizeof(int32_t) * 3 * (size_t)(V > 0 ? V : 1));
        const int32_t cnt = interior_vertices(V, ed, E, iv);
        double acc = 0.0;
        for (int32_t q = 0; q < cnt; q++) {
            const double d = ell[iv[3 * q + 1]] - ell[iv[3 * q + 2]];
            acc += d * d;
        }
        total += r.wDiff * acc;
        free(iv);
    }
    if (r.wField != 0.0) {
        double acc = 0.0;
        for (int32_t e = 0; e < E; e++) {
            const double* t = T + 3 * e;
            const double cx = t[1] * r.X[2] - t[2] * r.X[1];
            const double cy = t[2] * r.X[0] - t[0] * r.X[2];
            const double cz = t[0] * r.X[1] - t[1] * r.X[0];
            acc += ell[e] * (cx * cx + cy * cy + cz * cz);
        }
        total += r.wField * acc;
    }
    free(ell);
    free(T);
    return total;
}

/* penaltyGradient, penalties.ts:183-241. */
void tpeo_penalty_gradient(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                           const tpe_penalties* c, double* g) {
    const resolved_pen r = resolve_pen(c);
    double* ell = (double*)malloc(sizeof(double) * (size_t)E);
    double* T = (double*)malloc(sizeof(double) * 3 * (size_t)E);
    pen_geometry(xyz, ed, E, ell, T);
    memset(g, 0, sizeof(double) * 3 * (size_t)V);
    if (r.wLength != 0.0) {
        for (int32_t e = 0; e < E; e++) {
            const int32_t a = ed[2 * e], b = ed[2 * e + 1];
            const double* t = T + 3 * e;
            for (int q = 0; q < 3; q++) g[3 * a + q] -= r.wLength * t[q];
            for (int q = 0; q < 3; q++) g[3 * b + q] += r.wLength * t[q];
        }
    }
    if (r.wDiff != 0.0) {
        int32_t* iv = (int32_t*)malloc(sizeof(int32_t) * 3 * (size_t)(V > 0 ? V : 1));
        const int32_t cnt = interior_vertices(V, ed, E, iv);
        for (int32_t q = 0; q < cnt; q++) {
            const int32_t rI = iv[3 * q + 1], rJ = iv[3 * q + 2];
            const double s = 2.0 * r.wDiff * (ell[rI] - ell[rJ]);
            const double* tI = T + 3 * rI;
            const int32_t aI = ed[2 * rI], bI = ed[2 * rI + 1];
            for (int u = 0; u < 3; u++) g[3 * aI + u] -= s * tI[u];
            for (int u = 0; u < 3; u++) g[3 * bI + u] += s * tI[u];
            const double* tJ = T + 3 * rJ;
            const int32_t aJ = ed[2 * rJ], bJ = ed[2 * rJ + 1];
            for (int u = 0; u < 3; u++) g[3 * aJ + u] += s * tJ[u];
            for (int u = 0; u < 3; u++) g[3 * bJ + u] -= s * tJ[u];
        }
        free(iv);
    }
    if (r.wField != 0.0) {
        for (int32_t e = 0; e < E; e++) {
            if (ell[e] < 1e-14) continue;
            const double* t = T + 3 * e;
            const double u = t[0] * r.X[0] + t[1] * r.X[1] + t[2] * r.X[2];
            const double cc = 1.0 + u * u;
            const double gv[3] = {cc * t[0] - 2.0 * u * r.X[0], cc * t[1] - 2.0 * u * r.X[1],
                                  cc * t[2] - 2.0 * u * r.X[2]};
            const int32_t a = ed[2 * e], b = ed[2 * e + 1];
            for (int q = 0; q < 3; q++) g[3 * a + q] -= r.wField * gv[q];
            for (int q = 0; q < 3; q++) g[3 * b + q] += r.wField * gv[q];
        }
    }
    free(ell);
    free(T);
}

/* ------------------------------------------------------------------------- */
/* Gradient solve, projection, line search, step                             */
/* ------------------------------------------------------------------------- */

void tpeo_default_step_opts(tpe_step_opts* o) {
    memset(o, 0, sizeof(*o));
    o->struct_size = (int32_t)sizeof(*o);
    o->mode = TPE_DE_ANALYTICAL;
    o->alpha = 3.0;
    o->beta = 6.0;
    o->epsilon = 1e-10;
    o->h = 1e-6;
    o->projection_mode = TPE_PROJECTION_REASSEMBLE;
    o->factor_mode = TPE_FACTOR_LDLT;
    o->c1 = 1e-4;
    o->shrink = 0.5;
    o->tau0 = 1.0;
    o->tau_min = 1e-12;
    o->proj_tol_abs = 1e-4;
    o->proj_tol_rel = 1e-4;
    o->proj_max_iter = 8;
    o->precision = TPE_PRECISION_FP64;
    o->trials = 1;
    o->refine_max_iter = 30;
    o->refine_tol = 1e-12;
}

static void to_block(const double* v3, int32_t n, double* flat) {
    for (int32_t i = 0; i < n; i++) {
        flat[i] = v3[3 * i];
        flat[n + i] = v3[3 * i + 1];
        flat[2 * n + i] = v3[3 * i + 2];
    }
}

static void from_block(const double* flat, int32_t n, double* v3) {
    for (int32_t i = 0; i < n; i++) {
        v3[3 * i] = flat[i];
        v3[3 * i + 1] = flat[n + i];
        v3[3 * i + 2] = flat[2 * n + i];
    }
}

/* Build the frozen operator K(xyz) for `set` (solveConstrainedGradientSetFrozen,
 * gradient.ts:84-115): owns a, C and the factorization. */
static int32_t build_operator(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                              const tpe_constraint* set, int32_t nb, const tpe_step_opts* o,
                              saddle_op* op) {
    const int32_t k = tpeo_constraint_rows(set, nb, E);
    double* a = (double*)malloc(sizeof(double) * (size_t)V * V);
    double* C = (double*)malloc(sizeof(double) * (size_t)(k > 0 ? k : 1) * 3 * V);
    double* phi = (double*)malloc(sizeof(double) * (size_t)(k > 0 ? k : 1));
    tpeo_assemble_a(xyz, V, ed, E, o->alpha, o->beta, o->epsilon, a);
    tpeo_evaluate_constraint_set(set, nb, xyz, V, ed, E, phi, C);
    free(phi);
    op->a = a;
    op->n = V;
    op->C = C;
    op->k = k;
    op->fac = NULL;
    op->piv = NULL;
    op->factor_mode = o->factor_mode;
    return op_factor(op);
}

static void free_operator(saddle_op* op) {
    free((double*)op->a);
    free((double*)op->C);
    op_free(op);
}

int32_t tpeo_solve_constrained_gradient(const double* xyz, int32_t V, const int32_t* ed,
                                        int32_t E, const tpe_constraint* set, int32_t nb,
                                        const tpe_step_opts* o, const double* dE,
                                        double* g_tilde, double* lambda, double* residual) {
    saddle_op op;
    int32_t st = build_operator(xyz, V, ed, E, set, nb, o, &op);
    if (st == TPE_OK) {
        const size_t m = 3 * (size_t)V, size = m + (size_t)op.k;
        double* rhs = (double*)calloc(size, sizeof(double));
        double* z = (double*)malloc(sizeof(double) * size);
        to_block(dE, V, rhs);
        st = op_solve(&op, rhs, z, residual);
        if (st == TPE_OK) {
            from_block(z, V, g_tilde);
            if (lambda) memcpy(lambda, z + m, sizeof(double) * (size_t)op.k);
        }
        free(rhs);
        free(z);
    }
    free_operator(&op);
    return st;
}

/* projectOntoConstraintSet, lineSearch.ts:196-295, with an optional frozen op. */
static void project_impl(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                         const tpe_constraint* set, int32_t nb, const tpe_step_opts* o,
                         const saddle_op* frozen, double* cur, int32_t* ok, int32_t* iters,
                         double* phi_norm) {
    const int32_t k = tpeo_constraint_rows(set, nb, E);
    const size_t m = 3 * (size_t)V;
    memcpy(cur, xyz, sizeof(double) * m);
    double finalPhiNorm = INFINITY;
    double* phi = (double*)malloc(sizeof(double) * (size_t)(k > 0 ? k : 1));
    double* C = (double*)malloc(sizeof(double) * (size_t)(k > 0 ? k : 1) * m);
    double* rhs = (double*)malloc(sizeof(double) * (m + (size_t)k));
    double* z = (double*)malloc(sizeof(double) * (m + (size_t)k));
    double* a = frozen ? NULL : (double*)malloc(sizeof(double) * (size_t)V * V);
    const int32_t maxIter = o->proj_max_iter;
    *ok = 0;
    *iters = maxIter;
    for (int32_t it = 0; it <= maxIter; it++) {
        tpeo_evaluate_constraint_set(set, nb, cur, V, ed, E, phi, C);
        double sq = 0.0;
        for (int32_t r = 0; r < k; r++) sq += phi[r] * phi[r];
        finalPhiNorm = sqrt(sq);
        int converged = 1;
        int32_t row = 0;
        for (int32_t b = 0; b < nb; b++) {
            const int32_t rows = block_rows(&set[b], E);
            double bs = 0.0;
            for (int32_t r = 0; r < rows; r++) bs += phi[row + r] * phi[row + r];
            row += rows;
            const double blockNorm = sqrt(bs);
            const double tol =
                js_max2(o->proj_tol_abs, o->proj_tol_rel * tpeo_block_scale(&set[b], cur, V, ed, E));
            if (blockNorm > tol) {
                converged = 0;
                break;
            }
        }
        if (converged) {
            *ok = 1;
            *iters = it;
            break;
        }
        if (it == maxIter) break;
        memset(rhs, 0, sizeof(double) * m);
        for (int32_t r = 0; r < k; r++) rhs[m + r] = -phi[r];
        int32_t st;
        if (frozen) {
            st = op_solve(frozen, rhs, z, NULL);
        } else {
            tpeo_assemble_a(cur, V, ed, E, o->alpha, o->beta, o->epsilon, a);
            saddle_op op = {a, V, C, k, NULL, NULL, o->factor_mode};
            st = op_factor(&op);
            if (st == TPE_OK) st = op_solve(&op, rhs, z, NULL);
            op_free(&op);
        }
        if (st != TPE_OK) {
            *iters = it;
            break;
        }
        int finite = 1;
        for (size_t i = 0; i < m; i++)
            if (!isfinite(z[i])) finite = 0;
        if (!finite) {
            *iters = it;
            break;
        }
        for (int32_t i = 0; i < V; i++) {
            cur[3 * i] = cur[3 * i] + z[i];
            cur[3 * i + 1] = cur[3 * i + 1] + z[V + i];
            cur[3 * i + 2] = cur[3 * i + 2] + z[2 * V + i];
        }
    }
    *phi_norm = finalPhiNorm;
    free(phi);
    free(C);
    free(rhs);
    free(z);
    free(a);
}

int32_t tpeo_project(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                     const tpe_constraint* set, int32_t nb, const tpe_step_opts* o,
                     const double* base_xyz, double* xyz_out, int32_t* ok, int32_t* iterations,
                     double* phi_norm) {
    saddle_op op;
    const saddle_op* fr = NULL;
    if (base_xyz) {
        if (build_operator(base_xyz, V, ed, E, set, nb, o, &op) != TPE_OK) {
            free_operator(&op);
            memcpy(xyz_out, xyz, sizeof(double) * 3 * (size_t)V);
            *ok = 0;
            *iterations = 0;
            *phi_norm = INFINITY;
            return TPE_ERR_SINGULAR;
        }
        fr = &op;
    }
    project_impl(xyz, V, ed, E, set, nb, o, fr, xyz_out, ok, iterations, phi_norm);
    if (fr) free_operator(&op);
    return TPE_OK;
}

static double objective(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                        const tpe_step_opts* o, int pen) {
    const double e = tpeo_energy(xyz, V, ed, E, o->alpha, o->beta, o->epsilon);
    return pen ? e + tpeo_penalty_energy(xyz, V, ed, E, &o->penalties) : e;
}

static void stats_reset(tpe_step_stats* st) {
    memset(st, 0, sizeof(*st));
    st->slope = NAN;
    st->projection_phi_norm = NAN;
    st->projection_iterations = -1;
}

/* lineSearchStepSet with an optional frozen operator. */
static void line_search_impl(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                             const double* dE, const double* g, const tpe_constraint* set,
                             int32_t nb, const tpe_step_opts* o, const saddle_op* frozen,
                             double* out, tpe_step_stats* st) {
    const int pen = o->has_penalties && tpeo_penalties_active(&o->penalties);
    const size_t m = 3 * (size_t)V;
    const double e0 = o->has_energy_before ? o->energy_before : objective(xyz, V, ed, E, o, pen);
    const double gradNorm = tpeo_l2_curve_norm(g, xyz, ed, E);
    st->energy_before = e0;
    st->energy = e0;
    st->tau = 0.0;
    st->accepted = 0;
    memcpy(out, xyz, sizeof(double) * m);
    if (!isfinite(gradNorm) || gradNorm <= 0) {
        st->reason = TPE_REASON_ZERO_OR_NONFINITE_GRADIENT_NORM;
        st->projection_iterations = 0;
        return;
    }
    st->gradient_l2_norm = gradNorm;
    double* dir = (double*)calloc(m, sizeof(double));
    for (size_t i = 0; i < m; i++) dir[i] = g[i] / gradNorm;
    double* dEf = (double*)malloc(sizeof(double) * m);
    double* dirf = (double*)malloc(sizeof(double) * m);
    to_block(dE, V, dEf);
    to_block(dir, V, dirf);
    double slope = 0.0;
    for (size_t i = 0; i < m; i++) slope += dEf[i] * dirf[i];
    st->slope = slope;
    free(dEf);
    free(dirf);
    if (!isfinite(slope) || slope <= 0) {
        st->reason = TPE_REASON_NOT_A_DESCENT_DIRECTION;
        st->projection_iterations = 0;
        free(dir);
        return;
    }
    double* raw = (double*)malloc(sizeof(double) * m);
    double* proj = (double*)malloc(sizeof(double) * m);
    double tau = o->tau0;
    int32_t lastReason = TPE_REASON_TAU_BELOW_MIN;
    int32_t trials = 0;
    while (tau >= o->tau_min) {
        for (size_t i = 0; i < m; i++) raw[i] = xyz[i] - tau * dir[i];
        int32_t ok = 0, iters = 0;
        double phiNorm = 0.0;
        project_impl(raw, V, ed, E, set, nb, o, frozen, proj, &ok, &iters, &phiNorm);
        int finite = 1;
        for (size_t i = 0; i < m; i++)
            if (!isfinite(proj[i])) finite = 0;
        if (ok && finite) {
            const double e1 = objective(proj, V, ed, E, o, pen);
            trials++;
            if (isfinite(e1) && e1 <= e0 - o->c1 * tau * slope) {
                st->accepted = 1;
                st->reason = TPE_REASON_NONE;
                st->tau = tau;
                st->energy = e1;
                st->projection_iterations = iters;
                st->projection_phi_norm = phiNorm;
                st->trials_evaluated = trials;
                memcpy(out, proj, sizeof(double) * m);
                free(raw);
                free(proj);
                free(dir);
                return;
            }
            lastReason = TPE_REASON_ARMIJO_FAILED;
        } else {
            lastReason = TPE_REASON_PROJECTION_FAILED;
        }
        tau *= o->shrink;
    }
    st->reason = lastReason;
    st->trials_evaluated = trials;
    free(raw);
    free(proj);
    free(dir);
}

int32_t tpeo_line_search_step(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                              const double* dE, const double* g, const tpe_constraint* set,
                              int32_t nb, const tpe_step_opts* o, double* out,
                              tpe_step_stats* st) {
    stats_reset(st);
    saddle_op op;
    const saddle_op* fr = NULL;
    if (o->projection_mode == TPE_PROJECTION_FROZEN) {
        if (build_operator(xyz, V, ed, E, set, nb, o, &op) != TPE_OK) {
            free_operator(&op);
            return TPE_ERR_SINGULAR;
        }
        fr = &op;
    }
    line_search_impl(xyz, V, ed, E, dE, g, set, nb, o, fr, out, st);
    if (fr) free_operator(&op);
    return TPE_OK;
}

/* sobolevStepSet, optimizer.ts:231-440 (SOBOLEV_CONVERGENCE_TOL = 1e-4, :78). */
int32_t tpeo_sobolev_step(const double* xyz, int32_t V, const int32_t* ed, int32_t E,
                          const tpe_constraint* set, int32_t nb, const tpe_step_opts* o,
                          double* out, tpe_step_stats* st, double* descent_field) {
    stats_reset(st);
    const size_t m = 3 * (size_t)V;
    const int pen = o->has_penalties && tpeo_penalties_active(&o->penalties);
    double* dE = (double*)malloc(sizeof(double) * m);
    if (o->mode == TPE_DE_FINITE_DIFF)
        tpeo_gradient_fd(xyz, V, ed, E, o->alpha, o->beta, o->epsilon, o->h, dE);
    else
        tpeo_gradient(xyz, V, ed, E, o->alpha, o->beta, o->epsilon, dE);
    if (pen) {
        double* pg = (double*)malloc(sizeof(double) * m);
        tpeo_penalty_gradient(xyz, V, ed, E, &o->penalties, pg);
        for (size_t i = 0; i < m; i++) dE[i] = dE[i] + pg[i];
        free(pg);
    }
    memcpy(out, xyz, sizeof(double) * m);
    saddle_op op;
    int32_t sst = build_operator(xyz, V, ed, E, set, nb, o, &op);
    double* g = (double*)malloc(sizeof(double) * m);
    double residual = NAN;
    if (sst == TPE_OK) {
        const size_t size = m + (size_t)op.k;
        double* rhs = (double*)calloc(size, sizeof(double));
        double* z = (double*)malloc(sizeof(double) * size);
        to_block(dE, V, rhs);
        sst = op_solve(&op, rhs, z, &residual);
        if (sst == TPE_OK) from_block(z, V, g);
        free(rhs);
        free(z);
    }
    if (sst != TPE_OK) {
        st->energy = o->has_energy_before ? o->energy_before : objective(xyz, V, ed, E, o, pen);
        st->energy_before = st->energy;
        st->residual = NAN;
        st->gradient_l2_norm = NAN;
        st->reason = TPE_REASON_SINGULAR_SYSTEM;
        free_operator(&op);
        free(dE);
        free(g);
        return TPE_OK;
    }
    if (descent_field) memcpy(descent_field, g, sizeof(double) * m);
    const double gn = tpeo_l2_curve_norm(g, xyz, ed, E);
    st->residual = residual;
    st->gradient_l2_norm = gn;
    if (gn < 1e-4) {
        st->energy = o->has_energy_before ? o->energy_before : objective(xyz, V, ed, E, o, pen);
        st->energy_before = st->energy;
        st->converged = 1;
        st->projection_iterations = 0;
        free_operator(&op);
        free(dE);
        free(g);
        return TPE_OK;
    }
    tpe_step_stats ls;
    stats_reset(&ls);
    line_search_impl(xyz, V, ed, E, dE, g, set, nb, o,
                     o->projection_mode == TPE_PROJECTION_FROZEN ? &op : NULL, out, &ls);
    st->energy = ls.energy;
    st->energy_before = ls.energy_before;
    st->accepted = ls.accepted;
    st->tau = ls.tau;
    st->projection_iterations = ls.projection_iterations;
    st->projection_phi_norm = ls.projection_phi_norm;
    st->slope = ls.slope;
    st->reason = ls.reason;
    st->trials_evaluated = ls.trials_evaluated;
    st->residual = residual;
    st->gradient_l2_norm = gn;
    free_operator(&op);
    free(dE);
    free(g);
    return TPE_OK;
}
