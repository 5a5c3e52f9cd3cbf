/*
 * tpe_oracle.h — TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * Scalar FP64 CPU restatement of the reference's TypeScript hot path
 * (src/core/tangentPointEnergy.ts, src/core/sobolev/, src/core/optimizer.ts),
 * following its operation order so that results can be compared bit for bit
 * where the reference's own tests compare bit for bit. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline legs may load it.
 *
 * Conventions: vertices are double[3*V] interleaved, edges int32_t[2*E];
 * flat vectors of length 3V use the coordinate-block layout
 * [x0..x(V-1), y0.., z0..] (src/core/sobolev/layout.ts:23-56).
 */
#ifndef TPE_ORACLE_H
#define TPE_ORACLE_H

#include <stdint.h>
#include "../include/tpe.h"

#ifdef __cplusplus
extern "C" {
#endif

/* JavaScriptCore Math.pow semantics (exponentiation by squaring for small
 * non-negative integer exponents, libm pow otherwise). */
double tpeo_js_pow(double x, double y);

/* calculateDisjointPairs (tangentPointEnergy.ts:33-47). Returns the number of
 * ordered pairs; fills offsets[E+1] and partners[<= cap] when non-NULL. */
int64_t tpeo_disjoint_pairs(const int32_t* edges, int32_t E, int32_t* offsets,
                            int32_t* partners, int64_t cap);

/* calculateEnergy over edge rows I in [I0, I1) (the full energy is rows
 * [0, E)); the /2 of tangentPointEnergy.ts:110 is applied. */
double tpeo_energy_rows(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                        double alpha, double beta, double eps, int32_t I0, int32_t I1);
double tpeo_energy(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                   double alpha, double beta, double eps);
/* gradientAnalytical (tangentPointEnergy.ts:139-392) over rows [I0, I1). */
void tpeo_gradient_rows(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                        double alpha, double beta, double eps, int32_t I0, int32_t I1,
                        double* grad);
void tpeo_gradient(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                   double alpha, double beta, double eps, double* grad);
/* gradientFiniteDiff (tangentPointEnergy.ts:114-136). */
void tpeo_gradient_fd(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                      double alpha, double beta, double eps, double h, double* grad);

/* assembleBHighFlat / assembleBLowFlat / assembleAFlat (innerProduct.ts). */
void tpeo_assemble_bhigh(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                         double alpha, double beta, double eps, double* B);
void tpeo_assemble_blow(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                        double alpha, double beta, double eps, double* B0);
void tpeo_assemble_a(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                     double alpha, double beta, double eps, double* A);
/* Pair-weight part of assembly over rows [I0, I1) only (no symmetrisation),
 * accumulating into A; used to time a bounded sample. */
void tpeo_assemble_a_rows(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                          double alpha, double beta, double eps, int32_t I0, int32_t I1,
                          double* A);

/* Geometry helpers (constraints.ts, constraintSet.ts, lineSearch.ts). */
void tpeo_barycenter_target(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                            double* x0);
double tpeo_total_length(const double* xyz, const int32_t* edges, int32_t E);
void tpeo_edge_lengths(const double* xyz, const int32_t* edges, int32_t E, double* ell);
double tpeo_l2_curve_norm(const double* values, const double* xyz, const int32_t* edges,
                          int32_t E);

/* Stacked rows k of a set; evaluateConstraintSet into phi[k] and dense C[k*3V]
 * (C may be NULL); block_scale = ConstraintBlock.scale. */
int32_t tpeo_constraint_rows(const tpe_constraint* set, int32_t nblocks, int32_t E);
void tpeo_evaluate_constraint_set(const tpe_constraint* set, int32_t nblocks,
                                  const double* xyz, int32_t V, const int32_t* edges,
                                  int32_t E, double* phi, double* C);
double tpeo_block_scale(const tpe_constraint* block, const double* xyz, int32_t V,
                        const int32_t* edges, int32_t E);

/* Dense factorizations (linsolve.ts). Return TPE_OK or TPE_ERR_SINGULAR
 * (non-finite entry or zero pivot column). Factor in place. */
int32_t tpeo_lu_factor(double* K, int32_t n, int32_t* piv);
int32_t tpeo_lu_solve(const double* K, int32_t n, const int32_t* piv, const double* rhs,
                      double* x);
int32_t tpeo_ldlt_factor(double* K, int32_t n, int32_t* ipiv);
int32_t tpeo_ldlt_solve(const double* K, int32_t n, const int32_t* ipiv, const double* rhs,
                        double* x);
/* solveSaddleFromA (linsolve.ts:742-803). rhs_bottom NULL = zeros. */
int32_t tpeo_solve_saddle_from_a(const double* A, int32_t n, const double* C, int32_t k,
                                 const double* rhs_top, const double* rhs_bottom,
                                 int32_t factor_mode, double* x, double* lambda,
                                 double* residual);

/* Penalties (penalties.ts:86-241). */
int32_t tpeo_penalties_active(const tpe_penalties* pen);
double tpeo_penalty_energy(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                           const tpe_penalties* pen);
void tpeo_penalty_gradient(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                           const tpe_penalties* pen, double* grad);

/* solveConstrainedGradientSet (gradient.ts:42-65): dE and g_tilde V x 3
 * interleaved; lambda[k]. */
int32_t tpeo_solve_constrained_gradient(const double* xyz, int32_t V, const int32_t* edges,
                                        int32_t E, const tpe_constraint* set, int32_t nblocks,
                                        const tpe_step_opts* o, const double* dE,
                                        double* g_tilde, double* lambda, double* residual);
/* projectOntoConstraintSet (lineSearch.ts:196-295); base_xyz != NULL freezes K
 * at base_xyz. */
int32_t tpeo_project(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                     const tpe_constraint* set, int32_t nblocks, const tpe_step_opts* o,
                     const double* base_xyz, double* xyz_out, int32_t* ok, int32_t* iterations,
                     double* phi_norm);
/* lineSearchStepSet (lineSearch.ts:423-562). */
int32_t tpeo_line_search_step(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                              const double* dE, const double* g_tilde,
                              const tpe_constraint* set, int32_t nblocks,
                              const tpe_step_opts* o, double* xyz_out, tpe_step_stats* st);
/* sobolevStepSet (optimizer.ts:231-440). */
int32_t tpeo_sobolev_step(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                          const tpe_constraint* set, int32_t nblocks, const tpe_step_opts* o,
                          double* xyz_out, tpe_step_stats* st, double* descent_field);

void tpeo_default_step_opts(tpe_step_opts* o);

#ifdef __cplusplus
}
#endif
#endif
