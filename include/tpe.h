/*
 * tpe.h — C ABI of libtpe, the sm_100a implementation of the constrained
 * fractional-Sobolev descent step for repulsive curves (tangent-point energy).
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, returns an
 * int status (TPE_OK = 0) and never throws, traps or aborts across the
 * boundary. Host buffers are owned by the caller; the library copies them to
 * device memory owned by the context and writes only into caller-provided
 * outputs. Vertices are `double[3*V]` interleaved (x0,y0,z0,x1,...), edges are
 * `int32_t[2*E]` index pairs — the packing a TypeScript shim produces from
 * `Vec3[]` / `Edge[]` (src/core/testConfigs.ts:1-2).
 *
 * The reference interface each entry point replaces is cited beside it
 * (paths are relative to the reference repository root).
 */
#ifndef TPE_H
#define TPE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TPE_ABI_VERSION 1

/* ---- status codes -------------------------------------------------------- */
enum {
    TPE_OK = 0,
    TPE_ERR_BAD_ARG = 1,          /* null pointer, size mismatch, index out of range */
    TPE_ERR_CUDA = 2,             /* a CUDA runtime call failed; see tpe_last_error */
    TPE_ERR_SINGULAR = 3,         /* saddle system singular or non-finite (linsolve.ts:247-276 "singular") */
    TPE_ERR_NONFINITE_INPUT = 4,  /* non-finite right-hand side (linsolve.ts:333-337) */
    TPE_ERR_NO_TOPOLOGY = 5,      /* tpe_set_topology has not been called */
    TPE_ERR_OUT_OF_MEMORY = 6,
    TPE_ERR_INVALID_SET = 7,      /* totalLength + edgeLengths in one set (constraintSet.ts:333-344) */
    TPE_ERR_REFINE_NOT_CONVERGED = 8, /* mixed path: the FP64 CG hit its cap */
    TPE_ERR_DEVICE_TIMEOUT = 9,   /* a bounded device-side wait gave up */
    TPE_ERR_TOO_LARGE = 10,       /* request exceeds a fixed-capacity buffer */
    TPE_ERR_INTERNAL = 11         /* a host-side C++ exception; see tpe_last_error */
};

/* ---- step outcome reasons (optimizer.ts:186, lineSearch.ts:374-379) ------- */
enum {
    TPE_REASON_NONE = 0,
    TPE_REASON_ZERO_OR_NONFINITE_GRADIENT_NORM = 1,
    TPE_REASON_NOT_A_DESCENT_DIRECTION = 2,
    TPE_REASON_ARMIJO_FAILED = 3,
    TPE_REASON_PROJECTION_FAILED = 4,
    TPE_REASON_TAU_BELOW_MIN = 5,
    TPE_REASON_SINGULAR_SYSTEM = 6
};

/* ---- constraint blocks (constraintSet.ts:39-43 ConstraintBlock) ---------- */
enum {
    TPE_BLOCK_BARYCENTER = 0,     /* barycenterBlock(x0)      constraintSet.ts:87-98, 3 rows  */
    TPE_BLOCK_TOTAL_LENGTH = 1,   /* totalLengthBlock(L0)     constraintSet.ts:119-162, 1 row */
    TPE_BLOCK_EDGE_LENGTHS = 2,   /* edgeLengthsBlock(ell0)   constraintSet.ts:206-250, E rows */
    TPE_BLOCK_POINT = 3           /* pointBlock(v, target)    constraintSet.ts:271-301, 3 rows */
};

/* The plain-data form of one ConstraintBlock: the closure-captured target of
 * the TypeScript block made explicit so it can cross the FFI. */
typedef struct {
    int32_t kind;          /* TPE_BLOCK_* */
    int32_t vertex;        /* point: pinned vertex (out of range -> NaN rows, as pointBlock) */
    double target[3];      /* barycenter: x0; point: pin target */
    double L0;             /* totalLength: frozen L0 (NaN allowed: projection then fails) */
    const double* ell0;    /* edgeLengths: frozen per-edge targets */
    int32_t n_ell0;        /* length of ell0; != E -> missing entries are NaN */
    int32_t reserved;
} tpe_constraint;

typedef struct {
    double alpha, beta, epsilon;   /* DEFAULTS = {3, 6, 1e-10} (optimizer.ts:18) */
} tpe_params;

/* PenaltyConfig (penalties.ts:33-49); weight 0 = off. */
typedef struct {
    double total_length;   /* totalLength weight */
    double length_diff;    /* lengthDiff weight */
    double field_weight;   /* field.weight */
    double field_X[3];     /* field.X (normalised inside, |X| < 1e-14 -> off) */
} tpe_penalties;

enum { TPE_DE_ANALYTICAL = 0, TPE_DE_FINITE_DIFF = 1 };          /* SobolevStepOptions.mode */
enum { TPE_PROJECTION_REASSEMBLE = 0, TPE_PROJECTION_FROZEN = 1 }; /* ProjectionMode (optimizer.ts:86) */
enum { TPE_FACTOR_LDLT = 0, TPE_FACTOR_LU = 1 };                  /* FactorMode (linsolve.ts:370) */
enum { TPE_PRECISION_FP64 = 0, TPE_PRECISION_MIXED = 1 };

/* SobolevStepOptions (optimizer.ts:95-175) + LineSearchOptions (lineSearch.ts:333-371)
 * + ProjectConstraintSetOptions (lineSearch.ts:120-145), flattened. Fill it with
 * tpe_default_step_opts() and override fields. */
typedef struct {
    int32_t struct_size;           /* sizeof(tpe_step_opts), for versioning */
    int32_t mode;                  /* TPE_DE_* */
    double alpha, beta, epsilon, h;
    int32_t has_energy_before;     /* energyBefore supplied? */
    int32_t projection_mode;       /* TPE_PROJECTION_* (function default: reassemble) */
    double energy_before;
    int32_t factor_mode;           /* TPE_FACTOR_* (accepted; the structured solve ignores it) */
    int32_t has_penalties;
    tpe_penalties penalties;
    double c1, shrink, tau0, tau_min;          /* 1e-4, 0.5, 1, 1e-12 */
    double proj_tol_abs, proj_tol_rel;         /* 1e-4, 1e-4 */
    int32_t proj_max_iter;                     /* 8 */
    int32_t precision;             /* TPE_PRECISION_* (extension): MIXED factors in 3xTF32 on the
                                      tensor cores with an FP64 CG, or, for more than 64
                                      constraint rows with frozen projection, forms the
                                      explicit inverses from int8 digit products */
    int32_t trials;                /* frozen projection: step sizes projected together per batch
                                      (extension; default 8, 1 = one at a time; the accepted tau
                                      and vertices do not depend on it) */
    int32_t collect_field;         /* write g~ into descent_field when non-null */
    int32_t refine_max_iter;       /* mixed path: CG iteration cap, default 60 (extension) */
    int32_t reserved;
    double refine_tol;             /* mixed path: relative residual target (extension) */
} tpe_step_opts;

/* SobolevStepStats (optimizer.ts:196-202) + LineSearchStepResult (lineSearch.ts:389-400). */
typedef struct {
    double energy;                 /* returned objective (energyAfter on accept) */
    double energy_before;
    double tau;
    double residual;               /* saddle relative residual (NaN on singular) */
    double gradient_l2_norm;       /* ||g~||_{L2h} (NaN on singular) */
    double slope;                  /* NaN where the reference leaves it undefined */
    double projection_phi_norm;    /* NaN = null */
    int32_t accepted;
    int32_t converged;
    int32_t projection_iterations; /* -1 = null */
    int32_t reason;                /* TPE_REASON_* */
    int32_t refine_iterations;     /* mixed path: CG iterations of the gradient solve;
                                      0 = FP64 factorization, or (large constraint sets)
                                      the int8-tensor-core inverses; -1 = mixed requested but
                                      the FP32 factor broke down, CG missed refine_tol, or the
                                      int8 inverses missed the residual gate (FP64 used) */
    int32_t trials_evaluated;      /* tau trials whose energy was evaluated */
} tpe_step_stats;

/* Phase keys of the timing ledger (phaseTimings.ts:9-20; extra keys appended).
 * The timings array is double[2*TPE_PHASE_COUNT]: {ms, calls} per key. */
enum {
    TPE_PHASE_DE = 0, TPE_PHASE_ENERGY, TPE_PHASE_BHIGH, TPE_PHASE_BLOW, TPE_PHASE_ASSEMBLEA,
    TPE_PHASE_EXPAND, TPE_PHASE_SADDLE, TPE_PHASE_FACTOR, TPE_PHASE_PROJECTION,
    TPE_PHASE_LINESEARCH, TPE_PHASE_STEP, TPE_PHASE_REFINE, TPE_PHASE_COUNT
};

typedef struct tpe_ctx tpe_ctx;

/* ---- context -------------------------------------------------------------- */
int32_t tpe_abi_version(void);
void tpe_default_step_opts(tpe_step_opts* opts);
/* Creates a context bound to CUDA device `device` (the TypeScript side holds
 * one per Web Worker). Every entry point that takes a context holds that
 * context's mutex for the whole call, so calls on one context from several
 * host threads run one after another; tpe_destroy must not overlap them.
 * Returns NULL on failure with *status set. */
tpe_ctx* tpe_create(int32_t device, int32_t* status);
void tpe_destroy(tpe_ctx* ctx);
/* Message for the last non-OK status returned on this context. */
const char* tpe_last_error(const tpe_ctx* ctx);

/* ---- topology ------------------------------------------------------------- */
/* Replaces calculateDisjointPairs (src/core/tangentPointEnergy.ts:33-47): the
 * ordered disjoint-pair lists are never materialised; disjointness is tested
 * in-kernel from endpoint indices. Uploads edges and the vertex->edge
 * incidence used by the gather kernels. */
int32_t tpe_set_topology(tpe_ctx* ctx, const int32_t* edges, int32_t E, int32_t V);
/* Optional: materialise the ordered lists exactly as calculateDisjointPairs
 * (offsets[E+1], partners[cap]); for callers that still want them. */
int32_t tpe_disjoint_pairs(tpe_ctx* ctx, int32_t* offsets, int32_t* partners, int64_t cap);

/* ---- energy and its gradient (one FFI energy/gradient entry) -------------- */
/* calculateEnergy (tangentPointEnergy.ts:50-111). */
int32_t tpe_energy(tpe_ctx* ctx, const double* xyz, const tpe_params* p, double* energy);
/* gradientAnalytical (tangentPointEnergy.ts:139-392) fused with the forward
 * energy; grad may be NULL (energy only) and energy may be NULL. */
int32_t tpe_energy_grad(tpe_ctx* ctx, const double* xyz, const tpe_params* p,
                        double* energy, double* grad);
/* gradientFiniteDiff (tangentPointEnergy.ts:114-136): forward differences. */
int32_t tpe_gradient_fd(tpe_ctx* ctx, const double* xyz, const tpe_params* p, double h,
                        double* grad);

/* ---- Gram assembly -------------------------------------------------------- */
/* assembleBHighFlat / assembleBLowFlat / assembleAFlat (sobolev/innerProduct.ts:38-140,
 * 177-285, 325-350): V*V row-major outputs, each may be NULL. */
int32_t tpe_assemble(tpe_ctx* ctx, const double* xyz, const tpe_params* p,
                     double* B_out, double* B0_out, double* A_out);

/* ---- constraints ---------------------------------------------------------- */
/* Number of stacked rows k of a set (sum of block row counts). */
int32_t tpe_constraint_rows(const tpe_ctx* ctx, const tpe_constraint* set, int32_t nblocks);
/* evaluateConstraintSet (sobolev/constraintSet.ts:309-322): phi[k] and the dense
 * k x 3V Jacobian C (coordinate-block columns, layout.ts:56); C may be NULL. */
int32_t tpe_evaluate_constraints(tpe_ctx* ctx, const double* xyz, const tpe_constraint* set,
                                 int32_t nblocks, double* phi, double* C);
/* l2CurveNorm (sobolev/lineSearch.ts:53-75). */
int32_t tpe_l2_curve_norm(tpe_ctx* ctx, const double* values, const double* xyz, double* out);

/* ---- saddle solve --------------------------------------------------------- */
/* solveSaddleFromA (sobolev/linsolve.ts:742-803): solves
 * [[diag(A,A,A), C^T],[C, 0]] [x; lambda] = [rhs_top; rhs_bottom] with A the
 * V x V scalar matrix (row-major), C dense k x 3V, rhs_bottom NULL = zeros.
 * x[3V] coordinate-block layout, lambda[k], residual = ||Kz-rhs||/max(1,||rhs||). */
int32_t tpe_solve_saddle(tpe_ctx* ctx, const double* A, int32_t n, const double* C, int32_t k,
                         const double* rhs_top, const double* rhs_bottom, int32_t factor_mode,
                         double* x, double* lambda, double* residual);
/* solveConstrainedGradientSet (sobolev/gradient.ts:42-65): assembles A and C at
 * xyz and solves [[A3,C^T],[C,0]][g;l] = [dE;0]. dE and g_tilde are V x 3 interleaved. */
int32_t tpe_solve_constrained_gradient(tpe_ctx* ctx, const double* xyz, const double* dE,
                                       const tpe_constraint* set, int32_t nblocks,
                                       const tpe_step_opts* opts, double* g_tilde,
                                       double* lambda, double* residual);

/* ---- projection, line search, the step ------------------------------------ */
/* projectOntoConstraintSet (sobolev/lineSearch.ts:196-295). base_xyz != NULL
 * selects the frozen operator K(base) (solveConstrainedGradientSetFrozen's
 * operator); NULL reassembles at every iterate. */
int32_t tpe_project(tpe_ctx* ctx, const double* xyz, const tpe_constraint* set, int32_t nblocks,
                    const tpe_step_opts* opts, const double* base_xyz, double* xyz_out,
                    int32_t* ok, int32_t* iterations, double* phi_norm);
/* lineSearchStepSet (sobolev/lineSearch.ts:423-562), dE / g_tilde supplied by
 * the caller; opts->projection_mode FROZEN freezes K at xyz. */
int32_t tpe_line_search_step(tpe_ctx* ctx, const double* xyz, const double* dE,
                             const double* g_tilde, const tpe_constraint* set, int32_t nblocks,
                             const tpe_step_opts* opts, double* xyz_out, tpe_step_stats* stats);
/* sobolevStepSet (src/core/optimizer.ts:231-440): the whole step. timings is
 * double[2*TPE_PHASE_COUNT] or NULL; descent_field (V x 3) receives g~ when
 * opts->collect_field and non-NULL. */
int32_t tpe_sobolev_step(tpe_ctx* ctx, const double* xyz, const tpe_constraint* set,
                         int32_t nblocks, const tpe_step_opts* opts, double* xyz_out,
                         tpe_step_stats* stats, double* timings, double* descent_field);

/* ---- penalties (sobolev/penalties.ts:139-241) ----------------------------- */
int32_t tpe_penalty_energy(tpe_ctx* ctx, const double* xyz, const tpe_penalties* pen,
                           double* energy);
int32_t tpe_penalty_gradient(tpe_ctx* ctx, const double* xyz, const tpe_penalties* pen,
                             double* grad);

/* ---- batching (no single reference counterpart: many sobolevStepSet calls) */
/* A batch of `ncurves` independent curves, one context (streams, buffers) each;
 * replaces calling sobolevStepSet (src/core/optimizer.ts:231-440) once per
 * curve. */
typedef struct tpe_batch tpe_batch;
tpe_batch* tpe_batch_create(int32_t device, int32_t ncurves, int32_t* status);
void tpe_batch_destroy(tpe_batch* batch);
/* Context of curve i (tpe_last_error, or any single-curve call). */
tpe_ctx* tpe_batch_context(tpe_batch* batch, int32_t i);
int32_t tpe_batch_set_topology(tpe_batch* batch, int32_t i, const int32_t* edges, int32_t E,
                               int32_t V);
/* One tpe_sobolev_step per curve, all curves concurrently (host threads drive
 * the curves' contexts, largest first; max_threads <= 0: one per host core).
 * Per curve i: xyz[i] (V_i x 3), sets[i] / nblocks[i], opts[i], xyz_out[i],
 * stats[i] and status[i] (the step's return code). Returns TPE_OK when every
 * curve did, else the status of the first failing curve. */
int32_t tpe_step_batch(tpe_batch* batch, const double* const* xyz,
                       const tpe_constraint* const* sets, const int32_t* nblocks,
                       const tpe_step_opts* opts, double* const* xyz_out, tpe_step_stats* stats,
                       int32_t* status, int32_t max_threads);

/* Barnes-Hut energy for curves far beyond the dense kernels' sizes: the
 * reference's stage-2 oracle bh_energy (oracle/tpe_stage2_oracle.py:532-589),
 * same tree (build_edge_bvh :467-502, built on the host), same admissibility
 * (a node of >= 2 edges sharing no vertex with the target edge, node radius /
 * distance <= theta, tangent radius <= theta_t; theta_t < 0 means 1.5 theta)
 * and cluster term. theta = 0 gives the exact energy. stats (nullable, 3):
 * tree visits, approximated edge references, exactly summed pairs. */
int32_t tpe_energy_bh(tpe_ctx* ctx, const double* xyz, const tpe_params* p, double theta,
                      double theta_t, int32_t leaf_size, double* energy, int64_t* stats);

/* phi = K psi for the high-order (kind TPE_BCT_HIGH) or low-order (TPE_BCT_LOW)
 * edge kernel of the Sobolev inner product by the block cluster tree: the
 * stage-2 oracle's bct_matvec_kernel (oracle/tpe_stage2_oracle.py:649-703), same
 * tree, same block recursion and admissibility (>= 3 edges in the block, no
 * shared vertex, max radius / distance <= theta, max tangent radius <=
 * theta_t; theta_t < 0 means 1.5 theta), node kernel bct_kernel_node (:634-643)
 * and exact pair kernel exact_edge_kernel_pair (:706-730). psi and phi are E x
 * ncols host arrays, ncols 1 or 3. theta = 0 gives the exact product. stats
 * (nullable, 4): block-tree leaves, admissible blocks, direct blocks, direct
 * pairs. */
enum { TPE_BCT_HIGH = 0, TPE_BCT_LOW = 1 };
/* The edge tree those two calls build (build_edge_bvh, oracle/tpe_stage2_oracle.py:467-502),
 * on the host only (no device, no context), for checking it node by node: per node
 * node_f[9] = center xyz, mean tangent xyz, mass, rx, rT and node_i[4] = first
 * position in perm, edge count, left, right (-1 for a leaf); perm[E] lists the
 * edges so that every node's edges are one contiguous range. *n_nodes receives
 * the node count; TPE_ERR_TOO_LARGE when it exceeds max_nodes. */
int32_t tpe_edge_tree(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                      double epsilon, int32_t leaf_size, int32_t max_nodes, double* node_f,
                      int32_t* node_i, int32_t* perm, int32_t* n_nodes);
int32_t tpe_bct_matvec(tpe_ctx* ctx, const double* xyz, int32_t kind, const double* psi,
                       int32_t ncols, double epsilon, double theta, double theta_t,
                       int32_t leaf_size, double* phi, int64_t* stats);

/* One coarsening step of the stage-2 multigrid hierarchy (build_coarse_level,
 * oracle/tpe_stage2_oracle.py:816-937), on the host (no device, no context):
 * anchors (degree != 2, pinned), alternate coloring of the chains and cycles,
 * the black vertices as the coarse level, a prolongation from the first two
 * black neighbours (weights 1/2, or 1 from a single one), coarse edges along
 * the fine paths with their original edges. Inputs: the level's V vertices, E
 * edges, orig[V] (original vertex of each), each edge's original fine edges
 * (path_edges with offsets path_off[E + 1]) and the pinned original vertices.
 * Outputs, caller-allocated (at most V coarse vertices, E coarse edges and
 * path_off[E] path entries): black[Vc], the prolongation p_idx[2V] / p_w[2V]
 * (-1 where a slot is empty), cedges[2 Ec], cpath_off[Ec + 1], cpath_edges.
 * *Vc = 0 where the oracle stops (no coarser level). */
int32_t tpe_mg_coarsen(int32_t V, const int32_t* edges, int32_t E, const int32_t* orig,
                       const int32_t* path_off, const int32_t* path_edges, const int32_t* pinned,
                       int32_t npinned, int32_t min_vertices, int32_t* black, int32_t* p_idx,
                       double* p_w, int32_t* cedges, int32_t* cpath_off, int32_t* cpath_edges,
                       int32_t* Vc, int32_t* Ec);

/* Energies of `ncurves` curves that share this context's topology (e.g. the K
 * tau-trial candidates of one line search) in one launch: xyz is
 * ncurves x V x 3, energies[ncurves]. */
int32_t tpe_energy_batch(tpe_ctx* ctx, const double* xyz, int32_t ncurves, const tpe_params* p,
                         int32_t precision, double* energies);

/* ---- allocation-free energy (no counterpart in the reference) --------------- */
/* calculateEnergy for callers that cannot call cudaMalloc: an application whose
 * device memory all comes from its own allocator or pool, or a real-time loop
 * that must never enter the driver's allocator (cudaMalloc/cudaFree can
 * synchronise the device). d_xyz (V x 3 FP64) and d_edges (E x 2 int32) are
 * device pointers on the current device, d_energy receives one double there;
 * `stream` is a cudaStream_t (NULL = the legacy default stream). No context is
 * created and nothing is allocated: the scratch is a static device array of
 * about 1 MiB that every GPU loading the library holds until exit, so E is
 * limited to 16384 (larger E returns TPE_ERR_TOO_LARGE before any launch).
 * Edge indices must lie in [0, V): they are checked on the device, and an
 * index outside that range leaves the curve's energy NaN (no access outside
 * d_xyz). The first call on a device looks up the scratch's device address
 * (cudaGetSymbolAddress) and keeps it for the life of the process, so make that
 * first call before any stream capture, and do not use this entry point across
 * a cudaDeviceReset. All calls share the one scratch array: calls that overlap
 * on the GPU (different streams, or different host threads) race; serialise
 * them. A CUDA error left pending by the caller's earlier launches is reported
 * as TPE_ERR_CUDA (and cleared) by this call. */
int32_t tpe_energy_noalloc(const double* d_xyz, const int32_t* d_edges, int32_t V, int32_t E,
                           const tpe_params* p, double* d_energy, void* stream);

/* ---- device-resident step and instrumentation (extensions) ------------------ */
/* sobolevStepSet with the vertices already in device memory (d_xyz, d_xyz_out
 * are V x 3 device pointers on this context's device); for callers that keep
 * the curve resident between steps. Same semantics as tpe_sobolev_step. */
int32_t tpe_sobolev_step_device(tpe_ctx* ctx, const double* d_xyz, const tpe_constraint* set,
                                int32_t nblocks, const tpe_step_opts* opts, double* d_xyz_out,
                                tpe_step_stats* stats, double* timings);
/* The dense FP64 product the large-constraint-set solve is built from, exposed
 * for checking and timing (no counterpart in the reference, whose dense algebra
 * is scalar JavaScript): C = alpha * A * B^T + beta * C with row-major device
 * matrices A (M x K, row stride lda), B (N x K, ldb), C (M x N, ldc) on this
 * context's device and stream. method TPE_GEMM_FP64 runs on the FP64 tensor
 * cores; TPE_GEMM_INT8_EMULATED cuts each row into eight 8-bit digits under a
 * power-of-two row scale and forms the exact integer digit products on the
 * int8 tensor cores (FP64-class accuracy: error within a few units of 2^-53
 * of max_k |A[i][k]| * max_k |B[j][k]| per term). mode: bit 0 only output
 * tiles on or below the diagonal (M == N), bit 1/2 A upper/lower triangular
 * (the K range skips its zeros), bits 3/4 the same for B and bit 5 writes only
 * elements with column <= row (bits 3-5 with the integer method only). */
enum { TPE_GEMM_FP64 = 0, TPE_GEMM_INT8_EMULATED = 1 };
int32_t tpe_gemm_nt_device(tpe_ctx* ctx, int32_t method, int32_t M, int32_t N, int32_t K,
                           const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                           int64_t ldc, double alpha, double beta, int32_t mode);
/* The CUDA stream (cudaStream_t) every launch of this context is issued on. */
void* tpe_stream(tpe_ctx* ctx);
/* Kernel groups timed with CUDA events on that stream while profiling is on. */
enum {
    TPE_KGROUP_ENERGY = 0, TPE_KGROUP_GRADIENT, TPE_KGROUP_PAIR_WEIGHTS, TPE_KGROUP_GATHER_A,
    TPE_KGROUP_CHOLESKY, TPE_KGROUP_TRSV, TPE_KGROUP_OTHER, TPE_KGROUP_COUNT
};
/* on != 0 resets and starts event timing; 0 stops it. */
int32_t tpe_profile(tpe_ctx* ctx, int32_t on);
/* Per group: total milliseconds and kernel launches since tpe_profile(ctx, 1);
 * launches[TPE_KGROUP_COUNT] also counts every kernel this context launched. */
int32_t tpe_profile_read(tpe_ctx* ctx, double* ms, int64_t* launches);

#ifdef __cplusplus
}
#endif
#endif /* TPE_H */
