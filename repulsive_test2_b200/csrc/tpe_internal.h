// Internal declarations of libtpe: the context, device buffers and the
// launchers each .cu file provides. Not part of the ABI (include/tpe.h is).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tpe.h"
#include "tc.h"

#define TPE_CUDA_TRY(expr)                                                              \
    do {                                                                                \
        cudaError_t _e = (expr);                                                        \
        if (_e != cudaSuccess) {                                                        \
            tpe::set_error(ctx, TPE_ERR_CUDA, std::string(#expr) + ": " +               \
                                                  cudaGetErrorString(_e));              \
            return TPE_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)

#define TPE_TRY(expr)                       \
    do {                                    \
        int32_t _s = (expr);                \
        if (_s != TPE_OK) return _s;        \
    } while (0)

namespace tpe {

// A grow-only device allocation owned by the context.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    template <class T>
    T* as() const { return static_cast<T*>(ptr); }
};

// Dense Cholesky block size (diagonal blocks are factored by one CTA).
constexpr int kNB = 64;
// Most right-hand sides (3 per constraint row, +3 for b) the mixed solve takes
// at factor time; larger sets use the FP64 factorization.
constexpr int kMixedMaxRhs = 48;
// Most step sizes one batched line-search launch projects together.
constexpr int kMaxTrials = 16;

// Everything the structured saddle solve keeps between the factorization and
// later solves: the frozen operator of optimizer.ts's 'frozen' projection.
struct SaddleOp {
    bool valid = false;
    int V = 0, k = 0;
    bool trans_constrained = false;  // set contains a barycenter or point block
    bool mixed = false;              // solves use the FP32 factor + FP64 CG (mixed.cu)
    bool mixed_fallback = false;     // mixed requested, FP64 factorization used instead
    int refine_iters = 0;            // CG iterations of the factor-time solve
    int refine_max_iter = 60;
    double refine_tol = 1e-12;
    double rho = 0.0;                // A_rho = A + (rho/V) 1 1^T
    // device (views into ctx buffers)
    double* A = nullptr;     // V x V original A (unfactored, for residuals)
    double* L = nullptr;     // V x V Cholesky factor of A_rho (lower, row-major)
    double* Linv = nullptr;  // nb x 64 x 64 inverses of the diagonal blocks of L
    double* C = nullptr;     // k x 3V dense constraint Jacobian
    double* Y = nullptr;     // k x 3V: Abar_rho^{-1} C^T (row s = column s of C^T)
    double* W = nullptr;     // 3V: Abar_rho^{-1} b for the b given at factor time (row k of Y)
    const double* w_src = nullptr;  // that b (device), or null
    // large constraint sets (schur.cu): explicit inverses on the device
    bool large = false;
    double* Ainv = nullptr;  // V x V: A_rho^{-1}
    double* Sinv = nullptr;  // k x k: (C A3^{-1} C^T)^{-1}
    bool int8 = false;       // both inverses with their products on the int8 tensor cores
    double chol_tol = 0.0;   // pivot tolerance of A_rho's Cholesky
    // host: small Schur complement and its factors
    std::vector<double> Scc;   // k x k, then its Cholesky factor (lower)
    std::vector<double> Scu;   // k x 3 = C U / rho
    std::vector<double> M;     // 3 x 3 = Scu^T Scc^{-1} Scu, then its Cholesky factor
};

// FP32 tensor-core factor of the Jacobi-scaled A_rho (mixed.cu): S ~ L L^T,
// Z = L^{-1}, W = Z^T, all Vp x Vp split-FP32; T is the TRTRI scratch.
struct MixedFactor {
    bool valid = false;
    int V = 0, Vp = 0;
    double rho = 0.0;
    tc::SplitMat L, Z, W, T, T2;  // T: level scratch; T2: the top level's T^T
    tc::SplitMat Zf;              // plain FP32 view of the CG's copy of Z
    tc::SplitMat S;  // plain FP32 trailing matrix (hi only)
};

struct DevBlock {
    int32_t kind;
    int32_t row0;
    int32_t vertex;
    int32_t rows;
    double target[3];
    double L0;
    const double* ell0;  // device copy, E entries (NaN where the host array ended)
};

}  // namespace tpe

struct tpe_ctx {
    // Held by every entry point for the whole call (tpe::guarded): calls on one
    // context from several host threads run one after another. Recursive, so an
    // entry point may call another on the same context.
    std::recursive_mutex mu;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;           // look-ahead stream of the factorization
    cudaStream_t stream3 = nullptr;           // the gradient, concurrent with assembly + factor
    cudaStream_t stream4 = nullptr;           // first half of the mixed inverse, beside the factor
    cudaStream_t stream5 = nullptr;           // panel remainders of the mixed factor (high priority)
    cudaEvent_t ev_prep = nullptr, ev_grad = nullptr;
    // a gradient launched on stream3 and not yet joined (step_impl / finish_gradient)
    bool grad_pending = false;
    bool grad_unlaunched = false;
    double grad_params[3] = {0, 0, 0};  // alpha, beta, eps
    const double* grad_pos = nullptr;
    double* grad_dE = nullptr;
    double* grad_flat = nullptr;
    const tpe_penalties* grad_pen = nullptr;
    // SMs the concurrent gradient may occupy; the rest stay free for the
    // factorization's chain of small launches (TPE_GRAD_SMS overrides)
    int32_t grad_sms = 0;
    // SMs the persistent trailing updates leave free for the chain's and the
    // panel's launches (TPE_FACTOR_FREE_SMS overrides)
    int32_t free_sms = 8;
    std::vector<cudaEvent_t> fac_events;      // dependency events (no timing)
    std::string err;
    int32_t num_sms = 0;

    // topology
    bool has_topology = false;
    int32_t V = 0, E = 0;
    // one closed loop with edge I = (I, I+1 mod V), V >= 8: Gram assembly by the
    // fused stencil kernel (assembly.cu)
    bool closed_loop = false;
    std::vector<int32_t> h_edges;     // 2E
    std::vector<int32_t> h_inc_off;   // V+1
    std::vector<int32_t> h_inc;       // 2E entries: edge*2 + slot, ascending edge order per vertex
    tpe::DevBuf d_edges, d_inc_off, d_inc;

    // per-evaluation buffers
    tpe::DevBuf pos, pos2, pos3, edge_a, edge_b, grad, edge_acc, partial, scalars, flat0, flat1,
        flat2, flat3, dir;
    tpe::DevBuf grad_ctr;  // tile counter of the SM-bounded gradient kernel
    // large constraint sets (schur.cu)
    tpe::DevBuf mat_Ainv, inv_X, inv_W, inv_T, sch_nz, sch_S, sch_L, sch_Linv, sch_Sinv, sch_vec;
    tpe::DevBuf ref_r, ref_x;  // residual and correction of the refinement step
    tpe::DevBuf oz_planes, oz_err;  // digit planes and timeout flag of ozaki_gemm_nt
    tpe::DevBuf oz_base;            // the FP64 base blocks of spd_inverse_int8
    tpe::DevBuf bh_buf;             // Barnes-Hut tree, permutation and per-edge sums (bh.cu)
    tpe::DevBuf ycomb_part;    // split-over-rows partial sums of Y^T coef
    tpe::DevBuf mx_ctr;    // tile counters of the persistent trailing updates
    tpe::DevBuf pairM;                      // E x E double2 (Mb, M0) pair matrix
    tpe::DevBuf edge_m;                     // mixed-precision edge records (4 float4 per edge)
    tpe::DevBuf mat_A, mat_L, mat_Linv, mat_B, mat_B0;
    tpe::DevBuf con_C, con_Y, con_phi, con_blocks, con_ell0, con_red;
    tpe::DevBuf con_part;  // split partial reductions of the constraint rows
    tpe::DevBuf rhs, sol, tmp, solve_scratch;
    tpe::DevBuf status;                     // device-side int flags
    tpe::DevBuf trial_raw, trial_cur;       // batched line-search trials (K x 3V each)
    tpe::SaddleOp op;
    // mixed-precision factor (mixed.cu)
    tpe::DevBuf mx_T2hi, mx_T2lo;
    tpe::DevBuf mx_d, mx_dinv, mx_S, mx_Lhi, mx_Llo, mx_Zhi, mx_Zlo, mx_Whi, mx_Wlo, mx_Thi, mx_Tlo,
        mx_vec, mx_part, mx_Zd, mx_Wd;
    tpe::MixedFactor mf;
    void* h_stage = nullptr;  // pinned staging of small device-to-host copies (download_many)
    size_t h_stage_bytes = 0;
    std::vector<double> h_tmp;

    // instrumentation: kernel launch count and per-group CUDA-event timing
    int64_t launches = 0;
    bool profiling = false;
    double prof_ms[TPE_KGROUP_COUNT] = {};
    int64_t prof_launches[TPE_KGROUP_COUNT + 1] = {};
    struct PendingEvent {
        int group;
        cudaEvent_t a, b;
    };
    std::vector<PendingEvent> prof_pending;
    std::vector<cudaEvent_t> prof_pool;
};

namespace tpe {

// Times the launches issued while in scope under `group` (when profiling) and
// counts them; `n` = number of kernels the scope launches.
struct KernelScope {
    tpe_ctx* ctx;
    int group;
    cudaEvent_t b = nullptr;
    KernelScope(tpe_ctx* c, int g, int64_t n);
    ~KernelScope();
};

void set_error(tpe_ctx* ctx, int32_t code, const std::string& msg);

// Runs the body of a C entry point under the context's mutex (when there is a
// context). A C++ exception (a failed host allocation, a thread that could not
// start, a mutex that could not be taken) becomes an error status, with the
// message in the context when there is one, instead of leaving through the C ABI.
template <class F>
int32_t guarded(tpe_ctx* ctx, F&& body) noexcept {
    int32_t code = TPE_ERR_INTERNAL;
    const char* msg = "unexpected host-side exception";
    try {
        std::unique_lock<std::recursive_mutex> lock;
        if (ctx) lock = std::unique_lock<std::recursive_mutex>(ctx->mu);
        return body();
    } catch (const std::bad_alloc&) {
        code = TPE_ERR_OUT_OF_MEMORY;
        msg = "host allocation failed";
    } catch (const std::length_error&) {
        code = TPE_ERR_TOO_LARGE;
        msg = "host buffer size out of range";
    } catch (const std::exception& e) {
        msg = e.what();
    } catch (...) {
    }
    try {
        set_error(ctx, code, msg);
    } catch (...) {
    }
    return code;
}
int32_t ensure(tpe_ctx* ctx, DevBuf& b, size_t bytes);

// Device-to-host copies through the context's pinned staging area: the copies
// are issued on `stream`, the stream is synchronized once, and the bytes are
// copied out on the host. Pageable copies from many host threads (the
// multi-curve batch) would queue in the driver's shared staging buffer.
struct HostCopy {
    void* host;
    const void* dev;
    size_t bytes;
};
int32_t download_many(tpe_ctx* ctx, cudaStream_t stream, const HostCopy* copies, int n);
inline int32_t download_on(tpe_ctx* ctx, cudaStream_t stream, void* host, const void* dev,
                           size_t bytes) {
    const HostCopy c{host, dev, bytes};
    return download_many(ctx, stream, &c, 1);
}

// ---- pair kernels (pair_kernels.cu) ----------------------------------------
// Per-edge records from interleaved positions: a = (p1, ell^eps), b = (p2, |e|).
int32_t edge_prep(tpe_ctx* ctx, const double* d_pos, int32_t ncurves, double eps,
                  double alpha);
// Energy of ncurves position sets (edge records already prepared) into
// d_energy[ncurves] (device).
int32_t energy_fp64(tpe_ctx* ctx, int32_t ncurves, double alpha, double beta, double eps,
                    double* d_energy);
// Energy of one curve with caller-provided scratch and stream (no context);
// edge indices are checked on the device (*bad set, energy NaN).
int32_t energy_fp64_scratch(cudaStream_t stream, const double* d_pos, const int2* d_edges,
                            int32_t V, int32_t E, double alpha, double beta, double eps,
                            double4* ea, double4* eb, double* partial, int32_t max_parts,
                            int32_t* bad, double* d_energy);
// Energy (optional) and gradient (interleaved V x 3) of one curve. max_blocks > 0
// bounds the SMs the pair kernel occupies (one block per SM).
int32_t energy_grad_fp64(tpe_ctx* ctx, double alpha, double beta, double eps, double* d_energy,
                         double* d_grad, int32_t max_blocks = 0);

// Barnes-Hut energy (bh.cu) of this context's curve: h_xyz (host) builds the
// tree, d_xyz (device, the same positions) is traversed. stats (nullable):
// visits, approximated edge references, direct pairs.
int32_t bh_energy(tpe_ctx* ctx, const double* h_xyz, const double* d_xyz, double alpha, double beta,
                  double eps, double theta, double theta_t, int32_t leaf, double* energy,
                  int64_t* stats);

// phi = K psi (E x nr, nr = 1 or 3; host arrays) for the high (kind 0) or low
// (kind 1) edge kernel by the block cluster tree (bh.cu). stats (nullable, 4):
// block-tree leaves, admissible blocks, direct blocks, direct pairs.
int32_t bct_matvec(tpe_ctx* ctx, const double* h_xyz, const double* d_xyz, int32_t kind,
                   const double* h_psi, int32_t nr, double eps, double theta, double theta_t,
                   int32_t leaf, double* h_phi, int64_t* stats);

// ---- mixed precision energy (pair_mixed.cu) ----------------------------------
// FP32 pair terms, FP64 sums: tpe_energy_batch with TPE_PRECISION_MIXED only.
int32_t edge_prep_mixed(tpe_ctx* ctx, const double* d_pos, int32_t ncurves, double eps,
                        double alpha);
int32_t energy_mixed(tpe_ctx* ctx, int32_t ncurves, double alpha, double beta, double eps,
                     double* d_energy);

// ---- assembly (assembly.cu) -----------------------------------------------
// A (and optionally B, B0) V x V row-major FP64 from prepared edge records.
int32_t assemble_fp64(tpe_ctx* ctx, double alpha, double beta, double eps, double* d_A,
                      double* d_B, double* d_B0);

// ---- dense linear algebra (dense.cu) --------------------------------------
// In-place lower Cholesky of the V x V row-major matrix (lower triangle read);
// also writes the inverses of the 64x64 diagonal blocks. Sets *singular.
int32_t cholesky_fp64(tpe_ctx* ctx, double* d_L, double* d_Linv, int32_t n, double piv_tol,
                      int32_t* singular);
// Solves (L L^T) X = B in place for nrhs right-hand sides stored as B[nrhs][n].
int32_t chol_solve_fp64(tpe_ctx* ctx, const double* d_L, const double* d_Linv, int32_t n,
                        double* d_B, int32_t nrhs);
// out[i*ncols + j] = dot(X[i], Y[j]) over len (rows of length len): FP64, deterministic.
int32_t gram_dots(tpe_ctx* ctx, const double* X, int32_t nx, const double* Y, int32_t ny,
                  int64_t len, double* d_out);
// A_rho = A + shift (every entry) into L (lower triangle copied), and trace(A) into *d_trace.
int32_t shift_copy(tpe_ctx* ctx, const double* d_A, double* d_L, int32_t n, double shift);
// C = alpha A B^T + beta C, FP64 row-major, on the FP64 tensor cores (dense.cu).
// kDBUpper, kDBLower (B[j][k] = 0 for k < j, k > j) and kDMaskUpper (write only
// elements with column <= row) are for ozaki_gemm_nt only.
enum : int32_t {
    kDLowerTiles = 1, kDAUpper = 2, kDALower = 4, kDBUpper = 8, kDBLower = 16, kDMaskUpper = 32
};
struct DGemmArgs {
    const double* A = nullptr;
    int64_t lda = 0;
    const double* B = nullptr;
    int64_t ldb = 0;
    double* C = nullptr;
    int64_t ldc = 0;
    int32_t M = 0, N = 0, K = 0;
    double alpha = 1.0, beta = 0.0;
    int32_t mode = 0;
};
int32_t dgemm_nt(tpe_ctx* ctx, const DGemmArgs& g, cudaStream_t stream);
// The same product on the integer tensor cores (ozaki.cu): each operand row cut
// into eight 8-bit digits under a power-of-two row scale, the digit products
// exact int32 GEMMs, summed in FP64: FP64-class accuracy. Scratch: ctx->oz_planes
// (ozaki_scratch_bytes); calls on one context must share one stream. A pipeline
// timeout sets a device flag that ozaki_status reads (and clears).
size_t ozaki_scratch_bytes(int32_t M, int32_t N, int32_t K);
int32_t ozaki_reserve(tpe_ctx* ctx, size_t bytes);
int32_t ozaki_gemm_nt(tpe_ctx* ctx, const DGemmArgs& g, cudaStream_t stream,
                      int group = TPE_KGROUP_TRSV);
int32_t ozaki_status(tpe_ctx* ctx, cudaStream_t stream);
// out = (L L^T)^{-1}, n x n symmetric, from the Cholesky factor and its 64x64
// diagonal-block inverses (cholesky_fp64); X, W (n x n) and Tt ((n/2 + 64)^2)
// are scratch. X = L^{-1} by recursive halving, then out = X^T X.
int32_t spd_inverse_fp64(tpe_ctx* ctx, const double* d_L, const double* d_Linv, int32_t n,
                         double* X, double* W, double* Tt, double* out);
// X = L^{-1} (lower) and W = X^T (upper), n x n, from the Cholesky factor and its
// 64x64 diagonal-block inverses (the first half of spd_inverse_fp64).
int32_t lower_inverse_fp64(tpe_ctx* ctx, const double* d_L, const double* d_Linv, int32_t n,
                           double* X, double* W, double* Tt);
// M[j][i] = M[i][j] for j > i (n x n, row-major).
int32_t mirror_lower(tpe_ctx* ctx, double* M, int32_t n);
// dst[j][i] = src[i][j] for an m x c block (row strides lds, ldd).
int32_t transpose_fp64(tpe_ctx* ctx, const double* src, int64_t lds, int32_t m, int32_t c,
                       double* dst, int64_t ldd);
// out = A^{-1} for the SPD n x n matrix in Mat (lower triangle read; Mat is
// overwritten) with the heavy products on the integer tensor cores
// (ozaki_gemm_nt): recursive Cholesky and triangular inverse in halves down to
// blocks of at most 1024 (cholesky_fp64 + lower_inverse_fp64 there), then
// out = X^T X. X, W (n x n) and Tt ((n/2 + 64)^2) are scratch. A pivot at or
// below piv_tol sets *singular.
int32_t spd_inverse_int8(tpe_ctx* ctx, double* Mat, int32_t n, double piv_tol, double* X,
                         double* W, double* Tt, double* out, bool* singular);
// Y[c][i] = sum_j M[i][j] X[c][j] for c < nr <= 16: M n x n FP64 (row length n),
// X and Y nr rows of stride ldx >= n (mixed.cu: the CG's multi-RHS kernel).
int32_t mrhs_fp64(tpe_ctx* ctx, const double* M, int32_t n, const double* X, int32_t ldx,
                  int32_t nr, double* Y);
int32_t trace(tpe_ctx* ctx, const double* d_A, int32_t n, double* d_out);

// ---- mixed-precision solve (mixed.cu) ------------------------------------
int32_t mixed_padded_size(int32_t V);
// FP32 tensor-core factor + inverse of the Jacobi-scaled A_rho = A + (rho/V) 1 1^T
// into ctx->mf; *ok = false when the FP32 factorization broke down.
int32_t mixed_factor(tpe_ctx* ctx, const double* d_A, int32_t V, double rho, bool* ok);
// A_rho X = B for nr right-hand sides ([nr][V], FP64, may alias) by CG with the
// FP32 factor as preconditioner, to ||B - A_rho X|| <= tol ||B|| per column.
int32_t mixed_solve(tpe_ctx* ctx, const double* d_A, const double* d_B, double* d_X, int32_t nr,
                    int32_t maxit, double tol, int32_t* iters, bool* converged);

// ---- large constraint sets (schur.cu) ----------------------------------------
// Constraint sets with more rows than this take the explicit-inverse Schur path.
constexpr int32_t kLargeSchur = 64;
// Iterative refinement of the large-set gradient solve: stop at this relative
// saddle residual, or after kLargeRefineMax corrections, or when a correction
// no longer halves the residual.
constexpr double kRefineStop = 1e-13;
constexpr int32_t kLargeRefineMax = 4;
// The refined gradient-solve residual the int8-tensor-core inverses must reach;
// above it the step rebuilds them in FP64. The FP64 inverses reach 1e-14 after
// one or two corrections on every measured curve; the int8 ones either do the
// same or stall far above this (rows whose entries span many orders of
// magnitude lose digits under a per-row scale).
constexpr double kInt8ResidualGate = 1e-12;
// From the FP64 factor op.L: op.Ainv, op.Y (k x 3V), op.W = A3^{-1} b when b is
// given, and op.Sinv; *singular when the Schur complement is not SPD.
int32_t large_schur_build(tpe_ctx* ctx, SaddleOp& op, const double* b_flat, bool* singular);
// out[c] = Sinv rc[c] for nr host vectors of length k (host in and out).
int32_t large_schur_apply(tpe_ctx* ctx, const SaddleOp& op, const double* rc, int32_t nr,
                          double* out);
// Joins the gradient running on stream3 (api.cu).
int32_t finish_gradient(tpe_ctx* ctx);

// ---- constraints (constraints.cu) -----------------------------------------
// Upload the set, returns k (stacked rows).
int32_t upload_set(tpe_ctx* ctx, const tpe_constraint* set, int32_t nblocks, int32_t* k);
// Phi (k) and per-block {norm^2, scale} (2*nblocks) into host arrays; dense C
// (k x 3V, device) when d_C != nullptr.
int32_t eval_constraints(tpe_ctx* ctx, const double* d_pos, int32_t nblocks, int32_t k,
                         double* d_C, std::vector<double>& phi, std::vector<double>& norm_scale);

// Phi (d_phi: n x k) and per-block {norm^2, scale} (d_ns: n x 2 nblocks), on the
// device, for the position sets pos + idx[q] * stride, q < n (idx on the device).
int32_t eval_constraints_batch(tpe_ctx* ctx, const double* d_pos, int64_t stride,
                               const int32_t* d_idx, int32_t n, int32_t nblocks, int32_t k,
                               double* d_phi, double* d_ns);

// ---- small device helpers (dense.cu) --------------------------------------
int32_t interleaved_to_block(tpe_ctx* ctx, const double* d_v3, double* d_flat, int32_t V);
int32_t block_to_interleaved(tpe_ctx* ctx, const double* d_flat, double* d_v3, int32_t V);
// y = a*x + b*y (n)
int32_t axpby(tpe_ctx* ctx, int64_t n, double a, const double* x, double b, double* y);
// host result: sum(x*y) over n (deterministic)
int32_t dot(tpe_ctx* ctx, int64_t n, const double* x, const double* y, double* out);
// host result: number of non-finite entries in x[n]
int32_t count_nonfinite(tpe_ctx* ctx, int64_t n, const double* x, int64_t* out);
// l2CurveNorm of interleaved values at interleaved positions (host result)
int32_t l2_curve_norm(tpe_ctx* ctx, const double* d_vals, const double* d_pos, double* out);
// x_flat(3V) = w - sum_s Y[s] * lam[s] - U mu / rho ; lam/mu are host arrays
int32_t combine_solution(tpe_ctx* ctx, const double* d_w, const double* d_Y, int32_t k,
                         const double* lam, const double* mu, double rho, int32_t V, double* d_x);
// cur[idx[q]] (interleaved, rows stride apart) += -Y^T coef[q] - mu term for nu <= 16
// device coefficient vectors (k + 3 each), with combine_solution's sums.
int32_t project_update(tpe_ctx* ctx, const double* d_Y, int32_t k, int32_t V, const double* d_coef,
                       int32_t nu, const int32_t* d_idx, double* d_cur, int64_t stride,
                       int32_t* d_bad);
// Structured residual ||K z - rhs|| / max(1, ||rhs||) with A (V x V), C (k x 3V);
// optionally the residual vector rhs - K z itself: top (device, 3V) and bottom
// (host, k).
int32_t saddle_residual(tpe_ctx* ctx, const double* d_A, int32_t V, const double* d_C, int32_t k,
                        const double* d_x, const double* lam, const double* d_rhs_top,
                        const double* rhs_bottom, double* out, double* d_res_top = nullptr,
                        double* res_bottom = nullptr);

}  // namespace tpe
