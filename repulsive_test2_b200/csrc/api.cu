// libtpe C ABI (include/tpe.h) and the host orchestration of the step.
//
// The numerics run on the device (pair_kernels.cu, assembly.cu, dense.cu,
// constraints.cu); this file sequences them the way the reference's
// sobolevStepSet (src/core/optimizer.ts:231-440), lineSearchStepSet and
// projectOntoConstraintSet (src/core/sobolev/lineSearch.ts:196-562) do, and
// reads back only scalars (energies, norms, constraint values) for the
// control flow. No entry point throws or aborts; every failure is a status.
//
// Structured saddle solve (replaces solveSaddleFromA, linsolve.ts:742-803).
// With U = diag(u,u,u), u = 1/sqrt(V) (the constants, the kernel of A) and
// A_rho = A + rho u u^T (SPD), Abar = Abar_rho - rho U U^T and
// [[Abar, C^T],[C, 0]] [x; lam] = [b; d] becomes, with mu = -rho U^T x,
//   x = w - Y lam - U mu / rho,   w = Abar_rho^{-1} b,  Y = Abar_rho^{-1} C^T,
//   [Scc Scu; Scu^T 0] [lam; mu] = [C w - d; U^T w],
//   Scc = C Y (SPD), Scu = C U / rho (exact, since A_rho^{-1} u = u / rho).
// When no block fixes translations (C U = 0: no barycenter or point block),
// mu = 0 gives the solution with no constant component. Every solve reports
// the reference's residual ||Kz - rhs|| / max(1, ||rhs||) computed in FP64
// against the unfactored A and C.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <vector>

#include "tpe_internal.h"
#include <cstring>

namespace tpe {

bool penalties_active(const tpe_penalties* p);
int32_t penalty_energy_dev(tpe_ctx* ctx, const double* d_pos, const tpe_penalties* p, double* out);
int32_t penalty_gradient_dev(tpe_ctx* ctx, const double* d_pos, const tpe_penalties* p,
                             double* d_grad, int accumulate);

void set_error(tpe_ctx* ctx, int32_t code, const std::string& msg) {
    (void)code;
    if (ctx) ctx->err = msg;
}

KernelScope::KernelScope(tpe_ctx* c, int g, int64_t n) : ctx(c), group(g) {
    ctx->launches += n;
    ctx->prof_launches[TPE_KGROUP_COUNT] += n;
    if (!ctx->profiling) return;
    ctx->prof_launches[g] += n;
    cudaEvent_t a;
    if (ctx->prof_pool.size() >= 2) {
        a = ctx->prof_pool.back();
        ctx->prof_pool.pop_back();
        b = ctx->prof_pool.back();
        ctx->prof_pool.pop_back();
    } else {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    cudaEventRecord(a, ctx->stream);
    ctx->prof_pending.push_back({g, a, b});
}

KernelScope::~KernelScope() {
    if (b) cudaEventRecord(b, ctx->stream);
}

int32_t download_many(tpe_ctx* ctx, cudaStream_t stream, const HostCopy* copies, int n) {
    size_t total = 0;
    for (int i = 0; i < n; i++) total += (copies[i].bytes + 15) / 16 * 16;
    if (total > ctx->h_stage_bytes) {
        TPE_CUDA_TRY(cudaStreamSynchronize(stream));
        if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
        ctx->h_stage = nullptr;
        ctx->h_stage_bytes = 0;
        const size_t want = std::max<size_t>(total + total / 4, 64 * 1024);
        TPE_CUDA_TRY(cudaMallocHost(&ctx->h_stage, want));
        ctx->h_stage_bytes = want;
    }
    unsigned char* stage = static_cast<unsigned char*>(ctx->h_stage);
    size_t off = 0;
    for (int i = 0; i < n; i++) {
        if (copies[i].bytes)
            TPE_CUDA_TRY(cudaMemcpyAsync(stage + off, copies[i].dev, copies[i].bytes,
                                         cudaMemcpyDeviceToHost, stream));
        off += (copies[i].bytes + 15) / 16 * 16;
    }
    TPE_CUDA_TRY(cudaStreamSynchronize(stream));
    off = 0;
    for (int i = 0; i < n; i++) {
        if (copies[i].bytes) memcpy(copies[i].host, stage + off, copies[i].bytes);
        off += (copies[i].bytes + 15) / 16 * 16;
    }
    return TPE_OK;
}

int32_t ensure(tpe_ctx* ctx, DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return TPE_OK;
    if (b.ptr) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    const size_t want = bytes + bytes / 8;
    cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e != cudaSuccess) {
        b.ptr = nullptr;
        set_error(ctx, TPE_ERR_OUT_OF_MEMORY,
                  std::string("cudaMalloc of ") + std::to_string(want) + " bytes failed: " +
                      cudaGetErrorString(e));
        cudaGetLastError();
        return TPE_ERR_OUT_OF_MEMORY;
    }
    b.bytes = want;
    return TPE_OK;
}

namespace {

struct Timer {
    double* t;
    int key;
    tpe_ctx* ctx;
    std::chrono::steady_clock::time_point t0;
    Timer(tpe_ctx* c, double* timings, int k) : t(timings), key(k), ctx(c) {
        if (t) {
            cudaStreamSynchronize(ctx->stream);
            t0 = std::chrono::steady_clock::now();
        }
    }
    ~Timer() {
        if (!t) return;
        cudaStreamSynchronize(ctx->stream);
        const double ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        t[2 * key] += ms;
        t[2 * key + 1] += 1.0;
    }
};

int32_t upload(tpe_ctx* ctx, DevBuf& b, const void* host, size_t bytes) {
    TPE_TRY(ensure(ctx, b, bytes));
    TPE_CUDA_TRY(cudaMemcpyAsync(b.ptr, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return TPE_OK;
}

int32_t download(tpe_ctx* ctx, void* host, const void* dev, size_t bytes) {
    return download_on(ctx, ctx->stream, host, dev, bytes);
}

bool all_finite(const double* a, size_t n) {
    for (size_t i = 0; i < n; i++)
        if (!isfinite(a[i])) return false;
    return true;
}

// Host dense Cholesky (lower, row-major) of a small SPD matrix; false if not SPD.
bool host_chol(std::vector<double>& a, int n) {
    for (int j = 0; j < n; j++) {
        double d = a[(size_t)j * n + j];
        for (int m = 0; m < j; m++) d -= a[(size_t)j * n + m] * a[(size_t)j * n + m];
        if (!(d > 0.0) || !isfinite(d)) return false;
        d = sqrt(d);
        a[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; i++) {
            double s = a[(size_t)i * n + j];
            for (int m = 0; m < j; m++) s -= a[(size_t)i * n + m] * a[(size_t)j * n + m];
            a[(size_t)i * n + j] = s / d;
        }
    }
    return true;
}

void host_chol_solve(const std::vector<double>& L, int n, std::vector<double>& b) {
    for (int i = 0; i < n; i++) {
        double s = b[i];
        for (int m = 0; m < i; m++) s -= L[(size_t)i * n + m] * b[m];
        b[i] = s / L[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = b[i];
        for (int m = i + 1; m < n; m++) s -= L[(size_t)m * n + i] * b[m];
        b[i] = s / L[(size_t)i * n + i];
    }
}

struct RowStats {
    std::vector<double> CU;  // k x 3: sum of C over each coordinate block (times 1/sqrt(V) later)
    double Cabs = 0.0;
};

__global__ void row_stats_kernel(const double* __restrict__ C, int32_t V,
                                 double* __restrict__ out) {
    __shared__ double red[4][8];
    const int32_t r = blockIdx.x;
    const double* row = C + (int64_t)r * 3 * V;
    double s[4] = {0, 0, 0, 0};
    for (int32_t i = threadIdx.x; i < V; i += blockDim.x) {
        const double a = row[i], b = row[V + i], c = row[2 * V + i];
        s[0] += a;
        s[1] += b;
        s[2] += c;
        s[3] += fabs(a) + fabs(b) + fabs(c);
    }
    for (int q = 0; q < 4; q++)
        for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_down_sync(0xffffffffu, s[q], o);
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 4; q++) red[q][threadIdx.x >> 5] = s[q];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; q++) {
            double t = 0;
            for (int w = 0; w < 8; w++) t += red[q][w];
            out[4 * r + q] = t;
        }
}

// Per vertex: 1 if row v of A is exactly zero and column (c, v) of C is zero for
// some coordinate c (an exactly zero row of K: the reference's zero pivot column).
__global__ void zero_row_kernel(const double* __restrict__ A, int32_t V,
                                const double* __restrict__ C, int32_t k,
                                int32_t* __restrict__ count) {
    const int32_t v = blockIdx.x;
    __shared__ int nz;
    if (threadIdx.x == 0) nz = 0;
    __syncthreads();
    for (int32_t j = threadIdx.x; j < V; j += blockDim.x)
        if (A[(int64_t)v * V + j] != 0.0) nz = 1;
    __syncthreads();
    if (threadIdx.x == 0 && !nz) {
        const int64_t m = 3 * (int64_t)V;
        for (int c = 0; c < 3; c++) {
            bool zero = true;
            for (int32_t r = 0; r < k; r++)
                if (C[(int64_t)r * m + (int64_t)c * V + v] != 0.0) zero = false;
            if (zero) {
                atomicAdd(count, 1);
                break;
            }
        }
    }
}

// out[0] = trace, out[1] = max |diagonal| (NaN if any is NaN), out[2] = number of
// exactly zero diagonal entries: the only candidates for a zero row, since an
// assembled A gets a positive diagonal term from every pair that touches a row.
__global__ void trace_max_kernel(const double* __restrict__ A, int32_t n, double* __restrict__ out) {
    __shared__ double rs[8], rm[8];
    __shared__ int zc;
    if (threadIdx.x == 0) zc = 0;
    __syncthreads();
    double s = 0.0, mx = 0.0;
    for (int32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double d = A[(int64_t)i * n + i];
        s += d;
        mx = (d != d || mx != mx) ? NAN : fmax(mx, fabs(d));
        if (d == 0.0) atomicAdd(&zc, 1);
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        const double w = __shfl_down_sync(0xffffffffu, mx, o);
        mx = (w != w || mx != mx) ? NAN : fmax(mx, w);
    }
    if ((threadIdx.x & 31) == 0) {
        rs[threadIdx.x >> 5] = s;
        rm[threadIdx.x >> 5] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int w = 0; w < 8; w++) {
            a += rs[w];
            b = (rm[w] != rm[w] || b != b) ? NAN : fmax(b, rm[w]);
        }
        out[0] = a;
        out[1] = b;
        out[2] = (double)zc;
    }
}

__global__ void add_flat_kernel(double* __restrict__ v3, const double* __restrict__ f, int32_t V) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    v3[3 * i] = v3[3 * i] + f[i];
    v3[3 * i + 1] = v3[3 * i + 1] + f[V + i];
    v3[3 * i + 2] = v3[3 * i + 2] + f[2 * V + i];
}

// raw[a] = p - tau[a] dir for the trials of one batch.
__global__ void step_batch_kernel(const double* __restrict__ p, const double* __restrict__ dir,
                                  const double* __restrict__ taus, int64_t n,
                                  double* __restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[(int64_t)blockIdx.y * n + t] = p[t] - taus[blockIdx.y] * dir[t];
}

// One projection correction for each active trial a = idx[y]: the Newton step
// x = -sum_s Y[s] lam_a[s] - mu_a[c] / (rho sqrt V) (the same operations, in the
// same order, as combine_kernel) added to the positions cur[a]; bad[a] = 1 when
// x has a non-finite entry (the trial is then abandoned).
__global__ void step_kernel(const double* __restrict__ p, const double* __restrict__ dir,
                            double tau, int64_t n, double* __restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = p[t] - tau * dir[t];
}

__global__ void div_kernel(const double* __restrict__ g, double s, int64_t n,
                           double* __restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = g[t] / s;
}

// FD: curve c perturbs coordinate (base + c) by h.
__global__ void fd_positions_kernel(const double* __restrict__ p, int64_t m, int64_t base,
                                    int32_t ncurves, double h, double* __restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m * ncurves) return;
    const int64_t c = t / m, i = t % m;
    double v = p[i];
    if (i == base + c) v += h;
    out[t] = v;
}

int32_t check_topology(tpe_ctx* ctx) {
    if (!ctx) return TPE_ERR_BAD_ARG;
    if (!ctx->has_topology) {
        set_error(ctx, TPE_ERR_NO_TOPOLOGY, "tpe_set_topology has not been called");
        return TPE_ERR_NO_TOPOLOGY;
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) {
        set_error(ctx, TPE_ERR_CUDA, cudaGetErrorString(e));
        return TPE_ERR_CUDA;
    }
    return TPE_OK;
}

}  // namespace

// ---- gradient on the side stream ---------------------------------------------

// Launches issued while in scope go to stream s (KernelScope events included).
struct StreamSwap {
    tpe_ctx* ctx;
    cudaStream_t saved;
    StreamSwap(tpe_ctx* c, cudaStream_t s) : ctx(c), saved(c->stream) { ctx->stream = s; }
    ~StreamSwap() { ctx->stream = saved; }
};

// Launches the gradient prepared by step_impl on stream3 (after the work the
// main stream has issued so far, i.e. after the assembly).
int32_t launch_gradient(tpe_ctx* ctx) {
    if (!ctx->grad_unlaunched) return TPE_OK;
    ctx->grad_unlaunched = false;
    TPE_CUDA_TRY(cudaEventRecord(ctx->ev_prep, ctx->stream));
    TPE_CUDA_TRY(cudaStreamWaitEvent(ctx->stream3, ctx->ev_prep, 0));
    {
        StreamSwap sw(ctx, ctx->stream3);
        TPE_TRY(energy_grad_fp64(ctx, ctx->grad_params[0], ctx->grad_params[1], ctx->grad_params[2],
                                 nullptr, ctx->grad_dE, ctx->grad_sms));
    }
    TPE_CUDA_TRY(cudaEventRecord(ctx->ev_grad, ctx->stream3));
    return TPE_OK;
}

// Joins the gradient launched on stream3 (step_impl) into the main stream and
// finishes the right-hand side: penalty gradient, coordinate-block layout.
int32_t finish_gradient(tpe_ctx* ctx) {
    if (!ctx->grad_pending) return TPE_OK;
    TPE_TRY(launch_gradient(ctx));
    ctx->grad_pending = false;
    TPE_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_grad, 0));
    if (ctx->grad_pen)
        TPE_TRY(penalty_gradient_dev(ctx, ctx->grad_pos, ctx->grad_pen, ctx->grad_dE, 1));
    return interleaved_to_block(ctx, ctx->grad_dE, ctx->grad_flat, ctx->V);
}

namespace {

// ---- saddle operator ----------------------------------------------------------

// Factor A_rho and the Schur complement from ctx->mat_A (V x V) and ctx->con_C (k x 3V).
// *singular set when the reference would report a singular system.
int32_t op_finalize(tpe_ctx* ctx, int32_t V, int32_t k, bool* singular,
                    const double* b_flat = nullptr, const tpe_step_opts* o = nullptr) {
    SaddleOp& op = ctx->op;
    op.valid = false;
    op.mixed = false;
    op.mixed_fallback = false;
    op.refine_iters = 0;
    op.refine_max_iter = o ? o->refine_max_iter : 60;
    op.refine_tol = o ? o->refine_tol : 1e-12;
    op.V = V;
    op.k = k;
    op.A = ctx->mat_A.as<double>();
    op.C = ctx->con_C.as<double>();
    op.W = nullptr;
    op.w_src = nullptr;
    op.large = false;
    op.int8 = false;
    op.Ainv = op.Sinv = nullptr;
    *singular = false;
    const int32_t nb = (V + kNB - 1) / kNB;
    TPE_TRY(ensure(ctx, ctx->mat_L, sizeof(double) * (size_t)V * V));
    TPE_TRY(ensure(ctx, ctx->mat_Linv, sizeof(double) * (size_t)nb * kNB * kNB));
    TPE_TRY(ensure(ctx, ctx->scalars, sizeof(double) * 600));
    op.L = ctx->mat_L.as<double>();
    op.Linv = ctx->mat_Linv.as<double>();
    double tm[3];
    { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    trace_max_kernel<<<1, 256, 0, ctx->stream>>>(op.A, V, ctx->scalars.as<double>() + 512); }
    TPE_CUDA_TRY(cudaGetLastError());
    TPE_TRY(download(ctx, tm, ctx->scalars.as<double>() + 512, sizeof(tm)));
    const double rho = tm[0] / V;
    if (!(rho > 0.0) || !isfinite(rho) || !isfinite(tm[1])) {
        *singular = true;
        return TPE_OK;
    }
    op.rho = rho;
    // exactly zero rows of K (only rows with a zero diagonal of A can be)
    if (tm[2] > 0.0) {
        TPE_TRY(ensure(ctx, ctx->status, sizeof(int32_t) * 4));
        TPE_CUDA_TRY(cudaMemsetAsync(ctx->status.as<int32_t>() + 1, 0, sizeof(int32_t), ctx->stream));
        { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
        zero_row_kernel<<<V, 256, 0, ctx->stream>>>(op.A, V, op.C, k, ctx->status.as<int32_t>() + 1); }
        TPE_CUDA_TRY(cudaGetLastError());
        int32_t zr = 0;
        TPE_TRY(download(ctx, &zr, ctx->status.as<int32_t>() + 1, sizeof(int32_t)));
        if (zr > 0) {
            *singular = true;
            return TPE_OK;
        }
    }
    // (large sets keep their Schur complement on the device: no k x k host array)
    op.Scc.assign(k > kLargeSchur ? 0 : (size_t)k * k, 0.0);
    op.Scu.assign((size_t)k * 3, 0.0);
    op.trans_constrained = false;
    // Y = Abar_rho^{-1} C^T (3k right-hand sides of length V) and, when given,
    // w = Abar_rho^{-1} b (3 more), solved together.
    const int32_t rows = k + (b_flat ? 1 : 0);
    TPE_TRY(ensure(ctx, ctx->con_Y, sizeof(double) * (size_t)(rows > 0 ? rows : 1) * 3 * V));
    op.Y = ctx->con_Y.as<double>();
    if (b_flat) {
        op.W = op.Y + (size_t)k * 3 * V;
        op.w_src = b_flat;
    }
    // the right-hand sides, loaded right before the solves (b may still be in
    // the making on another stream: finish_gradient joins it)
    auto load_rhs = [&]() -> int32_t {
        TPE_TRY(finish_gradient(ctx));
        if (k > 0)
            TPE_CUDA_TRY(cudaMemcpyAsync(op.Y, op.C, sizeof(double) * (size_t)k * 3 * V,
                                         cudaMemcpyDeviceToDevice, ctx->stream));
        if (b_flat)
            TPE_CUDA_TRY(cudaMemcpyAsync(op.W, b_flat, sizeof(double) * 3 * (size_t)V,
                                         cudaMemcpyDeviceToDevice, ctx->stream));
        return TPE_OK;
    };
    const int32_t nrhs = 3 * rows;
    if (o && o->precision == TPE_PRECISION_MIXED && nrhs <= kMixedMaxRhs) {
        // FP32 tensor-core factor as the preconditioner of an FP64 CG; the FP64
        // factorization below is the fallback (breakdown or no convergence).
        bool ok = false;
        TPE_TRY(mixed_factor(ctx, op.A, V, rho, &ok));
        if (ok && nrhs > 0) {
            bool conv = false;
            int32_t it = 0;
            TPE_TRY(load_rhs());
            TPE_TRY(mixed_solve(ctx, op.A, op.Y, op.Y, nrhs, o->refine_max_iter, o->refine_tol,
                                &it, &conv));
            op.refine_iters = it;
            ok = conv;
        }
        if (ok) {
            op.mixed = true;
        } else {
            op.mixed_fallback = true;
        }
    }
    if (!op.mixed) {
        TPE_TRY(shift_copy(ctx, op.A, op.L, V, rho / V));
        const double tol = 32.0 * 2.220446049250313e-16 * (tm[1] + rho / V);
        // mixed precision with a large set: the explicit inverses with their
        // products on the integer tensor cores (schur.cu), no FP64 factor here
        op.int8 = o && o->precision == TPE_PRECISION_MIXED && k > kLargeSchur &&
                  o->projection_mode == TPE_PROJECTION_FROZEN;
        op.chol_tol = tol;
        if (!op.int8) {
            int32_t bad = 0;
            TPE_TRY(cholesky_fp64(ctx, op.L, op.Linv, V, tol, &bad));
            if (bad) {
                *singular = true;
                return TPE_OK;
            }
        }
        if (k > kLargeSchur) {
            // explicit inverses, Y by gathers, the Schur complement on the device
            op.large = true;
            op.Scc.clear();
            bool sing = false;
            TPE_TRY(large_schur_build(ctx, op, b_flat, &sing));
            if (sing) {
                *singular = true;
                return TPE_OK;
            }
        } else {
            TPE_TRY(load_rhs());
            for (int32_t r0 = 0; r0 < nrhs; r0 += 64) {
                const int32_t nr = (nrhs - r0) < 64 ? (nrhs - r0) : 64;
                TPE_TRY(chol_solve_fp64(ctx, op.L, op.Linv, V, op.Y + (size_t)r0 * V, nr));
            }
        }
    }
    if (k > 0) {
        TPE_TRY(ensure(ctx, ctx->tmp, sizeof(double) * ((op.large ? 0 : (size_t)k * k) +
                                                         4 * (size_t)k + 16)));
        double* dS = ctx->tmp.as<double>();
        if (!op.large) TPE_TRY(gram_dots(ctx, op.C, k, op.Y, k, 3 * (int64_t)V, dS));
        double* dR = dS + (op.large ? 0 : (size_t)k * k);
        { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
        row_stats_kernel<<<k, 256, 0, ctx->stream>>>(op.C, V, dR); }
        TPE_CUDA_TRY(cudaGetLastError());
        std::vector<double> rs((size_t)4 * k);
        if (!op.large) TPE_TRY(download(ctx, op.Scc.data(), dS, sizeof(double) * (size_t)k * k));
        TPE_TRY(download(ctx, rs.data(), dR, sizeof(double) * 4 * (size_t)k));
        // symmetrise the Gram matrix (two sides of one dot product)
        if (!op.large)
            for (int32_t i = 0; i < k; i++)
                for (int32_t j = i + 1; j < k; j++) {
                    const double a = 0.5 * (op.Scc[(size_t)i * k + j] + op.Scc[(size_t)j * k + i]);
                    op.Scc[(size_t)i * k + j] = op.Scc[(size_t)j * k + i] = a;
                }
        const double su = 1.0 / sqrt((double)V);
        double cu_abs = 0.0, c_abs = 0.0;
        for (int32_t r = 0; r < k; r++) {
            for (int c = 0; c < 3; c++) {
                op.Scu[(size_t)r * 3 + c] = rs[4 * r + c] * su / rho;
                cu_abs += fabs(rs[4 * r + c]);
            }
            c_abs += rs[4 * r + 3];
        }
        if (!isfinite(c_abs)) {
            *singular = true;
            return TPE_OK;
        }
        if (!op.large && !host_chol(op.Scc, k)) {
            *singular = true;
            return TPE_OK;
        }
        op.trans_constrained = cu_abs > 1e-9 * c_abs;
        if (op.trans_constrained) {
            // M = Scu^T Scc^{-1} Scu (3 x 3 SPD)
            op.M.assign(9, 0.0);
            std::vector<std::vector<double>> Z(3, std::vector<double>((size_t)k));
            if (op.large) {
                std::vector<double> su3((size_t)3 * k), z3((size_t)3 * k);
                for (int c = 0; c < 3; c++)
                    for (int32_t r = 0; r < k; r++) su3[(size_t)c * k + r] = op.Scu[(size_t)r * 3 + c];
                TPE_TRY(large_schur_apply(ctx, op, su3.data(), 3, z3.data()));
                for (int c = 0; c < 3; c++)
                    Z[c].assign(z3.begin() + (size_t)c * k, z3.begin() + (size_t)(c + 1) * k);
            } else {
                for (int c = 0; c < 3; c++) {
                    for (int32_t r = 0; r < k; r++) Z[c][r] = op.Scu[(size_t)r * 3 + c];
                    host_chol_solve(op.Scc, k, Z[c]);
                }
            }
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    double s = 0;
                    for (int32_t r = 0; r < k; r++) s += op.Scu[(size_t)r * 3 + a] * Z[b][r];
                    op.M[a * 3 + b] = s;
                }
            for (int a = 0; a < 3; a++)
                for (int b = a + 1; b < 3; b++) {
                    const double s = 0.5 * (op.M[a * 3 + b] + op.M[b * 3 + a]);
                    op.M[a * 3 + b] = op.M[b * 3 + a] = s;
                }
            if (!host_chol(op.M, 3)) {
                *singular = true;
                return TPE_OK;
            }
        }
    }
    op.valid = true;
    return TPE_OK;
}

// Assemble A and C at device positions d_pos (set already uploaded) and factor.
// A is assembled in FP64 in every precision mode: rounding its entries to FP32
// moves the Sobolev gradient by far more than the mixed mode's tolerance.
int32_t op_build(tpe_ctx* ctx, const double* d_pos, int32_t nblocks, int32_t k, double alpha,
                 double beta, double eps, bool* singular, double* timings,
                 const double* b_flat = nullptr, const tpe_step_opts* o = nullptr) {
    const int32_t V = ctx->V;
    {
        Timer t(ctx, timings, TPE_PHASE_ASSEMBLEA);
        TPE_TRY(ensure(ctx, ctx->mat_A, sizeof(double) * (size_t)V * V));
        // the edge records of d_pos may already be in place (step_impl prepares
        // them once for the gradient, which reads them concurrently)
        if (!(ctx->grad_pending && ctx->grad_pos == d_pos)) TPE_TRY(edge_prep(ctx, d_pos, 1, eps, alpha));
        TPE_TRY(assemble_fp64(ctx, alpha, beta, eps, ctx->mat_A.as<double>(), nullptr, nullptr));
        TPE_TRY(launch_gradient(ctx));
    }
    TPE_TRY(ensure(ctx, ctx->con_C, sizeof(double) * (size_t)(k > 0 ? k : 1) * 3 * V));
    std::vector<double> phi, ns;
    TPE_TRY(eval_constraints(ctx, d_pos, nblocks, k, ctx->con_C.as<double>(), phi, ns));
    Timer t(ctx, timings, TPE_PHASE_FACTOR);
    return op_finalize(ctx, V, k, singular, b_flat, o);
}

// Multipliers of the bordered Schur system for the reduced right-hand side
// rc = C w - d (k) and ru = U^T w (3): lam (k) and mu (3).
int32_t schur_multipliers(tpe_ctx* ctx, const SaddleOp& op, const std::vector<double>& rc,
                          const double* ru, std::vector<double>& lam, double mu[3]) {
    const int32_t k = op.k;
    lam.assign((size_t)k, 0.0);
    mu[0] = mu[1] = mu[2] = 0.0;
    if (k == 0) return TPE_OK;
    auto scc_solve = [&](std::vector<double>& b) -> int32_t {
        if (op.large) {
            std::vector<double> in = b;
            return large_schur_apply(ctx, op, in.data(), 1, b.data());
        }
        host_chol_solve(op.Scc, k, b);
        return TPE_OK;
    };
    std::vector<double> t = rc;
    TPE_TRY(scc_solve(t));
    if (op.trans_constrained) {
        std::vector<double> rhs(3);
        for (int c = 0; c < 3; c++) {
            double s = 0;
            for (int32_t r = 0; r < k; r++) s += op.Scu[(size_t)r * 3 + c] * t[r];
            rhs[c] = s - ru[c];
        }
        host_chol_solve(op.M, 3, rhs);
        for (int c = 0; c < 3; c++) mu[c] = rhs[c];
        std::vector<double> r2 = rc;
        for (int32_t r = 0; r < k; r++)
            for (int c = 0; c < 3; c++) r2[r] -= op.Scu[(size_t)r * 3 + c] * mu[c];
        TPE_TRY(scc_solve(r2));
        lam = r2;
    } else {
        lam = t;
    }
    return TPE_OK;
}

// schur_multipliers for several reduced right-hand sides at once (the trials
// of a batched projection): with a large constraint set the Sinv products of
// all of them share one pass over Sinv; otherwise one host solve each.
int32_t schur_multipliers_multi(tpe_ctx* ctx, const SaddleOp& op,
                                const std::vector<std::vector<double>>& rcs, const double* ru,
                                std::vector<std::vector<double>>& lams,
                                std::vector<std::array<double, 3>>& mus) {
    const int32_t k = op.k, n = (int32_t)rcs.size();
    lams.assign((size_t)n, std::vector<double>((size_t)k, 0.0));
    mus.assign((size_t)n, {0.0, 0.0, 0.0});
    if (n == 0 || k == 0) return TPE_OK;
    if (!op.large) {
        for (int32_t q = 0; q < n; q++) TPE_TRY(schur_multipliers(ctx, op, rcs[q], ru, lams[q], mus[q].data()));
        return TPE_OK;
    }
    std::vector<double> in((size_t)n * k), t((size_t)n * k);
    for (int32_t q = 0; q < n; q++) std::copy(rcs[q].begin(), rcs[q].end(), in.begin() + (size_t)q * k);
    TPE_TRY(large_schur_apply(ctx, op, in.data(), n, t.data()));
    if (!op.trans_constrained) {
        for (int32_t q = 0; q < n; q++)
            std::copy(t.begin() + (size_t)q * k, t.begin() + (size_t)(q + 1) * k, lams[q].begin());
        return TPE_OK;
    }
    for (int32_t q = 0; q < n; q++) {
        const double* tq = t.data() + (size_t)q * k;
        std::vector<double> rhs(3);
        for (int c = 0; c < 3; c++) {
            double s = 0;
            for (int32_t r = 0; r < k; r++) s += op.Scu[(size_t)r * 3 + c] * tq[r];
            rhs[c] = s - ru[c];
        }
        host_chol_solve(op.M, 3, rhs);
        for (int c = 0; c < 3; c++) mus[q][c] = rhs[c];
        double* r2 = in.data() + (size_t)q * k;
        for (int32_t r = 0; r < k; r++)
            for (int c = 0; c < 3; c++) r2[r] -= op.Scu[(size_t)r * 3 + c] * mus[q][c];
    }
    TPE_TRY(large_schur_apply(ctx, op, in.data(), n, t.data()));
    for (int32_t q = 0; q < n; q++)
        std::copy(t.begin() + (size_t)q * k, t.begin() + (size_t)(q + 1) * k, lams[q].begin());
    return TPE_OK;
}

// One solve with the current operator: b_flat (device, 3V, or null = 0), d
// (host, k, or null = 0). x_flat (device) and lam (host) out.
int32_t op_solve_once(tpe_ctx* ctx, const double* b_flat, const double* d, double* x_flat,
                      std::vector<double>& lam) {
    SaddleOp& op = ctx->op;
    const int32_t V = op.V, k = op.k;
    const int64_t m = 3 * (int64_t)V;
    TPE_TRY(ensure(ctx, ctx->flat0, sizeof(double) * (size_t)m));
    double* w = ctx->flat0.as<double>();
    std::vector<double> rc((size_t)k, 0.0), ru(3, 0.0);
    if (b_flat) {
        if (op.W && op.w_src == b_flat) {
            w = op.W;  // solved together with Y at factor time
        } else {
            TPE_CUDA_TRY(cudaMemcpyAsync(w, b_flat, sizeof(double) * m, cudaMemcpyDeviceToDevice,
                                         ctx->stream));
            if (op.mixed) {
                bool conv = false;
                int32_t it = 0;
                TPE_TRY(mixed_solve(ctx, op.A, w, w, 3, op.refine_max_iter, op.refine_tol, &it,
                                    &conv));
                if (!conv) {
                    set_error(ctx, TPE_ERR_REFINE_NOT_CONVERGED,
                              "mixed-precision solve did not converge");
                    return TPE_ERR_REFINE_NOT_CONVERGED;
                }
            } else if (op.large) {
                TPE_TRY(mrhs_fp64(ctx, op.Ainv, V, b_flat, V, 3, w));
            } else {
                TPE_TRY(chol_solve_fp64(ctx, op.L, op.Linv, V, w, 3));
            }
        }
        if (k > 0) {
            TPE_TRY(ensure(ctx, ctx->tmp, sizeof(double) * ((size_t)k + 16)));
            TPE_TRY(gram_dots(ctx, op.C, k, w, 1, m, ctx->tmp.as<double>()));
            TPE_TRY(download(ctx, rc.data(), ctx->tmp.as<double>(), sizeof(double) * k));
        }
        if (op.trans_constrained) {
            const double su = 1.0 / sqrt((double)V);
            for (int c = 0; c < 3; c++) {
                double s = 0.0;
                TPE_TRY(dot(ctx, V, w + (size_t)c * V, nullptr, &s));
                ru[c] = s * su;
            }
        }
    }
    if (d)
        for (int32_t r = 0; r < k; r++) rc[r] -= d[r];
    double mu[3] = {0, 0, 0};
    TPE_TRY(schur_multipliers(ctx, op, rc, ru.data(), lam, mu));
    TPE_TRY(combine_solution(ctx, b_flat ? w : nullptr, op.Y, k, lam.data(), mu, op.rho, V,
                             x_flat));
    return TPE_OK;
}

// op_solve_once, and with a large constraint set (explicit inverses, accurate
// to about cond(A_rho) eps) one step of iterative refinement on the FP64
// residual; residual computed when non-null.
int32_t op_solve(tpe_ctx* ctx, const double* b_flat, const double* d, double* x_flat,
                 std::vector<double>& lam, double* residual) {
    SaddleOp& op = ctx->op;
    const int32_t V = op.V, k = op.k;
    const int64_t m = 3 * (int64_t)V;
    TPE_TRY(op_solve_once(ctx, b_flat, d, x_flat, lam));
    if (op.large && b_flat && k > 0) {
        // iterative refinement on the FP64 residual until it reaches kRefineStop,
        // stops shrinking by half, or kLargeRefineMax corrections are made
        TPE_TRY(ensure(ctx, ctx->ref_r, sizeof(double) * (size_t)m));
        TPE_TRY(ensure(ctx, ctx->ref_x, sizeof(double) * (size_t)m));
        double* rt = ctx->ref_r.as<double>();
        double* dx = ctx->ref_x.as<double>();
        std::vector<double> bottom((size_t)k, 0.0), rb((size_t)k, 0.0), dlam;
        if (d)
            for (int32_t r = 0; r < k; r++) bottom[r] = d[r];
        double prev = 0.0;
        for (int32_t it = 0;; it++) {
            double r0 = 0.0;
            TPE_TRY(saddle_residual(ctx, op.A, V, op.C, k, x_flat, lam.data(), b_flat, bottom.data(),
                                    &r0, rt, rb.data()));
            const bool done = it > 0 && (!(r0 > kRefineStop) || !(r0 < 0.5 * prev) ||
                                         it >= kLargeRefineMax);
            if (done) {
                if (residual) *residual = r0;
                return TPE_OK;
            }
            prev = r0;
            TPE_TRY(op_solve_once(ctx, rt, rb.data(), dx, dlam));
            TPE_TRY(axpby(ctx, m, 1.0, dx, 1.0, x_flat));
            for (int32_t r = 0; r < k; r++) lam[r] += dlam[r];
        }
    }
    if (residual) {
        const double* top = b_flat;
        if (!top) {
            double* z = ctx->flat0.as<double>();
            TPE_CUDA_TRY(cudaMemsetAsync(z, 0, sizeof(double) * m, ctx->stream));
            top = z;
        }
        std::vector<double> bottom((size_t)k, 0.0);
        if (d)
            for (int32_t r = 0; r < k; r++) bottom[r] = d[r];
        TPE_TRY(saddle_residual(ctx, op.A, V, op.C, k, x_flat, lam.data(), top, bottom.data(),
                                residual));
    }
    return TPE_OK;
}

// ---- energies -------------------------------------------------------------------

int32_t energy_of(tpe_ctx* ctx, const double* d_pos, double alpha, double beta, double eps,
                  double* out, int32_t precision = TPE_PRECISION_FP64) {
    TPE_TRY(ensure(ctx, ctx->scalars, sizeof(double) * 600));
    double* de = ctx->scalars.as<double>() + 520;
    if (precision == TPE_PRECISION_MIXED) {
        TPE_TRY(edge_prep_mixed(ctx, d_pos, 1, eps, alpha));
        TPE_TRY(energy_mixed(ctx, 1, alpha, beta, eps, de));
    } else {
        TPE_TRY(edge_prep(ctx, d_pos, 1, eps, alpha));
        TPE_TRY(energy_fp64(ctx, 1, alpha, beta, eps, de));
    }
    return download(ctx, out, de, sizeof(double));
}

int32_t objective(tpe_ctx* ctx, const double* d_pos, const tpe_step_opts* o, bool pen,
                  double* out, double* timings) {
    double e = 0.0;
    {
        Timer t(ctx, timings, TPE_PHASE_ENERGY);
        TPE_TRY(energy_of(ctx, d_pos, o->alpha, o->beta, o->epsilon, &e));
    }
    if (pen) {
        double pe = 0.0;
        TPE_TRY(penalty_energy_dev(ctx, d_pos, &o->penalties, &pe));
        e = e + pe;
    }
    *out = e;
    return TPE_OK;
}

int32_t gradient_fd_dev(tpe_ctx* ctx, const double* d_pos, double alpha, double beta, double eps,
                        double h, double* d_grad) {
    const int32_t V = ctx->V;
    const int64_t m = 3 * (int64_t)V;
    double e0 = 0.0;
    TPE_TRY(energy_of(ctx, d_pos, alpha, beta, eps, &e0));
    int32_t chunk = (int32_t)(((int64_t)1 << 27) / (m * 8));  // ~128 MB of positions per batch
    chunk = chunk < 1 ? 1 : (chunk > 512 ? 512 : chunk);
    TPE_TRY(ensure(ctx, ctx->pos3, sizeof(double) * (size_t)m * chunk));
    std::vector<double> e1((size_t)chunk), g((size_t)m);
    TPE_TRY(ensure(ctx, ctx->scalars, sizeof(double) * (600 + (size_t)chunk)));
    for (int64_t base = 0; base < m; base += chunk) {
        const int32_t nc = (int32_t)((m - base) < chunk ? (m - base) : chunk);
        { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
        fd_positions_kernel<<<(unsigned)((m * nc + 255) / 256), 256, 0, ctx->stream>>>(
            d_pos, m, base, nc, h, ctx->pos3.as<double>()); }
        TPE_CUDA_TRY(cudaGetLastError());
        TPE_TRY(edge_prep(ctx, ctx->pos3.as<double>(), nc, eps, alpha));
        double* de = ctx->scalars.as<double>() + 600;
        TPE_TRY(energy_fp64(ctx, nc, alpha, beta, eps, de));
        TPE_TRY(download(ctx, e1.data(), de, sizeof(double) * nc));
        for (int32_t c = 0; c < nc; c++) g[(size_t)(base + c)] = (e1[c] - e0) / h;
    }
    TPE_CUDA_TRY(cudaMemcpyAsync(d_grad, g.data(), sizeof(double) * m, cudaMemcpyHostToDevice,
                                 ctx->stream));
    TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return TPE_OK;
}

// ---- projection and line search -----------------------------------------------------

struct SetInfo {
    const tpe_constraint* set;
    int32_t nblocks;
    int32_t k;
};

inline double js_max(double a, double b) {
    if (a != a || b != b) return NAN;
    return a > b ? a : b;
}

// projectOntoConstraintSet. d_start is copied to d_cur. Frozen uses ctx->op as is.
int32_t project_dev(tpe_ctx* ctx, const double* d_start, const SetInfo& S, const tpe_step_opts* o,
                    bool frozen, double* d_cur, int32_t* ok, int32_t* iters, double* phi_norm,
                    double* timings) {
    const int32_t V = ctx->V;
    const int64_t m = 3 * (int64_t)V;
    TPE_CUDA_TRY(cudaMemcpyAsync(d_cur, d_start, sizeof(double) * m, cudaMemcpyDeviceToDevice,
                                 ctx->stream));
    TPE_TRY(ensure(ctx, ctx->flat1, sizeof(double) * (size_t)m));
    double* x = ctx->flat1.as<double>();
    double finalPhiNorm = INFINITY;
    *ok = 0;
    *iters = o->proj_max_iter;
    std::vector<double> phi, ns, lam;
    for (int32_t it = 0; it <= o->proj_max_iter; it++) {
        TPE_TRY(eval_constraints(ctx, d_cur, S.nblocks, S.k, nullptr, phi, ns));
        double sq = 0.0;
        for (double v : phi) sq += v * v;
        finalPhiNorm = sqrt(sq);
        bool converged = true;
        for (int32_t b = 0; b < S.nblocks; b++) {
            const double bn = sqrt(ns[2 * b]);
            const double tol = js_max(o->proj_tol_abs, o->proj_tol_rel * ns[2 * b + 1]);
            if (bn > tol) {
                converged = false;
                break;
            }
        }
        if (converged) {
            *ok = 1;
            *iters = it;
            break;
        }
        if (it == o->proj_max_iter) break;
        if (!all_finite(phi.data(), phi.size())) {  // the solve would throw: ok = false
            *iters = it;
            break;
        }
        if (!frozen) {
            bool singular = false;
            TPE_TRY(op_build(ctx, d_cur, S.nblocks, S.k, o->alpha, o->beta, o->epsilon, &singular,
                             timings, nullptr, o));
            if (singular) {
                *iters = it;
                break;
            }
        }
        std::vector<double> negphi(phi.size());
        for (size_t r = 0; r < phi.size(); r++) negphi[r] = -phi[r];
        {
            Timer t(ctx, timings, TPE_PHASE_SADDLE);
            TPE_TRY(op_solve(ctx, nullptr, negphi.data(), x, lam, nullptr));
        }
        int64_t bad = 0;
        TPE_TRY(count_nonfinite(ctx, m, x, &bad));
        if (bad) {
            *iters = it;
            break;
        }
        { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
        add_flat_kernel<<<(V + 255) / 256, 256, 0, ctx->stream>>>(d_cur, x, V); }
        TPE_CUDA_TRY(cudaGetLastError());
    }
    *phi_norm = finalPhiNorm;
    return TPE_OK;
}

// projectOntoConstraintSet (lineSearch.ts:196-295) in frozen mode for several
// start points at once: trial a starts at start[a] (ntrial x 3V) and ends in
// cur[a]. Each iteration evaluates Phi for every trial still running in one
// launch and applies all their Newton corrections in one launch; the per-trial
// decisions (converged, iteration cap, non-finite Phi, non-finite correction)
// and their order are those of project_dev.
int32_t project_batch_dev(tpe_ctx* ctx, const double* d_start, int32_t ntrial, const SetInfo& S,
                          const tpe_step_opts* o, double* d_cur, int32_t* ok, int32_t* iters,
                          double* phi_norm, double* timings) {
    const int32_t V = ctx->V, k = S.k, nb = S.nblocks;
    const int64_t m = 3 * (int64_t)V;
    const SaddleOp& op = ctx->op;
    TPE_CUDA_TRY(cudaMemcpyAsync(d_cur, d_start, sizeof(double) * m * ntrial,
                                 cudaMemcpyDeviceToDevice, ctx->stream));
    std::vector<int32_t> active;
    for (int32_t a = 0; a < ntrial; a++) {
        active.push_back(a);
        ok[a] = 0;
        iters[a] = o->proj_max_iter;
        phi_norm[a] = INFINITY;
    }
    TPE_TRY(ensure(ctx, ctx->status, sizeof(int32_t) * (4 + 2 * (size_t)ntrial)));
    int32_t* d_bad = ctx->status.as<int32_t>() + 4;
    int32_t* d_idx = d_bad + ntrial;
    TPE_CUDA_TRY(cudaMemsetAsync(d_bad, 0, sizeof(int32_t) * ntrial, ctx->stream));
    TPE_TRY(ensure(ctx, ctx->con_red, sizeof(double) * (size_t)ntrial * ((size_t)k + 2 * nb + k + 3)));
    double* d_phi = ctx->con_red.as<double>();
    double* d_ns = d_phi + (size_t)ntrial * k;
    double* d_coef = d_ns + (size_t)ntrial * 2 * nb;
    std::vector<double> phi((size_t)ntrial * k), ns((size_t)ntrial * 2 * nb);
    std::vector<int32_t> hbad(ntrial, 0);
    std::vector<double> coef;
    std::vector<std::vector<double>> rcs, lams;
    std::vector<std::array<double, 3>> mus;
    std::vector<int32_t> upd;
    const double ru[3] = {0.0, 0.0, 0.0};
    for (int32_t it = 0; it <= o->proj_max_iter && !active.empty(); it++) {
        const int32_t na = (int32_t)active.size();
        TPE_CUDA_TRY(cudaMemcpyAsync(d_idx, active.data(), sizeof(int32_t) * na,
                                     cudaMemcpyHostToDevice, ctx->stream));
        TPE_TRY(eval_constraints_batch(ctx, d_cur, m, d_idx, na, nb, k, d_phi, d_ns));
        {
            const HostCopy cp[3] = {{phi.data(), d_phi, k > 0 ? sizeof(double) * na * k : 0},
                                    {ns.data(), d_ns, sizeof(double) * na * 2 * nb},
                                    {hbad.data(), d_bad, sizeof(int32_t) * ntrial}};
            TPE_TRY(download_many(ctx, ctx->stream, cp, 3));
        }
        std::vector<int32_t> next;
        upd.clear();
        coef.clear();
        rcs.clear();
        for (int32_t q = 0; q < na; q++) {
            const int32_t a = active[q];
            if (it > 0 && hbad[a]) {  // last correction was not finite
                iters[a] = it - 1;
                continue;
            }
            const double* ph = phi.data() + (size_t)q * k;
            const double* nsq = ns.data() + (size_t)q * 2 * nb;
            double sq = 0.0;
            for (int32_t r = 0; r < k; r++) sq += ph[r] * ph[r];
            phi_norm[a] = sqrt(sq);
            bool converged = true;
            for (int32_t b = 0; b < nb; b++) {
                const double bn = sqrt(nsq[2 * b]);
                const double tol = js_max(o->proj_tol_abs, o->proj_tol_rel * nsq[2 * b + 1]);
                if (bn > tol) {
                    converged = false;
                    break;
                }
            }
            if (converged) {
                ok[a] = 1;
                iters[a] = it;
                continue;
            }
            if (it == o->proj_max_iter) continue;
            if (!all_finite(ph, (size_t)k)) {
                iters[a] = it;
                continue;
            }
            std::vector<double> rc((size_t)k);
            for (int32_t r = 0; r < k; r++) rc[r] = 0.0 - (-ph[r]);
            rcs.push_back(std::move(rc));
            upd.push_back(a);
            next.push_back(a);
        }
        active = next;
        if (upd.empty()) break;
        // the Newton multipliers of every trial corrected this iteration, together
        TPE_TRY(schur_multipliers_multi(ctx, op, rcs, ru, lams, mus));
        const double su = 1.0 / (op.rho * sqrt((double)V));
        for (size_t q = 0; q < upd.size(); q++) {
            for (int32_t r = 0; r < k; r++) coef.push_back(lams[q][r]);
            for (int c = 0; c < 3; c++) coef.push_back(mus[q][c] * su);
        }
        {
            Timer t(ctx, timings, TPE_PHASE_SADDLE);
            const int32_t nu = (int32_t)upd.size();
            TPE_CUDA_TRY(cudaMemcpyAsync(d_idx, upd.data(), sizeof(int32_t) * nu,
                                         cudaMemcpyHostToDevice, ctx->stream));
            TPE_CUDA_TRY(cudaMemcpyAsync(d_coef, coef.data(), sizeof(double) * coef.size(),
                                         cudaMemcpyHostToDevice, ctx->stream));
            // (copies from pageable host memory return once the data is staged,
            // so the host vectors may change after them without a synchronization)
            TPE_TRY(project_update(ctx, op.Y, k, V, d_coef, nu, d_idx, d_cur, m, d_bad));
        }
    }
    return TPE_OK;
}

void stats_reset(tpe_step_stats* st) {
    memset(st, 0, sizeof(*st));
    st->slope = NAN;
    st->projection_phi_norm = NAN;
    st->projection_iterations = -1;
    st->residual = NAN;
    st->gradient_l2_norm = NAN;
}

// lineSearchStepSet on device data: d_pos (gamma_0), d_dE, d_g (interleaved).
// The accepted (or echoed) vertices end in d_out.
int32_t line_search_dev(tpe_ctx* ctx, const double* d_pos, const double* d_dE, const double* d_g,
                        const SetInfo& S, const tpe_step_opts* o, bool frozen, double* d_out,
                        tpe_step_stats* st, double* timings) {
    Timer tls(ctx, timings, TPE_PHASE_LINESEARCH);
    const int32_t V = ctx->V;
    const int64_t m = 3 * (int64_t)V;
    const bool pen = o->has_penalties && penalties_active(&o->penalties);
    double e0 = 0.0;
    if (o->has_energy_before)
        e0 = o->energy_before;
    else
        TPE_TRY(objective(ctx, d_pos, o, pen, &e0, timings));
    st->energy_before = e0;
    st->energy = e0;
    st->tau = 0.0;
    st->accepted = 0;
    TPE_CUDA_TRY(cudaMemcpyAsync(d_out, d_pos, sizeof(double) * m, cudaMemcpyDeviceToDevice,
                                 ctx->stream));
    double gradNorm = 0.0;
    TPE_TRY(l2_curve_norm(ctx, d_g, d_pos, &gradNorm));
    if (!isfinite(gradNorm) || gradNorm <= 0) {
        st->reason = TPE_REASON_ZERO_OR_NONFINITE_GRADIENT_NORM;
        st->projection_iterations = 0;
        return TPE_OK;
    }
    st->gradient_l2_norm = gradNorm;
    TPE_TRY(ensure(ctx, ctx->dir, sizeof(double) * (size_t)m));
    double* dir = ctx->dir.as<double>();
    { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
    div_kernel<<<(unsigned)((m + 255) / 256), 256, 0, ctx->stream>>>(d_g, gradNorm, m, dir); }
    TPE_CUDA_TRY(cudaGetLastError());
    double slope = 0.0;
    TPE_TRY(dot(ctx, m, d_dE, dir, &slope));
    st->slope = slope;
    if (!isfinite(slope) || slope <= 0) {
        st->reason = TPE_REASON_NOT_A_DESCENT_DIRECTION;
        st->projection_iterations = 0;
        return TPE_OK;
    }
    TPE_TRY(ensure(ctx, ctx->pos3, sizeof(double) * (size_t)m));
    TPE_TRY(ensure(ctx, ctx->pos2, sizeof(double) * (size_t)m));
    double* raw = ctx->pos3.as<double>();
    double* cur = ctx->pos2.as<double>();
    double tau = o->tau0;
    int32_t lastReason = TPE_REASON_TAU_BELOW_MIN;
    int32_t trials = 0;
    if (frozen && o->trials > 1) {
        // Batched trials: the projections of up to o->trials step sizes run
        // together; the energies are then evaluated in the sequential order
        // (largest tau first) until one passes Armijo, so the accepted tau and
        // vertices are those of the one-at-a-time search.
        const int32_t K = o->trials < kMaxTrials ? o->trials : kMaxTrials;
        TPE_TRY(ensure(ctx, ctx->trial_raw, sizeof(double) * (size_t)m * K));
        TPE_TRY(ensure(ctx, ctx->trial_cur, sizeof(double) * (size_t)m * K));
        TPE_TRY(ensure(ctx, ctx->scalars, sizeof(double) * 600));
        double* d_taus = ctx->scalars.as<double>() + 560;
        double* braw = ctx->trial_raw.as<double>();
        double* bcur = ctx->trial_cur.as<double>();
        while (tau >= o->tau_min) {
            double taus[kMaxTrials];
            int32_t nk = 0;
            for (double t = tau; nk < K && t >= o->tau_min; t *= o->shrink) taus[nk++] = t;
            TPE_CUDA_TRY(cudaMemcpyAsync(d_taus, taus, sizeof(double) * nk, cudaMemcpyHostToDevice,
                                         ctx->stream));
            { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
            step_batch_kernel<<<dim3((unsigned)((m + 255) / 256), (unsigned)nk), 256, 0,
                                ctx->stream>>>(d_pos, dir, d_taus, m, braw); }
            TPE_CUDA_TRY(cudaGetLastError());
            int32_t okv[kMaxTrials], itv[kMaxTrials];
            double pnv[kMaxTrials];
            {
                Timer tp(ctx, timings, TPE_PHASE_PROJECTION);
                TPE_TRY(project_batch_dev(ctx, braw, nk, S, o, bcur, okv, itv, pnv, timings));
            }
            for (int32_t a = 0; a < nk; a++) {
                double* ca = bcur + (size_t)a * m;
                int64_t bad = 0;
                if (okv[a]) TPE_TRY(count_nonfinite(ctx, m, ca, &bad));
                if (okv[a] && !bad) {
                    double e1 = 0.0;
                    TPE_TRY(objective(ctx, ca, o, pen, &e1, timings));
                    trials++;
                    if (isfinite(e1) && e1 <= e0 - o->c1 * taus[a] * slope) {
                        st->accepted = 1;
                        st->reason = TPE_REASON_NONE;
                        st->tau = taus[a];
                        st->energy = e1;
                        st->projection_iterations = itv[a];
                        st->projection_phi_norm = pnv[a];
                        st->trials_evaluated = trials;
                        TPE_CUDA_TRY(cudaMemcpyAsync(d_out, ca, sizeof(double) * m,
                                                     cudaMemcpyDeviceToDevice, ctx->stream));
                        return TPE_OK;
                    }
                    lastReason = TPE_REASON_ARMIJO_FAILED;
                } else {
                    lastReason = TPE_REASON_PROJECTION_FAILED;
                }
            }
            tau = taus[nk - 1] * o->shrink;
        }
        st->reason = lastReason;
        st->trials_evaluated = trials;
        return TPE_OK;
    }
    while (tau >= o->tau_min) {
        { KernelScope ks(ctx, TPE_KGROUP_OTHER, 1);
        step_kernel<<<(unsigned)((m + 255) / 256), 256, 0, ctx->stream>>>(d_pos, dir, tau, m, raw); }
        TPE_CUDA_TRY(cudaGetLastError());
        int32_t ok = 0, iters = 0;
        double phiNorm = 0.0;
        {
            Timer tp(ctx, timings, TPE_PHASE_PROJECTION);
            TPE_TRY(project_dev(ctx, raw, S, o, frozen, cur, &ok, &iters, &phiNorm, timings));
        }
        int64_t bad = 0;
        TPE_TRY(count_nonfinite(ctx, m, cur, &bad));
        if (ok && !bad) {
            double e1 = 0.0;
            TPE_TRY(objective(ctx, cur, o, pen, &e1, timings));
            trials++;
            if (isfinite(e1) && e1 <= e0 - o->c1 * tau * slope) {
                st->accepted = 1;
                st->reason = TPE_REASON_NONE;
                st->tau = tau;
                st->energy = e1;
                st->projection_iterations = iters;
                st->projection_phi_norm = phiNorm;
                st->trials_evaluated = trials;
                TPE_CUDA_TRY(cudaMemcpyAsync(d_out, cur, sizeof(double) * m,
                                             cudaMemcpyDeviceToDevice, ctx->stream));
                return TPE_OK;
            }
            lastReason = TPE_REASON_ARMIJO_FAILED;
        } else {
            lastReason = TPE_REASON_PROJECTION_FAILED;
        }
        tau *= o->shrink;
    }
    st->reason = lastReason;
    st->trials_evaluated = trials;
    return TPE_OK;
}

int32_t validate_opts(tpe_ctx* ctx, const tpe_step_opts* o) {
    if (!o || o->struct_size != (int32_t)sizeof(tpe_step_opts)) {
        set_error(ctx, TPE_ERR_BAD_ARG,
                  "tpe_step_opts.struct_size mismatch (fill opts with tpe_default_step_opts)");
        return TPE_ERR_BAD_ARG;
    }
    return TPE_OK;
}

int32_t set_k(tpe_ctx* ctx, const tpe_constraint* set, int32_t nblocks, SetInfo* S) {
    if (nblocks < 0 || (nblocks > 0 && !set)) {
        set_error(ctx, TPE_ERR_BAD_ARG, "bad constraint set");
        return TPE_ERR_BAD_ARG;
    }
    S->set = set;
    S->nblocks = nblocks;
    return upload_set(ctx, set, nblocks, &S->k);
}

}  // namespace
}  // namespace tpe

using namespace tpe;

extern "C" {

int32_t tpe_abi_version(void) { return TPE_ABI_VERSION; }

void tpe_default_step_opts(tpe_step_opts* o) {
    if (!o) return;
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
    o->trials = 8;
    o->refine_max_iter = 60;
    o->refine_tol = 1e-12;
}

tpe_ctx* tpe_create(int32_t device, int32_t* status) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        if (status) *status = TPE_ERR_CUDA;
        return nullptr;
    }
    if (device < 0 || device >= n) {
        if (status) *status = TPE_ERR_BAD_ARG;
        return nullptr;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        if (status) *status = TPE_ERR_CUDA;
        return nullptr;
    }
    tpe_ctx* ctx = new (std::nothrow) tpe_ctx();
    if (!ctx) {
        if (status) *status = TPE_ERR_OUT_OF_MEMORY;
        return nullptr;
    }
    ctx->device = device;
    // The main stream carries the factorization's critical path: give it the
    // highest priority so its one-CTA kernels are dispatched ahead of everything
    // else; stream5 (the panel rests) one step below it, the trailing updates,
    // the gradient and the inverse's first half lowest.
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    const int prio_side = prio_hi < prio_lo ? prio_hi + 1 : prio_hi;
    if (cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->stream2, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->stream3, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->stream4, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->stream5, cudaStreamNonBlocking, prio_side) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_prep, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_grad, cudaEventDisableTiming) != cudaSuccess) {
        delete ctx;
        if (status) *status = TPE_ERR_CUDA;
        return nullptr;
    }
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    // the concurrent gradient's share: the factorization and the gradient end
    // together at V = 8192 (a sweep of 49, 53, 57, 61 SMs: 15.55, 15.08, 14.82,
    // 14.84 ms per step), and smaller curves factor relatively faster still
    ctx->grad_sms = ctx->num_sms * 2 / 5;
    if (const char* g = getenv("TPE_GRAD_SMS")) {
        const int n = atoi(g);
        if (n >= 0) ctx->grad_sms = n;  // 0: an ordinary grid over all SMs
    }
    // SMs the trailing updates leave to the factorization's other launches
    ctx->free_sms = 8;
    if (const char* g = getenv("TPE_FACTOR_FREE_SMS")) {
        const int n = atoi(g);
        if (n >= 0) ctx->free_sms = n;
    }
    if (status) *status = TPE_OK;
    return ctx;
}

void tpe_destroy(tpe_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->stream2) cudaStreamSynchronize(ctx->stream2);
    if (ctx->stream3) cudaStreamSynchronize(ctx->stream3);
    if (ctx->stream4) cudaStreamSynchronize(ctx->stream4);
    if (ctx->stream5) cudaStreamSynchronize(ctx->stream5);
    DevBuf* bufs[] = {&ctx->d_edges, &ctx->d_inc_off, &ctx->d_inc, &ctx->pos, &ctx->pos2,
                      &ctx->pos3, &ctx->edge_a, &ctx->edge_b, &ctx->grad, &ctx->edge_acc,
                      &ctx->partial, &ctx->scalars, &ctx->flat0, &ctx->flat1, &ctx->flat2,
                      &ctx->flat3, &ctx->dir, &ctx->pairM, &ctx->edge_m, &ctx->mat_A, &ctx->mat_L,
                      &ctx->mat_Linv, &ctx->mat_B, &ctx->mat_B0, &ctx->con_C, &ctx->con_Y,
                      &ctx->con_phi, &ctx->con_blocks, &ctx->con_ell0, &ctx->con_red, &ctx->con_part, &ctx->oz_planes, &ctx->oz_err, &ctx->oz_base, &ctx->bh_buf, &ctx->rhs,
                      &ctx->sol, &ctx->tmp, &ctx->solve_scratch, &ctx->status,
                      &ctx->trial_raw, &ctx->trial_cur, &ctx->mx_d, &ctx->mx_dinv, &ctx->mx_S,
                      &ctx->mx_Lhi, &ctx->mx_Llo, &ctx->mx_Zhi, &ctx->mx_Zlo, &ctx->mx_Whi,
                      &ctx->mx_Wlo, &ctx->mx_Thi, &ctx->mx_Tlo, &ctx->mx_T2hi, &ctx->mx_T2lo, &ctx->mx_vec, &ctx->mx_part,
                      &ctx->mx_Zd, &ctx->mx_Wd, &ctx->grad_ctr, &ctx->mx_ctr, &ctx->mat_Ainv,
                      &ctx->inv_X, &ctx->inv_W, &ctx->inv_T, &ctx->sch_nz, &ctx->sch_S,
                      &ctx->sch_L, &ctx->sch_Linv, &ctx->sch_Sinv, &ctx->sch_vec,
                      &ctx->ref_r, &ctx->ref_x, &ctx->ycomb_part};
    for (DevBuf* b : bufs)
        if (b->ptr) cudaFree(b->ptr);
    for (auto& p : ctx->prof_pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (cudaEvent_t e : ctx->prof_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->fac_events) cudaEventDestroy(e);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    if (ctx->ev_prep) cudaEventDestroy(ctx->ev_prep);
    if (ctx->ev_grad) cudaEventDestroy(ctx->ev_grad);
    if (ctx->stream5) cudaStreamDestroy(ctx->stream5);
    if (ctx->stream4) cudaStreamDestroy(ctx->stream4);
    if (ctx->stream3) cudaStreamDestroy(ctx->stream3);
    if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* tpe_last_error(const tpe_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int32_t tpe_set_topology(tpe_ctx* ctx, const int32_t* edges, int32_t E, int32_t V) {
    return guarded(ctx, [&]() -> int32_t {
        if (!ctx) return TPE_ERR_BAD_ARG;
        if (E < 0 || V < 0 || (E > 0 && !edges)) {
            set_error(ctx, TPE_ERR_BAD_ARG, "tpe_set_topology: bad sizes");
            return TPE_ERR_BAD_ARG;
        }
        for (int64_t i = 0; i < 2 * (int64_t)E; i++)
            if (edges[i] < 0 || edges[i] >= V) {
                set_error(ctx, TPE_ERR_BAD_ARG, "tpe_set_topology: edge index out of range");
                return TPE_ERR_BAD_ARG;
            }
        TPE_CUDA_TRY(cudaSetDevice(ctx->device));
        ctx->V = V;
        ctx->E = E;
        ctx->h_edges.assign(edges, edges + 2 * (size_t)E);
        ctx->closed_loop = E == V && V >= 8;
        for (int32_t I = 0; I < E && ctx->closed_loop; I++)
            ctx->closed_loop = edges[2 * I] == I && edges[2 * I + 1] == (I + 1 == V ? 0 : I + 1);
        ctx->h_inc_off.assign((size_t)V + 1, 0);
        for (int32_t I = 0; I < E; I++) {
            ctx->h_inc_off[edges[2 * I] + 1]++;
            ctx->h_inc_off[edges[2 * I + 1] + 1]++;
        }
        for (int32_t v = 0; v < V; v++) ctx->h_inc_off[v + 1] += ctx->h_inc_off[v];
        ctx->h_inc.assign(2 * (size_t)E, 0);
        std::vector<int32_t> fill(ctx->h_inc_off.begin(), ctx->h_inc_off.end() - 1);
        for (int32_t I = 0; I < E; I++)
            for (int s = 0; s < 2; s++) ctx->h_inc[fill[edges[2 * I + s]]++] = 2 * I + s;
        TPE_TRY(upload(ctx, ctx->d_edges, ctx->h_edges.data(), sizeof(int32_t) * 2 * (size_t)(E > 0 ? E : 1)));
        TPE_TRY(upload(ctx, ctx->d_inc_off, ctx->h_inc_off.data(), sizeof(int32_t) * ((size_t)V + 1)));
        TPE_TRY(upload(ctx, ctx->d_inc, ctx->h_inc.data(), sizeof(int32_t) * 2 * (size_t)(E > 0 ? E : 1)));
        TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        ctx->has_topology = true;
        ctx->op.valid = false;
        return TPE_OK;
    });
}

int32_t tpe_disjoint_pairs(tpe_ctx* ctx, int32_t* offsets, int32_t* partners, int64_t cap) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        const int32_t E = ctx->E;
        const int32_t* ed = ctx->h_edges.data();
        int64_t count = 0;
        for (int32_t i = 0; i < E; i++) {
            if (offsets) offsets[i] = (int32_t)count;
            for (int32_t j = 0; j < E; j++) {
                if (i == j) continue;
                const int32_t a1 = ed[2 * i], a2 = ed[2 * i + 1], b1 = ed[2 * j], b2 = ed[2 * j + 1];
                if (a1 != b1 && a1 != b2 && a2 != b1 && a2 != b2) {
                    if (partners && count < cap) partners[count] = j;
                    count++;
                }
            }
        }
        if (offsets) offsets[E] = (int32_t)count;
        if (partners && count > cap) {
            set_error(ctx, TPE_ERR_TOO_LARGE, "tpe_disjoint_pairs: partners capacity too small");
            return TPE_ERR_TOO_LARGE;
        }
        return TPE_OK;
    });
}

int32_t tpe_energy(tpe_ctx* ctx, const double* xyz, const tpe_params* p, double* energy) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        if (!xyz || !p || !energy) return TPE_ERR_BAD_ARG;
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * 3 * (size_t)ctx->V));
        return energy_of(ctx, ctx->pos.as<double>(), p->alpha, p->beta, p->epsilon, energy);
    });
}

int32_t tpe_energy_bh(tpe_ctx* ctx, const double* xyz, const tpe_params* p, double theta,
                      double theta_t, int32_t leaf_size, double* energy, int64_t* stats) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        if (!xyz || !p || !energy) return TPE_ERR_BAD_ARG;
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * 3 * (size_t)ctx->V));
        return bh_energy(ctx, xyz, ctx->pos.as<double>(), p->alpha, p->beta, p->epsilon, theta,
                         theta_t < 0.0 ? 1.5 * theta : theta_t, leaf_size, energy, stats);
    });
}

int32_t tpe_bct_matvec(tpe_ctx* ctx, const double* xyz, int32_t kind, const double* psi,
                       int32_t ncols, double epsilon, double theta, double theta_t,
                       int32_t leaf_size, double* phi, int64_t* stats) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        if (!xyz || !psi || !phi) return TPE_ERR_BAD_ARG;
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * 3 * (size_t)ctx->V));
        return bct_matvec(ctx, xyz, ctx->pos.as<double>(), kind, psi, ncols, epsilon, theta,
                          theta_t < 0.0 ? 1.5 * theta : theta_t, leaf_size, phi, stats);
    });
}

int32_t tpe_energy_grad(tpe_ctx* ctx, const double* xyz, const tpe_params* p, double* energy,
                        double* grad) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        if (!xyz || !p) return TPE_ERR_BAD_ARG;
        const int32_t V = ctx->V;
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * 3 * (size_t)V));
        TPE_TRY(ensure(ctx, ctx->grad, sizeof(double) * 3 * (size_t)(V > 0 ? V : 1)));
        TPE_TRY(ensure(ctx, ctx->scalars, sizeof(double) * 600));
        TPE_TRY(edge_prep(ctx, ctx->pos.as<double>(), 1, p->epsilon, p->alpha));
        double* de = ctx->scalars.as<double>() + 530;
        TPE_TRY(energy_grad_fp64(ctx, p->alpha, p->beta, p->epsilon, energy ? de : nullptr,
                                 grad ? ctx->grad.as<double>() : nullptr));
        if (grad) TPE_TRY(download(ctx, grad, ctx->grad.ptr, sizeof(double) * 3 * (size_t)V));
        if (energy) TPE_TRY(download(ctx, energy, de, sizeof(double)));
        return TPE_OK;
    });
}

int32_t tpe_gradient_fd(tpe_ctx* ctx, const double* xyz, const tpe_params* p, double h,
                        double* grad) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        if (!xyz || !p || !grad) return TPE_ERR_BAD_ARG;
        const int32_t V = ctx->V;
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * 3 * (size_t)V));
        TPE_TRY(ensure(ctx, ctx->grad, sizeof(double) * 3 * (size_t)V));
        TPE_TRY(gradient_fd_dev(ctx, ctx->pos.as<double>(), p->alpha, p->beta, p->epsilon, h,
                                ctx->grad.as<double>()));
        return download(ctx, grad, ctx->grad.ptr, sizeof(double) * 3 * (size_t)V);
    });
}

int32_t tpe_assemble(tpe_ctx* ctx, const double* xyz, const tpe_params* p, double* B_out,
                     double* B0_out, double* A_out) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        if (!xyz || !p) return TPE_ERR_BAD_ARG;
        const int32_t V = ctx->V;
        const size_t nn = (size_t)V * V;
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * 3 * (size_t)V));
        TPE_TRY(ensure(ctx, ctx->mat_A, sizeof(double) * nn));
        if (B_out) TPE_TRY(ensure(ctx, ctx->mat_B, sizeof(double) * nn));
        if (B0_out) TPE_TRY(ensure(ctx, ctx->mat_B0, sizeof(double) * nn));
        TPE_TRY(edge_prep(ctx, ctx->pos.as<double>(), 1, p->epsilon, p->alpha));
        TPE_TRY(assemble_fp64(ctx, p->alpha, p->beta, p->epsilon, ctx->mat_A.as<double>(),
                              B_out ? ctx->mat_B.as<double>() : nullptr,
                              B0_out ? ctx->mat_B0.as<double>() : nullptr));
        ctx->op.valid = false;
        if (A_out) TPE_TRY(download(ctx, A_out, ctx->mat_A.ptr, sizeof(double) * nn));
        if (B_out) TPE_TRY(download(ctx, B_out, ctx->mat_B.ptr, sizeof(double) * nn));
        if (B0_out) TPE_TRY(download(ctx, B0_out, ctx->mat_B0.ptr, sizeof(double) * nn));
        TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        return TPE_OK;
    });
}

int32_t tpe_constraint_rows(const tpe_ctx* ctx, const tpe_constraint* set, int32_t nblocks) {
    return guarded(nullptr, [&]() -> int32_t {
        if (!ctx || (nblocks > 0 && !set)) return -1;
        int32_t k = 0;
        for (int32_t b = 0; b < nblocks; b++) {
            switch (set[b].kind) {
                case TPE_BLOCK_BARYCENTER:
                case TPE_BLOCK_POINT: k += 3; break;
                case TPE_BLOCK_TOTAL_LENGTH: k += 1; break;
                case TPE_BLOCK_EDGE_LENGTHS: k += ctx->E; break;
                default: return -1;
            }
        }
        return k;
    });
}

int32_t tpe_evaluate_constraints(tpe_ctx* ctx, const double* xyz, const tpe_constraint* set,
                                 int32_t nblocks, double* phi, double* C) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        if (!xyz || !phi) return TPE_ERR_BAD_ARG;
        const int32_t V = ctx->V;
        SetInfo S;
        TPE_TRY(set_k(ctx, set, nblocks, &S));
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * 3 * (size_t)V));
        if (C) TPE_TRY(ensure(ctx, ctx->con_C, sizeof(double) * (size_t)(S.k > 0 ? S.k : 1) * 3 * V));
        std::vector<double> ph, ns;
        TPE_TRY(eval_constraints(ctx, ctx->pos.as<double>(), nblocks, S.k,
                                 C ? ctx->con_C.as<double>() : nullptr, ph, ns));
        ctx->op.valid = false;
        if (S.k > 0) memcpy(phi, ph.data(), sizeof(double) * S.k);
        if (C && S.k > 0)
            TPE_TRY(download(ctx, C, ctx->con_C.ptr, sizeof(double) * (size_t)S.k * 3 * V));
        return TPE_OK;
    });
}

int32_t tpe_l2_curve_norm(tpe_ctx* ctx, const double* values, const double* xyz, double* out) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        if (!values || !xyz || !out) return TPE_ERR_BAD_ARG;
        const int32_t V = ctx->V;
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * 3 * (size_t)V));
        TPE_TRY(upload(ctx, ctx->grad, values, sizeof(double) * 3 * (size_t)V));
        return l2_curve_norm(ctx, ctx->grad.as<double>(), ctx->pos.as<double>(), out);
    });
}

int32_t tpe_solve_saddle(tpe_ctx* ctx, const double* A, int32_t n, const double* C, int32_t k,
                         const double* rhs_top, const double* rhs_bottom, int32_t factor_mode,
                         double* x, double* lambda, double* residual) {
    return guarded(ctx, [&]() -> int32_t {
        (void)factor_mode;  // the structured Cholesky solve serves both factor modes
        if (!ctx || !A || n <= 0 || k < 0 || (k > 0 && !C) || !rhs_top || !x) return TPE_ERR_BAD_ARG;
        TPE_CUDA_TRY(cudaSetDevice(ctx->device));
        const size_t m = 3 * (size_t)n;
        if (!all_finite(rhs_top, m) || (rhs_bottom && !all_finite(rhs_bottom, (size_t)k))) {
            set_error(ctx, TPE_ERR_NONFINITE_INPUT, "non-finite right-hand side: treating as singular");
            return TPE_ERR_NONFINITE_INPUT;
        }
        TPE_TRY(upload(ctx, ctx->mat_A, A, sizeof(double) * (size_t)n * n));
        TPE_TRY(ensure(ctx, ctx->con_C, sizeof(double) * (size_t)(k > 0 ? k : 1) * m));
        if (k > 0) TPE_TRY(upload(ctx, ctx->con_C, C, sizeof(double) * (size_t)k * m));
        TPE_TRY(upload(ctx, ctx->flat2, rhs_top, sizeof(double) * m));
        bool singular = false;
        TPE_TRY(op_finalize(ctx, n, k, &singular, ctx->flat2.as<double>()));
        if (singular) {
            set_error(ctx, TPE_ERR_SINGULAR, "saddle system is singular");
            return TPE_ERR_SINGULAR;
        }
        TPE_TRY(ensure(ctx, ctx->flat1, sizeof(double) * m));
        std::vector<double> lam;
        double res = 0.0;
        TPE_TRY(op_solve(ctx, ctx->flat2.as<double>(), rhs_bottom, ctx->flat1.as<double>(), lam, &res));
        TPE_TRY(download(ctx, x, ctx->flat1.ptr, sizeof(double) * m));
        if (lambda && k > 0) memcpy(lambda, lam.data(), sizeof(double) * k);
        if (residual) *residual = res;
        return TPE_OK;
    });
}

int32_t tpe_solve_constrained_gradient(tpe_ctx* ctx, const double* xyz, const double* dE,
                                       const tpe_constraint* set, int32_t nblocks,
                                       const tpe_step_opts* o, double* g_tilde, double* lambda,
                                       double* residual) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        TPE_TRY(validate_opts(ctx, o));
        if (!xyz || !dE || !g_tilde) return TPE_ERR_BAD_ARG;
        const int32_t V = ctx->V;
        const size_t m = 3 * (size_t)V;
        SetInfo S;
        TPE_TRY(set_k(ctx, set, nblocks, &S));
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * m));
        TPE_TRY(upload(ctx, ctx->grad, dE, sizeof(double) * m));
        TPE_TRY(ensure(ctx, ctx->flat2, sizeof(double) * m));
        TPE_TRY(ensure(ctx, ctx->flat1, sizeof(double) * m));
        TPE_TRY(interleaved_to_block(ctx, ctx->grad.as<double>(), ctx->flat2.as<double>(), V));
        bool singular = false;
        TPE_TRY(op_build(ctx, ctx->pos.as<double>(), nblocks, S.k, o->alpha, o->beta, o->epsilon,
                         &singular, nullptr, ctx->flat2.as<double>()));
        if (singular) {
            set_error(ctx, TPE_ERR_SINGULAR, "saddle system is singular");
            return TPE_ERR_SINGULAR;
        }
        std::vector<double> lam;
        double res = 0.0;
        TPE_TRY(op_solve(ctx, ctx->flat2.as<double>(), nullptr, ctx->flat1.as<double>(), lam, &res));
        TPE_TRY(block_to_interleaved(ctx, ctx->flat1.as<double>(), ctx->grad.as<double>(), V));
        TPE_TRY(download(ctx, g_tilde, ctx->grad.ptr, sizeof(double) * m));
        if (lambda && S.k > 0) memcpy(lambda, lam.data(), sizeof(double) * S.k);
        if (residual) *residual = res;
        return TPE_OK;
    });
}

int32_t tpe_project(tpe_ctx* ctx, const double* xyz, const tpe_constraint* set, int32_t nblocks,
                    const tpe_step_opts* o, const double* base_xyz, double* xyz_out, int32_t* ok,
                    int32_t* iterations, double* phi_norm) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        TPE_TRY(validate_opts(ctx, o));
        if (!xyz || !xyz_out || !ok || !iterations || !phi_norm) return TPE_ERR_BAD_ARG;
        const int32_t V = ctx->V;
        const size_t m = 3 * (size_t)V;
        SetInfo S;
        TPE_TRY(set_k(ctx, set, nblocks, &S));
        if (base_xyz) {
            TPE_TRY(upload(ctx, ctx->pos, base_xyz, sizeof(double) * m));
            bool singular = false;
            TPE_TRY(op_build(ctx, ctx->pos.as<double>(), nblocks, S.k, o->alpha, o->beta, o->epsilon,
                             &singular, nullptr));
            if (singular) {
                set_error(ctx, TPE_ERR_SINGULAR, "frozen operator is singular");
                return TPE_ERR_SINGULAR;
            }
        }
        TPE_TRY(upload(ctx, ctx->pos3, xyz, sizeof(double) * m));
        TPE_TRY(ensure(ctx, ctx->pos2, sizeof(double) * m));
        TPE_TRY(project_dev(ctx, ctx->pos3.as<double>(), S, o, base_xyz != nullptr,
                            ctx->pos2.as<double>(), ok, iterations, phi_norm, nullptr));
        return download(ctx, xyz_out, ctx->pos2.ptr, sizeof(double) * m);
    });
}

int32_t tpe_line_search_step(tpe_ctx* ctx, const double* xyz, const double* dE,
                             const double* g_tilde, const tpe_constraint* set, int32_t nblocks,
                             const tpe_step_opts* o, double* xyz_out, tpe_step_stats* st) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        TPE_TRY(validate_opts(ctx, o));
        if (!xyz || !dE || !g_tilde || !xyz_out || !st) return TPE_ERR_BAD_ARG;
        stats_reset(st);
        const int32_t V = ctx->V;
        const size_t m = 3 * (size_t)V;
        SetInfo S;
        TPE_TRY(set_k(ctx, set, nblocks, &S));
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * m));
        TPE_TRY(upload(ctx, ctx->grad, dE, sizeof(double) * m));
        TPE_TRY(upload(ctx, ctx->flat3, g_tilde, sizeof(double) * m));
        const bool frozen = o->projection_mode == TPE_PROJECTION_FROZEN;
        if (frozen) {
            bool singular = false;
            TPE_TRY(op_build(ctx, ctx->pos.as<double>(), nblocks, S.k, o->alpha, o->beta, o->epsilon,
                             &singular, nullptr));
            if (singular) {
                set_error(ctx, TPE_ERR_SINGULAR, "frozen operator is singular");
                return TPE_ERR_SINGULAR;
            }
        }
        // flat3 is reused by the penalty kernels; keep g~ in a dedicated buffer
        TPE_TRY(ensure(ctx, ctx->rhs, sizeof(double) * m));
        TPE_CUDA_TRY(cudaMemcpyAsync(ctx->rhs.ptr, ctx->flat3.ptr, sizeof(double) * m,
                                     cudaMemcpyDeviceToDevice, ctx->stream));
        TPE_TRY(ensure(ctx, ctx->tmp, sizeof(double) * (m + 16)));
        TPE_TRY(ensure(ctx, ctx->sol, sizeof(double) * m));
        double* out = ctx->sol.as<double>();
        TPE_TRY(line_search_dev(ctx, ctx->pos.as<double>(), ctx->grad.as<double>(),
                                ctx->rhs.as<double>(), S, o, frozen, out, st, nullptr));
        return download(ctx, xyz_out, out, sizeof(double) * m);
    });
}

}  // extern "C"

namespace tpe {
namespace {

// sobolevStepSet with the input vertices already in ctx->pos; the result is
// left in *d_result (device, V x 3).
int32_t step_impl(tpe_ctx* ctx, const tpe_constraint* set, int32_t nblocks, const tpe_step_opts* o,
                  tpe_step_stats* st, double* timings, double* descent_field, const double** d_result) {
    const int32_t V = ctx->V;
    const size_t m = 3 * (size_t)V;
    SetInfo S;
    TPE_TRY(set_k(ctx, set, nblocks, &S));
    const double* P = ctx->pos.as<double>();
    *d_result = P;
    TPE_TRY(ensure(ctx, ctx->grad, sizeof(double) * m));
    double* dE = ctx->grad.as<double>();
    const bool pen = o->has_penalties && penalties_active(&o->penalties);
    TPE_TRY(ensure(ctx, ctx->flat2, sizeof(double) * m));
    if (o->mode != TPE_DE_FINITE_DIFF && !timings) {
        // The adjoint gradient (all SMs, FP64 pair work) does not depend on A:
        // it runs on the low-priority stream3 while the main stream assembles
        // and factors A_rho (a latency-bound chain); the solve joins it.
        // op_build launches it right after the assembly (launch_gradient), so it
        // overlaps the factorization and not the (equally compute-bound) Gram
        // assembly.
        TPE_TRY(edge_prep(ctx, P, 1, o->epsilon, o->alpha));
        ctx->grad_unlaunched = true;
        ctx->grad_params[0] = o->alpha;
        ctx->grad_params[1] = o->beta;
        ctx->grad_params[2] = o->epsilon;
        ctx->grad_pending = true;
        ctx->grad_pos = P;
        ctx->grad_dE = dE;
        ctx->grad_flat = ctx->flat2.as<double>();
        ctx->grad_pen = pen ? &o->penalties : nullptr;
    } else {
        // sequential (finite differences, or the per-phase timing ledger)
        {
            Timer t(ctx, timings, TPE_PHASE_DE);
            if (o->mode == TPE_DE_FINITE_DIFF) {
                TPE_TRY(gradient_fd_dev(ctx, P, o->alpha, o->beta, o->epsilon, o->h, dE));
            } else {
                TPE_TRY(edge_prep(ctx, P, 1, o->epsilon, o->alpha));
                TPE_TRY(energy_grad_fp64(ctx, o->alpha, o->beta, o->epsilon, nullptr, dE));
            }
        }
        if (pen) TPE_TRY(penalty_gradient_dev(ctx, P, &o->penalties, dE, 1));
        TPE_TRY(interleaved_to_block(ctx, dE, ctx->flat2.as<double>(), V));
    }
    bool singular = false;
    const int32_t bst = op_build(ctx, P, nblocks, S.k, o->alpha, o->beta, o->epsilon, &singular,
                                 timings, ctx->flat2.as<double>(), o);
    const int32_t fst = finish_gradient(ctx);  // joined even when the build returned early
    TPE_TRY(bst);
    TPE_TRY(fst);
    // The mixed mode's int8-tensor-core inverses (large constraint sets) are
    // rebuilt in FP64 when they come out singular or when the refined gradient
    // solve misses kInt8ResidualGate: conditioning that the digit products do
    // not resolve. The step is then the FP64 step.
    auto fallback_fp64 = [&]() -> int32_t {
        tpe_step_opts o64 = *o;
        o64.precision = TPE_PRECISION_FP64;
        singular = false;
        {
            Timer t(ctx, timings, TPE_PHASE_FACTOR);
            TPE_TRY(op_finalize(ctx, V, S.k, &singular, ctx->flat2.as<double>(), &o64));
        }
        ctx->op.mixed_fallback = true;
        return TPE_OK;
    };
    if (singular && ctx->op.int8) TPE_TRY(fallback_fp64());
    TPE_TRY(ensure(ctx, ctx->sol, sizeof(double) * m));
    double* out = ctx->sol.as<double>();
    std::vector<double> lam;
    double res = 0.0;
    if (!singular) {
        TPE_TRY(ensure(ctx, ctx->flat1, sizeof(double) * m));
        TPE_TRY(ensure(ctx, ctx->rhs, sizeof(double) * m));
        {
            Timer t(ctx, timings, TPE_PHASE_SADDLE);
            TPE_TRY(op_solve(ctx, ctx->flat2.as<double>(), nullptr, ctx->flat1.as<double>(), lam, &res));
        }
        if (ctx->op.int8 && !(res <= kInt8ResidualGate)) {
            TPE_TRY(fallback_fp64());
            if (!singular) {
                Timer t(ctx, timings, TPE_PHASE_SADDLE);
                TPE_TRY(op_solve(ctx, ctx->flat2.as<double>(), nullptr, ctx->flat1.as<double>(), lam,
                                 &res));
            }
        }
    }
    st->refine_iterations = ctx->op.mixed ? ctx->op.refine_iters : (ctx->op.mixed_fallback ? -1 : 0);
    if (singular) {
        double e = o->energy_before;
        if (!o->has_energy_before) TPE_TRY(objective(ctx, P, o, pen, &e, timings));
        st->energy = st->energy_before = e;
        st->reason = TPE_REASON_SINGULAR_SYSTEM;
        return TPE_OK;
    }
    double* g = ctx->rhs.as<double>();
    TPE_TRY(block_to_interleaved(ctx, ctx->flat1.as<double>(), g, V));
    if (descent_field && o->collect_field)
        TPE_TRY(download(ctx, descent_field, g, sizeof(double) * m));
    double gn = 0.0;
    TPE_TRY(l2_curve_norm(ctx, g, P, &gn));
    st->residual = res;
    st->gradient_l2_norm = gn;
    if (gn < 1e-4) {
        double e = o->energy_before;
        if (!o->has_energy_before) TPE_TRY(objective(ctx, P, o, pen, &e, timings));
        st->energy = st->energy_before = e;
        st->converged = 1;
        st->projection_iterations = 0;
        return TPE_OK;
    }
    tpe_step_stats ls;
    stats_reset(&ls);
    TPE_TRY(line_search_dev(ctx, P, dE, g, S, o, o->projection_mode == TPE_PROJECTION_FROZEN, out,
                            &ls, timings));
    st->energy = ls.energy;
    st->energy_before = ls.energy_before;
    st->accepted = ls.accepted;
    st->tau = ls.tau;
    st->projection_iterations = ls.projection_iterations;
    st->projection_phi_norm = ls.projection_phi_norm;
    st->slope = ls.slope;
    st->reason = ls.reason;
    st->trials_evaluated = ls.trials_evaluated;
    *d_result = out;
    return TPE_OK;
}

}  // namespace
}  // namespace tpe

extern "C" {

int32_t tpe_sobolev_step(tpe_ctx* ctx, const double* xyz, const tpe_constraint* set,
                         int32_t nblocks, const tpe_step_opts* o, double* xyz_out,
                         tpe_step_stats* st, double* timings, double* descent_field) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        TPE_TRY(validate_opts(ctx, o));
        if (!xyz || !xyz_out || !st) return TPE_ERR_BAD_ARG;
        stats_reset(st);
        if (timings) memset(timings, 0, sizeof(double) * 2 * TPE_PHASE_COUNT);
        const size_t m = 3 * (size_t)ctx->V;
        const double* res = nullptr;
        {
            Timer tstep(ctx, timings, TPE_PHASE_STEP);
            TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * m));
            TPE_TRY(step_impl(ctx, set, nblocks, o, st, timings, descent_field, &res));
            TPE_TRY(download(ctx, xyz_out, res, sizeof(double) * m));
        }
        return TPE_OK;
    });
}

int32_t tpe_sobolev_step_device(tpe_ctx* ctx, const double* d_xyz, const tpe_constraint* set,
                                int32_t nblocks, const tpe_step_opts* o, double* d_xyz_out,
                                tpe_step_stats* st, double* timings) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        TPE_TRY(validate_opts(ctx, o));
        if (!d_xyz || !d_xyz_out || !st) return TPE_ERR_BAD_ARG;
        stats_reset(st);
        if (timings) memset(timings, 0, sizeof(double) * 2 * TPE_PHASE_COUNT);
        const size_t m = 3 * (size_t)ctx->V;
        const double* res = nullptr;
        {
            Timer tstep(ctx, timings, TPE_PHASE_STEP);
            TPE_TRY(ensure(ctx, ctx->pos, sizeof(double) * m));
            TPE_CUDA_TRY(cudaMemcpyAsync(ctx->pos.ptr, d_xyz, sizeof(double) * m,
                                         cudaMemcpyDeviceToDevice, ctx->stream));
            TPE_TRY(step_impl(ctx, set, nblocks, o, st, timings, nullptr, &res));
            TPE_CUDA_TRY(cudaMemcpyAsync(d_xyz_out, res, sizeof(double) * m, cudaMemcpyDeviceToDevice,
                                         ctx->stream));
            TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        }
        return TPE_OK;
    });
}

void* tpe_stream(tpe_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int32_t tpe_gemm_nt_device(tpe_ctx* ctx, int32_t method, int32_t M, int32_t N, int32_t K,
                           const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                           int64_t ldc, double alpha, double beta, int32_t mode) {
    return guarded(ctx, [&]() -> int32_t {
        if (!ctx) return TPE_ERR_BAD_ARG;
        if (M < 0 || N < 0 || K <= 0 || !A || !B || !C || lda < K || ldb < K || ldc < N ||
            (mode & ~63) != 0 || ((mode & kDLowerTiles) && M != N) ||
            (method != TPE_GEMM_FP64 && method != TPE_GEMM_INT8_EMULATED) ||
            (method == TPE_GEMM_FP64 && (mode & ~7) != 0)) {
            set_error(ctx, TPE_ERR_BAD_ARG, "tpe_gemm_nt_device: bad arguments");
            return TPE_ERR_BAD_ARG;
        }
        TPE_CUDA_TRY(cudaSetDevice(ctx->device));
        DGemmArgs g;
        g.A = A;
        g.lda = lda;
        g.B = B;
        g.ldb = ldb;
        g.C = C;
        g.ldc = ldc;
        g.M = M;
        g.N = N;
        g.K = K;
        g.alpha = alpha;
        g.beta = beta;
        g.mode = mode;
        if (method == TPE_GEMM_FP64) {
            KernelScope ks(ctx, TPE_KGROUP_TRSV, 1);
            return dgemm_nt(ctx, g, ctx->stream);
        }
        TPE_TRY(ozaki_gemm_nt(ctx, g, ctx->stream));
        return ozaki_status(ctx, ctx->stream);
    });
}

int32_t tpe_profile(tpe_ctx* ctx, int32_t on) {
    return guarded(ctx, [&]() -> int32_t {
        if (!ctx) return TPE_ERR_BAD_ARG;
        TPE_CUDA_TRY(cudaSetDevice(ctx->device));
        TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        for (auto& p : ctx->prof_pending) {
            ctx->prof_pool.push_back(p.a);
            ctx->prof_pool.push_back(p.b);
        }
        ctx->prof_pending.clear();
        for (int g = 0; g < TPE_KGROUP_COUNT; g++) ctx->prof_ms[g] = 0.0;
        for (int g = 0; g <= TPE_KGROUP_COUNT; g++) ctx->prof_launches[g] = 0;
        ctx->profiling = on != 0;
        return TPE_OK;
    });
}

int32_t tpe_profile_read(tpe_ctx* ctx, double* ms, int64_t* launches) {
    return guarded(ctx, [&]() -> int32_t {
        if (!ctx) return TPE_ERR_BAD_ARG;
        TPE_CUDA_TRY(cudaSetDevice(ctx->device));
        TPE_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        for (auto& p : ctx->prof_pending) {
            float t = 0.0f;
            if (cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) ctx->prof_ms[p.group] += t;
            ctx->prof_pool.push_back(p.a);
            ctx->prof_pool.push_back(p.b);
        }
        ctx->prof_pending.clear();
        cudaGetLastError();
        if (ms)
            for (int g = 0; g < TPE_KGROUP_COUNT; g++) ms[g] = ctx->prof_ms[g];
        if (launches)
            for (int g = 0; g <= TPE_KGROUP_COUNT; g++) launches[g] = ctx->prof_launches[g];
        return TPE_OK;
    });
}

int32_t tpe_penalty_energy(tpe_ctx* ctx, const double* xyz, const tpe_penalties* pen,
                           double* energy) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        if (!xyz || !pen || !energy) return TPE_ERR_BAD_ARG;
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * 3 * (size_t)ctx->V));
        return penalty_energy_dev(ctx, ctx->pos.as<double>(), pen, energy);
    });
}

int32_t tpe_penalty_gradient(tpe_ctx* ctx, const double* xyz, const tpe_penalties* pen,
                             double* grad) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        if (!xyz || !pen || !grad) return TPE_ERR_BAD_ARG;
        const size_t m = 3 * (size_t)ctx->V;
        TPE_TRY(upload(ctx, ctx->pos, xyz, sizeof(double) * m));
        TPE_TRY(ensure(ctx, ctx->grad, sizeof(double) * m));
        TPE_TRY(penalty_gradient_dev(ctx, ctx->pos.as<double>(), pen, ctx->grad.as<double>(), 0));
        return download(ctx, grad, ctx->grad.ptr, sizeof(double) * m);
    });
}

int32_t tpe_energy_batch(tpe_ctx* ctx, const double* xyz, int32_t ncurves, const tpe_params* p,
                         int32_t precision, double* energies) {
    return guarded(ctx, [&]() -> int32_t {
        TPE_TRY(check_topology(ctx));
        if (!xyz || !p || !energies || ncurves <= 0) return TPE_ERR_BAD_ARG;
        const size_t m = 3 * (size_t)ctx->V;
        TPE_TRY(upload(ctx, ctx->pos3, xyz, sizeof(double) * m * ncurves));
        TPE_TRY(ensure(ctx, ctx->scalars, sizeof(double) * (600 + (size_t)ncurves)));
        double* de = ctx->scalars.as<double>() + 600;
        if (precision == TPE_PRECISION_MIXED) {
            TPE_TRY(edge_prep_mixed(ctx, ctx->pos3.as<double>(), ncurves, p->epsilon, p->alpha));
            TPE_TRY(energy_mixed(ctx, ncurves, p->alpha, p->beta, p->epsilon, de));
        } else {
            TPE_TRY(edge_prep(ctx, ctx->pos3.as<double>(), ncurves, p->epsilon, p->alpha));
            TPE_TRY(energy_fp64(ctx, ncurves, p->alpha, p->beta, p->epsilon, de));
        }
        return download(ctx, energies, de, sizeof(double) * ncurves);
    });
}

}  // extern "C"
