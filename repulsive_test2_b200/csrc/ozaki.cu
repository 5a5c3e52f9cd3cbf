// FP64 matrix products on the integer tensor cores (Ozaki splitting).
//
// C = alpha * A * B^T + beta * C for row-major FP64 A (M x K), B (N x K) and C.
// Each row of an operand is scaled by its own power of two, 2^e with every
// |x| < 2^e, and cut into kS 8-bit digits:
//     x = 2^e * (d0 * 2^-7 + d1 * 2^-15 + d2 * 2^-23 + ... ) + r,  |r| < 2^(e-63),
// d0 signed (-128..127), d1.. unsigned (0..255). Every step of the cut (scaling
// by a power of two, floor, subtraction) is exact in FP64. A digit product
// d^A_p (d^B_q)^T is an exact integer GEMM (tcgen05.mma kind::i8, int32
// accumulator in tensor memory). Products of equal level g = p + q share one
// accumulator, since they carry the same weight 2^-(14 + 8g); levels g < kS are
// formed (36 digit products for kS = 8), the rest lie below 2^-63 of the row
// scales and are dropped. The epilogue adds the level sums in FP64, smallest
// weight first, and applies 2^(e_i + e_j), alpha and beta. The result matches
// an FP64 GEMM to within a few units of 2^-53 of max_k |a_ik| * max_k |b_jk|
// per term: FP64-class accuracy from the int8 tensor cores, which run at
// several times the FP64 tensor-core rate. The bound is normwise per row: an
// entry 2^-d below its row's largest keeps 63 - d bits, so where the rows'
// entries span many orders of magnitude and the sum cancels, the product is
// less accurate than an FP64 GEMM (the large-set solve checks its residual and
// falls back to FP64 there).
//
// Int32 level sums are exact while K * kS * 255^2 < 2^31: one launch covers at
// most kMaxK = 4096 columns of K; longer products run as several launches that
// accumulate into C (beta = 1 after the first).
//
// Pipeline: one CTA per 128 x 64 output tile (four warps). One thread issues
// the TMA loads of all kS digit planes of A (128 x 64 bytes each) and B
// (64 x 64 bytes each) for a 64-column K stage into a two-stage ring (64B
// swizzle); one thread issues the 36 x 2 MMAs of a stage (M=128, N=64, K=32)
// into the kS level accumulators (all 512 TMEM columns); then all
// four warps read the accumulators back (tcgen05.ld) and write C. Every barrier
// wait is bounded (about 2 s): on a timeout the kernel raises *err, lets the
// copies it issued land, frees its tensor memory and returns.
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <cstdlib>

#include "tpe_internal.h"

namespace tpe {
namespace oz {
namespace {

constexpr int kS = 8;                       // digits per element
constexpr int kBM = 128, kBN = 64;          // output tile
constexpr int kBK = 64;                     // K digits (bytes) per stage: one 64B swizzle row
constexpr int kStages = 2;
constexpr int kATile = kBM * kBK;           // 8 KB
constexpr int kBTile = kBN * kBK;           // 4 KB
constexpr int kStageBytes = kS * (kATile + kBTile);
constexpr int kSmemBytes = kStages * kStageBytes + 1024 + 128;
constexpr int kTmemCols = 512;              // kS * kBN = 448 used
constexpr int kMaxK = 4096;
constexpr int kExpNaN = INT_MIN;            // row scale of a row holding NaN or Inf
constexpr long long kWaitCycles = 4000000000LL;
static_assert(kS * kBN <= kTmemCols, "level accumulators exceed tensor memory");
static_assert((long long)kMaxK * kS * 255 * 255 < (1LL << 31), "level sums overflow int32");

enum : int32_t {
    kLowerTiles = 1,  // only output tiles that reach the diagonal or below it
    kAUpper = 2,      // A[i][k] = 0 for k < i: tile row t starts its K range at 128 t
    kALower = 4,      // A[i][k] = 0 for k > i: tile row t ends it at 128 (t + 1)
    kBUpper = 8,      // B[j][k] = 0 for k < j: tile column u starts at 64 u
    kBLower = 16,     // B[j][k] = 0 for k > j: tile column u ends at 64 (u + 1)
    kMaskUpper = 32,  // write only elements with column <= row (a lower-triangle update)
};

struct Params {
    double* C;
    int64_t ldc;
    const int32_t* ea;  // row scales of A (exponents), indexed by A plane row
    const int32_t* eb;
    int32_t M, N;
    int32_t a_row0, b_row0;  // first plane row of the operands
    int32_t a_rows, b_rows;  // rows of one digit plane (tensor-map row stride of a plane)
    int32_t k0, k1;          // digit columns of this launch
    int32_t mode;
    double alpha, beta;
    int32_t* err;
};

// ---- digit planes ------------------------------------------------------------

// planes[p][r][k] (p < kS, r < rows_p, k < kp) of X[r][k] (r < R, k < K), and
// ex[r] with every |X[r][k]| < 2^ex[r]. Rows R.. and columns K.. are zero.
__global__ void __launch_bounds__(256)
split_kernel(const double* __restrict__ X, int64_t ld, int32_t R, int32_t K,
             uint8_t* __restrict__ planes, int32_t rows_p, int32_t kp, int32_t* __restrict__ ex) {
    const int32_t r = blockIdx.x;
    const int64_t plane = (int64_t)rows_p * kp;
    uint8_t* out = planes + (int64_t)r * kp;
    __shared__ double wmax[8];
    __shared__ int32_t e_sh;
    if (r >= R) {
        for (int32_t k = threadIdx.x * 8; k < kp; k += 256 * 8)
#pragma unroll
            for (int p = 0; p < kS; p++) *reinterpret_cast<uint2*>(out + p * plane + k) = make_uint2(0, 0);
        if (threadIdx.x == 0) ex[r] = 0;
        return;
    }
    const double* x = X + (int64_t)r * ld;
    double m = 0.0;
    bool finite = true;
    for (int32_t k = threadIdx.x; k < K; k += 256) {
        const double v = fabs(x[k]);
        finite = finite && isfinite(v);
        m = fmax(m, v);
    }
    finite = __syncthreads_and(finite) != 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mm = 0.0;
        for (int w = 0; w < 8; w++) mm = fmax(mm, wmax[w]);
        e_sh = !finite ? kExpNaN : (mm > 0.0 ? ilogb(mm) + 1 : 0);
        ex[r] = e_sh;
    }
    __syncthreads();
    const int32_t e = e_sh == kExpNaN ? 0 : e_sh;
    for (int32_t k0 = threadIdx.x * 8; k0 < kp; k0 += 256 * 8) {
        uint32_t w[kS][2];
#pragma unroll
        for (int p = 0; p < kS; p++) w[p][0] = w[p][1] = 0u;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int32_t k = k0 + j;
            double v = (k < K && e_sh != kExpNaN) ? x[k] : 0.0;
            v = scalbn(v, 7 - e);  // in (-128, 128)
            double f = floor(v);
            const int32_t d0 = (int32_t)f;
            double rem = v - f;  // [0, 1)
            w[0][j >> 2] |= ((uint32_t)d0 & 0xFFu) << (8 * (j & 3));
#pragma unroll
            for (int p = 1; p < kS; p++) {
                rem *= 256.0;
                f = floor(rem);
                rem -= f;
                w[p][j >> 2] |= ((uint32_t)f & 0xFFu) << (8 * (j & 3));
            }
        }
#pragma unroll
        for (int p = 0; p < kS; p++)
            *reinterpret_cast<uint2*>(out + p * plane + k0) = make_uint2(w[p][0], w[p][1]);
    }
}


// ---- pipeline primitives -------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t a) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of parity `parity`; false (and *err = 1) after kWaitCycles.
__device__ bool mbar_wait(uint32_t a, uint32_t parity, int32_t* err) {
    if (mbar_try(a, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try(a, parity)) {
        if (clock64() - t0 > kWaitCycles) {
            if (err) atomicExch(err, 1);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t mbar,
                                            int32_t x, int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"((uint64_t)map), "r"(mbar), "r"(x), "r"(y)
        : "memory");
}

// Shared-memory matrix descriptor: K-major operand, 64B swizzle (layout type 4),
// 8-row groups 512 bytes apart (SBO), descriptor version 1 (bit 46).
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) |
           ((uint64_t)(512 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

// Instruction descriptor of tcgen05.mma kind::i8: D format S32 (bits 4-5 = 2),
// A and B format signed (1) or unsigned (0) 8-bit (bits 7-9, 10-12), both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_i8(bool a_signed, bool b_signed) {
    return (2u << 4) | ((a_signed ? 1u : 0u) << 7) | ((b_signed ? 1u : 0u) << 10) |
           ((uint32_t)(kBN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     mbar)
                 : "memory");
}

// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int32_t (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = (int32_t)r[i];
}

// ---- the product ---------------------------------------------------------------

__global__ void __launch_bounds__(128, 1)
gemm_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
            const Params P) {
    const int32_t ti = blockIdx.y, tj = blockIdx.x;
    if ((P.mode & kLowerTiles) && tj * kBN > ti * kBM + kBM - 1) return;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + kStages * kStageBytes);  // full[2], empty[2], done
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * kStages + 1);
    volatile int32_t* aborted = (volatile int32_t*)(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    int32_t kb = P.k0, ke = P.k1;
    if (P.mode & kAUpper) kb = max(kb, ti * kBM);
    if (P.mode & kALower) ke = min(ke, (ti + 1) * kBM);
    if (P.mode & kBUpper) kb = max(kb, tj * kBN);
    if (P.mode & kBLower) ke = min(ke, (tj + 1) * kBN);
    kb -= kb % kBK;
    const int nk = ke > kb ? (ke - kb + kBK - 1) / kBK : 0;

    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kStages),
                   done = smem_u32(bars + 2 * kStages);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done, 1);
        *aborted = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const int32_t ay = P.a_row0 + ti * kBM, by = P.b_row0 + tj * kBN;

    if (warp == 0 && lane == 0) {
        // TMA producer: all digit planes of A and B for one K stage
        int issued = 0;
        for (int it = 0; it < nk; it++) {
            const int s = it % kStages;
            if (it >= kStages && !mbar_wait(empty0 + 8 * s, ((it / kStages) - 1) & 1, P.err)) {
                *aborted = 1;
                break;
            }
            if (*aborted) break;
            const uint32_t st = smem_u32(smem + s * kStageBytes);
            const uint32_t fb = full0 + 8 * s;
            mbar_expect_tx(fb, kStageBytes);
            const int32_t x = kb + it * kBK;
            for (int p = 0; p < kS; p++)
                tma_load_2d(st + p * kATile, &map_a, fb, x, p * P.a_rows + ay);
            for (int q = 0; q < kS; q++)
                tma_load_2d(st + kS * kATile + q * kBTile, &map_b, fb, x, q * P.b_rows + by);
            issued = it + 1;
        }
        // every copy issued has landed before the CTA may exit
        for (int it = issued > kStages ? issued - kStages : 0; it < issued; it++)
            mbar_wait(full0 + 8 * (it % kStages), (it / kStages) & 1, P.err);
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: level g = p + q accumulates d^A_p d^B_q^T in columns [64 g, 64 g + 64)
        for (int it = 0; it < nk; it++) {
            const int s = it % kStages;
            if (!mbar_wait(full0 + 8 * s, (it / kStages) & 1, P.err)) {
                *aborted = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = smem_u32(smem + s * kStageBytes);
#pragma unroll
            for (int p = 0; p < kS; p++) {
#pragma unroll
                for (int q = 0; q < kS - p; q++) {
                    const uint32_t id = idesc_i8(p == 0, q == 0);
                    const uint32_t d = tmem + (uint32_t)((p + q) * kBN);
#pragma unroll
                    for (int kk = 0; kk < kBK / 32; kk++) {
                        const uint64_t a = sw64_desc(st + p * kATile + kk * 32);
                        const uint64_t b = sw64_desc(st + kS * kATile + q * kBTile + kk * 32);
                        // the first product of each level (p = 0) starts its accumulator
                        mma_i8(d, a, b, id, (it | kk | p) ? 1u : 0u);
                    }
                }
            }
            mma_commit(empty0 + 8 * s);
        }
        if (nk > 0)
            mma_commit(done);
        else
            mbar_arrive(done);
    }
    __syncwarp();
    __syncthreads();

    bool ok = mbar_wait(done, 0, P.err);
    ok = __syncthreads_and(ok && !*aborted) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        const int32_t row = ti * kBM + warp * 32 + lane;
        const bool rin = row < P.M;
        const int32_t era = rin ? P.ea[P.a_row0 + row] : 0;
        double* crow = P.C + (int64_t)(rin ? row : 0) * P.ldc;
        for (int h = 0; h < kBN / 32; h++) {
            double acc[32];
#pragma unroll
            for (int c = 0; c < 32; c++) acc[c] = 0.0;
            if (nk > 0) {
#pragma unroll 1
                for (int g = kS - 1; g >= 0; g--) {
                    int32_t v[32];
                    tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(g * kBN + 32 * h), v);
                    const double w = scalbn(1.0, -(14 + 8 * g));
#pragma unroll
                    for (int c = 0; c < 32; c++) acc[c] += (double)v[c] * w;
                }
            }
            if (!rin) continue;
            const int32_t cend = min(P.N, (P.mode & kMaskUpper) ? row + 1 : P.N);
#pragma unroll
            for (int c = 0; c < 32; c++) {
                const int32_t col = tj * kBN + 32 * h + c;
                if (col >= cend) continue;
                const int32_t erb = P.eb[P.b_row0 + col];
                double y;
                if (era == kExpNaN || erb == kExpNaN)
                    y = __longlong_as_double(0x7FF8000000000000LL);
                else
                    y = P.alpha * scalbn(acc[c], era + erb);
                if (P.beta != 0.0) y += P.beta * crow[col];
                crow[col] = y;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols)
                     : "memory");
}


// 2-D uint8 tensor map over `rows` rows of `kp` digits (row stride kp bytes),
// boxes of box_rows x 64 digits, 64B swizzle.
bool encode_planes(CUtensorMap* map, uint8_t* base, int64_t rows, int32_t kp, int32_t box_rows) {
    auto enc = tc::tensor_map_encoder();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kp};
    cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

}  // namespace
}  // namespace oz

size_t ozaki_scratch_bytes(int32_t M, int32_t N, int32_t K) {
    const int64_t kp = oz::round_up(K, oz::kBK);
    return (size_t)oz::kS * (size_t)kp * (size_t)(oz::round_up(M, oz::kBM) + oz::round_up(N, oz::kBN)) +
           sizeof(int32_t) * (size_t)(oz::round_up(M, oz::kBM) + oz::round_up(N, oz::kBN)) + 2048;
}

int32_t ozaki_reserve(tpe_ctx* ctx, size_t bytes) {
    TPE_TRY(ensure(ctx, ctx->oz_planes, bytes));
    if (!ctx->oz_err.ptr) {
        TPE_TRY(ensure(ctx, ctx->oz_err, sizeof(int32_t)));
        TPE_CUDA_TRY(cudaMemset(ctx->oz_err.ptr, 0, sizeof(int32_t)));
    }
    return TPE_OK;
}

int32_t ozaki_gemm_nt(tpe_ctx* ctx, const DGemmArgs& g, cudaStream_t stream, int group) {
    using namespace oz;
    if (g.M <= 0 || g.N <= 0) return TPE_OK;
    if (g.K <= 0 || !g.A || !g.B || !g.C || g.lda < g.K || g.ldb < g.K || g.ldc < g.N ||
        ((g.mode & kDLowerTiles) && g.M != g.N)) {
        set_error(ctx, TPE_ERR_BAD_ARG, "ozaki_gemm_nt: bad shape");
        return TPE_ERR_BAD_ARG;
    }
    const int64_t kp = round_up(g.K, kBK);
    // B may be a band of A's rows (a symmetric update): its digits are then A's
    // (addresses compared as integers: A and B may be separate allocations)
    const uintptr_t pa_ = (uintptr_t)g.A, pb_ = (uintptr_t)g.B;
    const uintptr_t row = (uintptr_t)g.lda * sizeof(double);
    const int64_t off = pb_ >= pa_ ? (int64_t)((pb_ - pa_) / row) : -1;
    const bool shared = g.lda == g.ldb && pb_ >= pa_ && (pb_ - pa_) % row == 0 && off + g.N <= g.M;
    const int64_t mp = round_up(g.M, kBM);
    const int64_t np = shared ? 0 : round_up(g.N, kBN);
    const size_t need = ozaki_scratch_bytes(g.M, shared ? 0 : g.N, g.K);
    TPE_TRY(ozaki_reserve(ctx, need));
    uint8_t* pa = ctx->oz_planes.as<uint8_t>();
    uint8_t* pb = pa + (size_t)kS * mp * kp;
    // plane bytes are multiples of 8 KB, so the scales start aligned
    int32_t* ea = reinterpret_cast<int32_t*>(pb + (size_t)kS * np * kp);
    int32_t* eb = ea + mp;
    int32_t* err = ctx->oz_err.as<int32_t>();
    KernelScope ks(ctx, group, (shared ? 1 : 2) + (g.K + kMaxK - 1) / kMaxK);
    split_kernel<<<(unsigned)mp, 256, 0, stream>>>(g.A, g.lda, g.M, g.K, pa, (int32_t)mp, (int32_t)kp, ea);
    TPE_CUDA_TRY(cudaGetLastError());
    if (!shared) {
        split_kernel<<<(unsigned)np, 256, 0, stream>>>(g.B, g.ldb, g.N, g.K, pb, (int32_t)np, (int32_t)kp, eb);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    CUtensorMap ma, mb;
    if (!encode_planes(&ma, pa, kS * mp, (int32_t)kp, kBM) ||
        !encode_planes(&mb, shared ? pa : pb, kS * (shared ? mp : np), (int32_t)kp, kBN)) {
        set_error(ctx, TPE_ERR_CUDA, "ozaki_gemm_nt: tensor map encoding failed");
        return TPE_ERR_CUDA;
    }
    TPE_CUDA_TRY(cudaFuncSetAttribute(gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      kSmemBytes));
    Params P;
    P.C = g.C;
    P.ldc = g.ldc;
    P.ea = ea;
    P.eb = shared ? ea : eb;
    P.M = g.M;
    P.N = g.N;
    P.a_row0 = 0;
    P.b_row0 = shared ? (int32_t)off : 0;
    P.a_rows = (int32_t)mp;
    P.b_rows = (int32_t)(shared ? mp : np);
    P.mode = g.mode;
    P.alpha = g.alpha;
    P.err = err;
    const dim3 grid((unsigned)((g.N + kBN - 1) / kBN), (unsigned)((g.M + kBM - 1) / kBM));
    for (int32_t k0 = 0; k0 < g.K; k0 += kMaxK) {
        P.k0 = k0;
        P.k1 = std::min(g.K, k0 + kMaxK);
        P.beta = k0 == 0 ? g.beta : 1.0;
        gemm_kernel<<<grid, 128, kSmemBytes, stream>>>(ma, mb, P);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    return TPE_OK;
}

int32_t ozaki_status(tpe_ctx* ctx, cudaStream_t stream) {
    if (!ctx->oz_err.ptr) return TPE_OK;
    int32_t h = 0;
    TPE_CUDA_TRY(cudaMemcpyAsync(&h, ctx->oz_err.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
    TPE_CUDA_TRY(cudaStreamSynchronize(stream));
    if (h) {
        TPE_CUDA_TRY(cudaMemsetAsync(ctx->oz_err.ptr, 0, sizeof(int32_t), stream));
        set_error(ctx, TPE_ERR_DEVICE_TIMEOUT, "integer tensor-core pipeline wait timed out");
        return TPE_ERR_DEVICE_TIMEOUT;
    }
    return TPE_OK;
}


// ---- SPD inverse on the integer tensor cores -------------------------------------

namespace {

constexpr int32_t kBase = 1024;  // largest block factored and inverted by the FP64 kernels

// The base block size: kBase, or TPE_INT8_BASE (128..kBase) to test the
// recursion at small orders.
int32_t base_size() {
    const char* s = getenv("TPE_INT8_BASE");
    if (!s) return kBase;
    const int v = atoi(s);
    return v < 128 ? 128 : (v > kBase ? kBase : v);
}

struct InvCtx {
    tpe_ctx* ctx;
    double* M;  // n x n, lower triangle: A, overwritten by L below the diagonal blocks
    double* X;  // L^{-1}, lower
    double* W;  // X^T, upper
    double* Tt;
    double* base;  // kBase^2 (block) + 64 kBase (diagonal inverses) + 2 kBase^2 (X, W) + T
    int32_t n;
    double tol;
    int32_t nbase;
    bool singular;
};

DGemmArgs gemm_args(const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                    int64_t ldc, int32_t M, int32_t N, int32_t K, double alpha, double beta,
                    int32_t mode) {
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
    return g;
}

int32_t inv_base(InvCtx& c, int32_t o, int32_t m) {
    tpe_ctx* ctx = c.ctx;
    const cudaStream_t st = ctx->stream;
    const int64_t n = c.n;
    double* Bm = c.base;
    double* Binv = Bm + (size_t)kBase * kBase;
    double* Xb = Binv + (size_t)kBase * kNB;  // (kBase / 64) diagonal 64 x 64 inverses
    double* Wb = Xb + (size_t)kBase * kBase;
    double* Tb = Wb + (size_t)kBase * kBase;
    TPE_CUDA_TRY(cudaMemcpy2DAsync(Bm, sizeof(double) * m, c.M + o * n + o, sizeof(double) * n,
                                   sizeof(double) * m, m, cudaMemcpyDeviceToDevice, st));
    int32_t bad = 0;
    TPE_TRY(cholesky_fp64(ctx, Bm, Binv, m, c.tol, &bad));
    if (bad) {
        c.singular = true;
        return TPE_OK;
    }
    TPE_TRY(lower_inverse_fp64(ctx, Bm, Binv, m, Xb, Wb, Tb));
    TPE_CUDA_TRY(cudaMemcpy2DAsync(c.X + o * n + o, sizeof(double) * n, Xb, sizeof(double) * m,
                                   sizeof(double) * m, m, cudaMemcpyDeviceToDevice, st));
    TPE_CUDA_TRY(cudaMemcpy2DAsync(c.W + o * n + o, sizeof(double) * n, Wb, sizeof(double) * m,
                                   sizeof(double) * m, m, cudaMemcpyDeviceToDevice, st));
    return TPE_OK;
}

// Block [o, o + m) of the diagonal: L, X = L^{-1} and W = X^T, from the trailing
// matrix held in c.M (updated by the blocks before it).
int32_t inv_rec(InvCtx& c, int32_t o, int32_t m) {
    if (m <= c.nbase) return inv_base(c, o, m);
    tpe_ctx* ctx = c.ctx;
    const cudaStream_t st = ctx->stream;
    const int64_t n = c.n;
    const int32_t h = (m / 2 + 63) / 64 * 64, m2 = m - h;
    const int32_t o2 = o + h;
    TPE_TRY(inv_rec(c, o, h));
    if (c.singular) return TPE_OK;
    double* A21 = c.M + o2 * n + o;
    // L21 = A21 X11^T, in place (the product reads A21's digits, not A21)
    TPE_TRY(ozaki_gemm_nt(ctx, gemm_args(A21, n, c.X + o * n + o, n, A21, n, m2, h, h, 1.0, 0.0,
                                         kDBLower), st));
    // A22 -= L21 L21^T (lower triangle)
    TPE_TRY(ozaki_gemm_nt(ctx, gemm_args(A21, n, A21, n, c.M + o2 * n + o2, n, m2, m2, h, -1.0, 1.0,
                                         kDLowerTiles | kDMaskUpper), st));
    TPE_TRY(inv_rec(c, o2, m2));
    if (c.singular) return TPE_OK;
    // T^T (h x m2) = W11 L21^T, then X21 = -X22 T, W12 = X21^T
    TPE_TRY(ozaki_gemm_nt(ctx, gemm_args(c.W + o * n + o, n, A21, n, c.Tt, m2, h, m2, h, 1.0, 0.0,
                                         kDAUpper), st));
    TPE_TRY(ozaki_gemm_nt(ctx, gemm_args(c.X + o2 * n + o2, n, c.Tt, m2, c.X + o2 * n + o, n, m2, h,
                                         m2, -1.0, 0.0, kDALower), st));
    TPE_TRY(transpose_fp64(ctx, c.X + o2 * n + o, n, m2, h, c.W + o * n + o2, n));
    return TPE_OK;
}

}  // namespace

int32_t spd_inverse_int8(tpe_ctx* ctx, double* Mat, int32_t n, double piv_tol, double* X,
                         double* W, double* Tt, double* out, bool* singular) {
    *singular = false;
    if (n <= 0) return TPE_OK;
    TPE_TRY(ozaki_reserve(ctx, ozaki_scratch_bytes(n, 0, n)));
    const size_t base_doubles = (size_t)kBase * kBase * 3 + (size_t)kBase * kNB +
                                (size_t)(kBase / 2 + kNB) * (kBase / 2 + kNB);
    TPE_TRY(ensure(ctx, ctx->oz_base, sizeof(double) * base_doubles));
    TPE_CUDA_TRY(cudaMemsetAsync(X, 0, sizeof(double) * (size_t)n * n, ctx->stream));
    TPE_CUDA_TRY(cudaMemsetAsync(W, 0, sizeof(double) * (size_t)n * n, ctx->stream));
    InvCtx c{ctx, Mat, X, W, Tt, ctx->oz_base.as<double>(), n, piv_tol, base_size(), false};
    TPE_TRY(inv_rec(c, 0, n));
    TPE_TRY(ozaki_status(ctx, ctx->stream));
    if (c.singular) {
        *singular = true;
        return TPE_OK;
    }
    // out = X^T X = W W^T (lower tiles; W[i][k] = 0 for k < i), mirrored
    TPE_TRY(ozaki_gemm_nt(ctx, gemm_args(W, n, W, n, out, n, n, n, n, 1.0, 0.0,
                                         kDLowerTiles | kDAUpper), ctx->stream));
    TPE_TRY(mirror_lower(ctx, out, n));
    return ozaki_status(ctx, ctx->stream);
}

}  // namespace tpe
