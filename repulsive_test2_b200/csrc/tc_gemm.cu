// 3xTF32 tensor-core GEMM for sm_100a: C = alpha * A * B^T + beta * C on
// split-FP32 matrices (tc.h).
//
// One CTA computes one 128 x 128 output tile with the fifth-generation tensor
// cores: operand tiles arrive by TMA (128B swizzle, K-major) into a 3-stage
// shared-memory ring, one elected thread issues tcgen05.mma (kind::tf32,
// M=128, N=128, K=8) with the FP32 accumulator in tensor memory, and the four
// warps read the accumulator back with tcgen05.ld for the epilogue, which
// adds beta * C and writes C again as a split pair. Every wait on a pipeline
// barrier is bounded: when one gives up, the kernel raises *err, lets the
// copies it issued land, frees its tensor memory and returns.
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "tc.h"

namespace tpe {
namespace tc {
namespace {

constexpr int kStages = 3;
constexpr int kTileBytes = kBM * kBK * 4;  // one 128 x 32 FP32 operand tile (A and B alike)
constexpr int kStageBytes = 4 * kTileBytes;  // A_hi, A_lo, B_hi, B_lo
constexpr int kSmemBytes = kStages * kStageBytes + 1024 + 128;
constexpr int kTmemCols = 128;
// Instruction descriptor of tcgen05.mma kind::tf32: D format F32 (bits 4-5),
// A and B format TF32 (bits 7-9, 10-12), both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) |
                            ((uint32_t)(kBN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
constexpr long long kWaitCycles = 4000000000LL;  // about 2 s at 1.9 GHz

struct KParams {
    GemmArgs g;
    float* c_hi;
    float* c_lo;
    int32_t ldc;
    int32_t tma_epi;  // 0: register epilogue; 1: TMA store (beta 0); 2: TMA reduce-add (beta 1, plain C)
    int32_t* err;
};

__host__ __device__ __forceinline__ void split(float x, float& hi, float& lo) {
    // round to nearest (ties away) at TF32 precision, then the exact remainder
    union {
        float f;
        uint32_t u;
    } v;
    v.f = x;
    v.u = (v.u + 0x1000u) & 0xFFFFE000u;
    hi = v.f;
    lo = x - hi;
}

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

// Waits for the phase of parity `parity` to complete; false (and *err = 1)
// when it has not completed within kWaitCycles.
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

__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, uint32_t src, int32_t x,
                                             int32_t y) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                     (uint64_t)map),
                 "r"(src), "r"(x), "r"(y)
                 : "memory");
}

__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap* map, uint32_t src, int32_t x,
                                                  int32_t y) {
    asm volatile(
        "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
            (uint64_t)map),
        "r"(src), "r"(x), "r"(y)
        : "memory");
}

// Shared-memory matrix descriptor: K-major operand, 128B swizzle, 8-row groups
// 1024 bytes apart (SBO), descriptor version 1 (bit 46), layout 2 = SWIZZLE_128B.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) |
           ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     mbar)
                 : "memory");
}

// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
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
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(128, 1)
gemm_nt_kernel(const __grid_constant__ CUtensorMap a_hi, const __grid_constant__ CUtensorMap a_lo,
               const __grid_constant__ CUtensorMap b_hi, const __grid_constant__ CUtensorMap b_lo,
               const __grid_constant__ CUtensorMap c_hi, const __grid_constant__ CUtensorMap c_lo,
               const KParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + kStages * kStageBytes);  // full[S], empty[S], done
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * kStages + 1);
    volatile int32_t* aborted = (volatile int32_t*)(tmem_slot + 1);
    const GemmArgs& g = P.g;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int z = blockIdx.z;

    int ti, tj;
    if (g.mode & kLowerTiles) {
        const int x = blockIdx.x;
        int t = (int)((sqrtf(8.0f * (float)x + 1.0f) - 1.0f) * 0.5f);
        while ((t + 1) * (t + 2) / 2 <= x) t++;
        while (t * (t + 1) / 2 > x) t--;
        ti = t;
        tj = x - t * (t + 1) / 2;
    } else {
        ti = blockIdx.y;
        tj = blockIdx.x;
    }
    int k_begin = 0, k_end = g.K;
    if (g.mode & kAUpper) k_begin = min(g.K, ti * kBM);
    if (g.mode & kALower) k_end = min(g.K, (ti + 1) * kBM);
    const int nk = k_end > k_begin ? (k_end - k_begin) / kBK : 0;

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

    const int32_t ax = g.a_c0 + z * g.a_zc + k_begin, ay = g.a_r0 + z * g.a_zr + ti * kBM;
    const int32_t bx = g.b_c0 + z * g.b_zc + k_begin, by = g.b_r0 + z * g.b_zr + tj * kBN;

    if (warp == 0 && lane == 0) {
        // TMA producer
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
            const int32_t k = it * kBK;
            tma_load_2d(st, &a_hi, fb, ax + k, ay);
            tma_load_2d(st + kTileBytes, &a_lo, fb, ax + k, ay);
            tma_load_2d(st + 2 * kTileBytes, &b_hi, fb, bx + k, by);
            tma_load_2d(st + 3 * kTileBytes, &b_lo, fb, bx + k, by);
            issued = it + 1;
        }
        // every copy issued has landed before the CTA may exit
        for (int it = issued > kStages ? issued - kStages : 0; it < issued; it++)
            mbar_wait(full0 + 8 * (it % kStages), (it / kStages) & 1, P.err);
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: D += Ahi*Bhi + Ahi*Blo + Alo*Bhi per K=8 step
        for (int it = 0; it < nk; it++) {
            const int s = it % kStages;
            if (!mbar_wait(full0 + 8 * s, (it / kStages) & 1, P.err)) {
                *aborted = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = smem_u32(smem + s * kStageBytes);
#pragma unroll
            for (int kk = 0; kk < kBK / 8; kk++) {
                const uint64_t ah = sw128_desc(st + kk * 32);
                const uint64_t al = sw128_desc(st + kTileBytes + kk * 32);
                const uint64_t bh = sw128_desc(st + 2 * kTileBytes + kk * 32);
                const uint64_t bl = sw128_desc(st + 3 * kTileBytes + kk * 32);
                mma_tf32(tmem, ah, bh, (it | kk) ? 1u : 0u);
                mma_tf32(tmem, ah, bl, 1u);
                mma_tf32(tmem, al, bh, 1u);
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
    if (ok && P.tma_epi) {
        // Stage the tile in the (now idle) pipeline buffers in the 128B-swizzled
        // box layout of the C tensor maps (4 boxes of 128 rows x 32 columns; a
        // second set for lo), then one thread stores or reduce-adds the boxes.
        const bool split_out = P.c_lo != nullptr;
        const int r = warp * 32 + lane;
        const float alpha = g.alpha;
        for (int b = 0; b < 4; b++) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(32 * b), v);
            uint8_t* row_hi = smem + b * kTileBytes + r * 128;
            uint8_t* row_lo = smem + 4 * kTileBytes + b * kTileBytes + r * 128;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int pq = (q ^ (r & 7)) * 16;
                float4 y = make_float4(alpha * v[4 * q], alpha * v[4 * q + 1], alpha * v[4 * q + 2],
                                       alpha * v[4 * q + 3]);
                if (split_out) {
                    float4 h, l;
                    split(y.x, h.x, l.x);
                    split(y.y, h.y, l.y);
                    split(y.z, h.z, l.z);
                    split(y.w, h.w, l.w);
                    *reinterpret_cast<float4*>(row_hi + pq) = h;
                    *reinterpret_cast<float4*>(row_lo + pq) = l;
                } else {
                    *reinterpret_cast<float4*>(row_hi + pq) = y;
                }
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            const int32_t x0 = g.c_c0 + z * g.c_zc + tj * kBN, y0 = g.c_r0 + z * g.c_zr + ti * kBM;
            for (int b = 0; b < 4; b++) {
                const uint32_t src = smem_u32(smem + b * kTileBytes);
                if (P.tma_epi == 2)
                    tma_reduce_add_2d(&c_hi, src, x0 + 32 * b, y0);
                else
                    tma_store_2d(&c_hi, src, x0 + 32 * b, y0);
            }
            if (split_out)
                for (int b = 0; b < 4; b++)
                    tma_store_2d(&c_lo, smem_u32(smem + 4 * kTileBytes + b * kTileBytes),
                                 x0 + 32 * b, y0);
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
        }
    } else if (ok) {
        const int row = ti * kBM + warp * 32 + lane;
        const bool rin = row < g.M;
        const int32_t cr = g.c_r0 + z * g.c_zr + (rin ? row : 0);
        const int32_t cc = g.c_c0 + z * g.c_zc;
        float* ch = P.c_hi + (size_t)cr * P.ldc + cc;
        float* cl = P.c_lo ? P.c_lo + (size_t)cr * P.ldc + cc : nullptr;
        const bool vec_ok = (cc & 3) == 0;
        const float alpha = g.alpha, beta = g.beta;
        for (int c0 = 0; c0 < kBN; c0 += 32) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (!rin) continue;
            const int col0 = tj * kBN + c0;
            if (!cl) {
                // plain FP32 output
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int col = col0 + 4 * q;
                    if (vec_ok && col + 3 < g.N) {
                        float4 y = make_float4(alpha * v[4 * q], alpha * v[4 * q + 1],
                                               alpha * v[4 * q + 2], alpha * v[4 * q + 3]);
                        if (beta != 0.0f) {
                            const float4 h = *reinterpret_cast<const float4*>(ch + col);
                            y.x += beta * h.x;
                            y.y += beta * h.y;
                            y.z += beta * h.z;
                            y.w += beta * h.w;
                        }
                        *reinterpret_cast<float4*>(ch + col) = y;
                    } else {
                        for (int e = 0; e < 4; e++) {
                            if (col + e >= g.N) break;
                            float y = alpha * v[4 * q + e];
                            if (beta != 0.0f) y += beta * ch[col + e];
                            ch[col + e] = y;
                        }
                    }
                }
                continue;
            }
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int col = col0 + 4 * q;
                if (vec_ok && col + 3 < g.N) {
                    float y[4] = {alpha * v[4 * q], alpha * v[4 * q + 1], alpha * v[4 * q + 2],
                                  alpha * v[4 * q + 3]};
                    if (beta != 0.0f) {
                        const float4 h = *reinterpret_cast<const float4*>(ch + col);
                        const float4 l = *reinterpret_cast<const float4*>(cl + col);
                        y[0] += beta * (h.x + l.x);
                        y[1] += beta * (h.y + l.y);
                        y[2] += beta * (h.z + l.z);
                        y[3] += beta * (h.w + l.w);
                    }
                    float4 h, l;
                    split(y[0], h.x, l.x);
                    split(y[1], h.y, l.y);
                    split(y[2], h.z, l.z);
                    split(y[3], h.w, l.w);
                    *reinterpret_cast<float4*>(ch + col) = h;
                    *reinterpret_cast<float4*>(cl + col) = l;
                } else {
                    for (int e = 0; e < 4; e++) {
                        if (col + e >= g.N) break;
                        float y = alpha * v[4 * q + e];
                        if (beta != 0.0f) y += beta * (ch[col + e] + cl[col + e]);
                        float h, l;
                        split(y, h, l);
                        ch[col + e] = h;
                        cl[col + e] = l;
                    }
                }
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

// ---- persistent form ----------------------------------------------------------
//
// The same product with one CTA per SM walking many output tiles: warp 0 is
// the TMA producer, warp 1 issues the MMAs into one of two TMEM accumulators
// (256 columns), warps 2-5 drain the other accumulator through a 32 KB staging
// buffer and TMA stores / reduce-adds, so a tile's epilogue overlaps the next
// tile's loads and MMAs and the set-up (barriers, TMEM, tensor maps) is paid
// once per SM. Tiles come from a device counter (zeroed by the caller) when one
// is given, else round-robin. The tile index travels from the producer to the
// MMA thread in the ring slot of the tile's first stage and from there to the
// epilogue with the accumulator, each published by an ordinary mbarrier
// arrive (release) before the consumer's wait (acquire). TMA epilogues only
// (whole 128 x 128 tiles).
constexpr int kPThreads = 192;
constexpr int kOutBytes = 2 * kTileBytes;  // epilogue staging: 2 x (128 rows x 32 columns)
constexpr int kPSmemBytes = kStages * kStageBytes + kOutBytes + 1024 + 256;
static_assert(kPSmemBytes <= 232448, "persistent GEMM shared memory exceeds the per-block limit");

__device__ __forceinline__ void decode_tile(int x, const GemmArgs& g, int tm, int tn, int& z,
                                            int& ti, int& tj) {
    const int per = (g.mode & kLowerTiles) ? tm * (tm + 1) / 2 : tm * tn;
    z = x / per;
    const int r = x - z * per;
    if (g.mode & kLowerTiles) {
        int t = (int)((sqrtf(8.0f * (float)r + 1.0f) - 1.0f) * 0.5f);
        while ((t + 1) * (t + 2) / 2 <= r) t++;
        while (t * (t + 1) / 2 > r) t--;
        ti = t;
        tj = r - t * (t + 1) / 2;
    } else {
        ti = r / tn;
        tj = r - ti * tn;
    }
}

__device__ __forceinline__ void tile_k_range(const GemmArgs& g, int ti, int& k_begin, int& nk) {
    int kb = 0, ke = g.K;
    if (g.mode & kAUpper) kb = min(g.K, ti * kBM);
    if (g.mode & kALower) ke = min(g.K, (ti + 1) * kBM);
    k_begin = kb;
    nk = ke > kb ? (ke - kb) / kBK : 0;
}

__device__ __forceinline__ void epi_sync() {
    asm volatile("bar.sync 1, 128;" ::: "memory");
}

__global__ void __launch_bounds__(kPThreads, 1)
gemm_nt_persist_kernel(const __grid_constant__ CUtensorMap a_hi,
                       const __grid_constant__ CUtensorMap a_lo,
                       const __grid_constant__ CUtensorMap b_hi,
                       const __grid_constant__ CUtensorMap b_lo,
                       const __grid_constant__ CUtensorMap c_hi,
                       const __grid_constant__ CUtensorMap c_lo, const KParams P, int32_t tm,
                       int32_t tn, int32_t ntiles, int32_t* __restrict__ tile_ctr) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* stage_out = smem + kStages * kStageBytes;
    // full[S], empty[S], acc_full[2], acc_empty[2], done
    uint64_t* bars = (uint64_t*)(stage_out + kOutBytes);
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * kStages + 5);
    volatile int32_t* aborted = (volatile int32_t*)(tmem_slot + 1);
    volatile int32_t* tileq = aborted + 1;          // [kStages]
    volatile int32_t* accq = tileq + kStages;       // [2]
    const GemmArgs& g = P.g;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kStages),
                   accf0 = smem_u32(bars + 2 * kStages), acce0 = smem_u32(bars + 2 * kStages + 2),
                   done = smem_u32(bars + 2 * kStages + 4);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(accf0 + 8 * b, 2);    // the MMA thread's arrive + the MMA commit
            mbar_init(acce0 + 8 * b, 128);  // every epilogue thread
        }
        mbar_init(done, 1);
        *aborted = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(2 * kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int it = 0;  // ring slots used so far
            for (int i = 0;; i++) {
                int x = (tile_ctr ? atomicAdd(tile_ctr, 1) : (int)blockIdx.x + i * (int)gridDim.x) +
                        g.tile_skip;
                if (x >= ntiles) x = -1;
                int z = 0, ti = 0, tj = 0, kb = 0, nk = 0;
                if (x >= 0) {
                    decode_tile(x, g, tm, tn, z, ti, tj);
                    tile_k_range(g, ti, kb, nk);
                }
                const int32_t ax = g.a_c0 + z * g.a_zc + kb, ay = g.a_r0 + z * g.a_zr + ti * kBM;
                const int32_t bx = g.b_c0 + z * g.b_zc + kb, by = g.b_r0 + z * g.b_zr + tj * kBN;
                const int nslots = nk > 0 ? nk : 1;
                bool stop = false;
                for (int k = 0; k < nslots; k++, it++) {
                    const int s = it % kStages;
                    if (it >= kStages &&
                        !mbar_wait(empty0 + 8 * s, ((it / kStages) - 1) & 1, P.err)) {
                        *aborted = 1;
                        stop = true;
                        break;
                    }
                    if (*aborted) {
                        stop = true;
                        break;
                    }
                    const uint32_t fb = full0 + 8 * s;
                    if (k == 0) tileq[s] = x;
                    if (nk == 0) {
                        mbar_arrive(fb);  // the index alone (end of work or an empty K range)
                        continue;
                    }
                    const uint32_t st = smem_u32(smem + s * kStageBytes);
                    mbar_expect_tx(fb, kStageBytes);
                    const int32_t kk = k * kBK;
                    tma_load_2d(st, &a_hi, fb, ax + kk, ay);
                    tma_load_2d(st + kTileBytes, &a_lo, fb, ax + kk, ay);
                    tma_load_2d(st + 2 * kTileBytes, &b_hi, fb, bx + kk, by);
                    tma_load_2d(st + 3 * kTileBytes, &b_lo, fb, bx + kk, by);
                }
                if (stop || x < 0) break;
            }
            // every copy issued has landed before the CTA may exit
            for (int j = it > kStages ? it - kStages : 0; j < it; j++)
                mbar_wait(full0 + 8 * (j % kStages), (j / kStages) & 1, P.err);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            int it = 0;
            bool any = false;
            for (int i = 0;; i++) {
                const int b = i & 1;
                int s = it % kStages;
                if (!mbar_wait(full0 + 8 * s, (it / kStages) & 1, P.err)) {
                    *aborted = 1;
                    break;
                }
                const int x = tileq[s];
                if (i >= 2 && !mbar_wait(acce0 + 8 * b, ((i >> 1) - 1) & 1, P.err)) {
                    *aborted = 1;
                    break;
                }
                accq[b] = x;
                mbar_arrive(accf0 + 8 * b);  // publishes accq[b]
                int z = 0, ti = 0, tj = 0, kb = 0, nk = 0;
                if (x >= 0) {
                    decode_tile(x, g, tm, tn, z, ti, tj);
                    tile_k_range(g, ti, kb, nk);
                }
                if (nk == 0) {
                    mbar_arrive(empty0 + 8 * s);
                    mbar_arrive(accf0 + 8 * b);
                    it++;
                    if (x < 0) break;
                    continue;
                }
                const uint32_t d = tmem + (uint32_t)(b * kTmemCols);
                bool stop = false;
                for (int k = 0; k < nk; k++, it++) {
                    s = it % kStages;
                    if (k > 0 && !mbar_wait(full0 + 8 * s, (it / kStages) & 1, P.err)) {
                        *aborted = 1;
                        stop = true;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t st = smem_u32(smem + s * kStageBytes);
#pragma unroll
                    for (int kk = 0; kk < kBK / 8; kk++) {
                        const uint64_t ah = sw128_desc(st + kk * 32);
                        const uint64_t al = sw128_desc(st + kTileBytes + kk * 32);
                        const uint64_t bh = sw128_desc(st + 2 * kTileBytes + kk * 32);
                        const uint64_t bl = sw128_desc(st + 3 * kTileBytes + kk * 32);
                        mma_tf32(d, ah, bh, (k | kk) ? 1u : 0u);
                        mma_tf32(d, ah, bl, 1u);
                        mma_tf32(d, al, bh, 1u);
                    }
                    mma_commit(empty0 + 8 * s);
                    any = true;
                }
                if (stop) break;
                mma_commit(accf0 + 8 * b);
            }
            if (any)
                mma_commit(done);
            else
                mbar_arrive(done);
        }
        __syncwarp();
    } else {
        // epilogue: warps 2-5 own TMEM lane quarters (warp % 4)
        const int q4 = warp & 3;
        const int r = q4 * 32 + lane;
        const bool issuer = threadIdx.x == 64;
        const bool split_out = P.c_lo != nullptr;
        const float alpha = g.alpha;
        int cc = 0;  // staging chunks used so far
        for (int i = 0;; i++) {
            const int b = i & 1;
            if (!mbar_wait(accf0 + 8 * b, (i >> 1) & 1, P.err)) {
                *aborted = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int x = accq[b];
            if (x < 0) break;
            int z, ti, tj, kb, nk;
            decode_tile(x, g, tm, tn, z, ti, tj);
            tile_k_range(g, ti, kb, nk);
            const int32_t x0 = g.c_c0 + z * g.c_zc + tj * kBN, y0 = g.c_r0 + z * g.c_zr + ti * kBM;
            for (int c = 0; c < 4; c++, cc++) {
                float v[32];
                if (nk > 0) {
                    tmem_ld32(tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(b * kTmemCols + 32 * c),
                              v);
                } else {
#pragma unroll
                    for (int e = 0; e < 32; e++) v[e] = 0.0f;
                }
                if (c == 3) {
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    mbar_arrive(acce0 + 8 * b);
                }
                uint8_t* buf = stage_out + (split_out ? 0 : (cc & 1) * kTileBytes);
                if (issuer) {
                    if (split_out)
                        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                    else
                        asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
                }
                epi_sync();
                uint8_t* row_hi = buf + r * 128;
                uint8_t* row_lo = buf + kTileBytes + r * 128;
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int pq = (q ^ (r & 7)) * 16;
                    float4 y = make_float4(alpha * v[4 * q], alpha * v[4 * q + 1],
                                           alpha * v[4 * q + 2], alpha * v[4 * q + 3]);
                    if (split_out) {
                        float4 h, l;
                        split(y.x, h.x, l.x);
                        split(y.y, h.y, l.y);
                        split(y.z, h.z, l.z);
                        split(y.w, h.w, l.w);
                        *reinterpret_cast<float4*>(row_hi + pq) = h;
                        *reinterpret_cast<float4*>(row_lo + pq) = l;
                    } else {
                        *reinterpret_cast<float4*>(row_hi + pq) = y;
                    }
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                epi_sync();
                if (issuer) {
                    const uint32_t src = smem_u32(buf);
                    if (P.tma_epi == 2)
                        tma_reduce_add_2d(&c_hi, src, x0 + 32 * c, y0);
                    else
                        tma_store_2d(&c_hi, src, x0 + 32 * c, y0);
                    if (split_out) tma_store_2d(&c_lo, smem_u32(buf + kTileBytes), x0 + 32 * c, y0);
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                }
            }
            if (*aborted) break;
        }
        if (issuer) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        mbar_wait(done, 0, P.err);  // every MMA issued has completed
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(2 * kTmemCols)
                     : "memory");
    }
}

// ---- one-tile panel solve fused with the next diagonal update ----------------
//
// For diagonal block j (origin j0): L1 = S1 Z^T with S1 = D[j0+128 .., j0 ..]
// (the panel's first row tile, read from the plain FP32 trailing matrix D and
// split in shared memory) and Z = Z[j0 .., j0 ..]; L1 is written split into L,
// kept in shared memory in the MMA operand layout, and
// D[j0+128 .., j0+128 ..] -= L1 L1^T follows as a second product on the same
// CTA (TMA reduce-add into D). 128 threads: warp 0 lane 0 loads, warp 1 lane 0
// issues the MMAs, all four warps split S1 and drain TMEM. Each product is
// hi*hi + hi*lo + lo*hi (3xTF32) in gemm_nt_kernel's order, so the results
// equal a split copy of S1 followed by two gemm_nt launches bit for bit.
// Shared memory (16 KB tiles): 0-3 S1 split in place to hi, 4-7 its lo, 8-11 a
// two-stage ring of Z (hi, lo) boxes; later L1 (hi 0-3, lo 4-7) and the staged
// update (8-11).
static_assert(12 * kTileBytes + 8 * 8 + 2 * 4 + 1023 <= kSmemBytes,
              "chain_tile_kernel: twelve tiles, eight barriers and two words after alignment");

__global__ void __launch_bounds__(128, 1)
chain_tile_kernel(const __grid_constant__ CUtensorMap l_hi, const __grid_constant__ CUtensorMap l_lo,
                  const __grid_constant__ CUtensorMap z_hi, const __grid_constant__ CUtensorMap z_lo,
                  const __grid_constant__ CUtensorMap d_map, int32_t j0, int32_t* err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr int kZS = 2;  // Z ring stages
    // sfull, zfull[2], zempty[2], done1, done2
    uint64_t* bars = (uint64_t*)(smem + 12 * kTileBytes);
    uint32_t* tmem_slot = (uint32_t*)(bars + 8);
    volatile int32_t* aborted = (volatile int32_t*)(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t sfull = smem_u32(bars), zfull0 = smem_u32(bars + 1),
                   zempty0 = smem_u32(bars + 1 + kZS), done1 = smem_u32(bars + 1 + 2 * kZS),
                   done2 = smem_u32(bars + 2 + 2 * kZS);
    constexpr int nk = kBM / kBK;  // K = 128: four boxes of 32 columns
    const int32_t r1 = j0 + kBM;   // rows of L1 (and of the diagonal block it updates)
    if (threadIdx.x == 0) {
        mbar_init(sfull, 1);
        for (int st = 0; st < kZS; st++) {
            mbar_init(zfull0 + 8 * st, 1);
            mbar_init(zempty0 + 8 * st, 1);
        }
        mbar_init(done1, 1);
        mbar_init(done2, 1);
        *aborted = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(2 * kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    auto load_z = [&](int it) {
        const int st = it % kZS;
        const uint32_t fb = zfull0 + 8 * st;
        const uint32_t dz = smem_u32(smem + (8 + 2 * st) * kTileBytes);
        mbar_expect_tx(fb, 2 * kTileBytes);
        tma_load_2d(dz, &z_hi, fb, j0 + it * kBK, j0);
        tma_load_2d(dz + kTileBytes, &z_lo, fb, j0 + it * kBK, j0);
    };
    if (threadIdx.x == 0) {
        mbar_expect_tx(sfull, 4 * kTileBytes);
        for (int b = 0; b < nk; b++)
            tma_load_2d(smem_u32(smem + b * kTileBytes), &d_map, sfull, j0 + b * kBK, r1);
        for (int it = 0; it < kZS; it++) load_z(it);
    }
    // S1 -> (hi in place, lo four tiles on); elementwise, so the swizzle carries over
    bool ok = mbar_wait(sfull, 0, err);
    ok = __syncthreads_and(ok) != 0;
    if (ok) {
        for (int i = threadIdx.x; i < nk * kTileBytes / 16; i += blockDim.x) {
            float4* ph = reinterpret_cast<float4*>(smem) + i;
            float4 x = *ph, h, l;
            split(x.x, h.x, l.x);
            split(x.y, h.y, l.y);
            split(x.z, h.z, l.z);
            split(x.w, h.w, l.w);
            *ph = h;
            *reinterpret_cast<float4*>(smem + nk * kTileBytes + 16 * i) = l;
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();

    // phase 1: L1 = S1 Z^T into TMEM columns 0 .. 127
    if (threadIdx.x == 0) {
        int issued = kZS;
        if (ok) {
            for (int it = kZS; it < nk; it++) {
                const int st = it % kZS;
                if (!mbar_wait(zempty0 + 8 * st, ((it / kZS) - 1) & 1, err)) {
                    *aborted = 1;
                    break;
                }
                if (*aborted) break;
                load_z(it);
                issued = it + 1;
            }
        }
        for (int it = issued - kZS; it < issued; it++)
            mbar_wait(zfull0 + 8 * (it % kZS), (it / kZS) & 1, err);
    } else if (warp == 1 && lane == 0) {
        bool any = false;
        for (int it = 0; ok && it < nk; it++) {
            const int st = it % kZS;
            if (!mbar_wait(zfull0 + 8 * st, (it / kZS) & 1, err)) {
                *aborted = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sh = smem_u32(smem + it * kTileBytes);
            const uint32_t sl = smem_u32(smem + (nk + it) * kTileBytes);
            const uint32_t zh = smem_u32(smem + (8 + 2 * st) * kTileBytes);
#pragma unroll
            for (int kk = 0; kk < kBK / 8; kk++) {
                const uint64_t ah = sw128_desc(sh + kk * 32);
                const uint64_t al = sw128_desc(sl + kk * 32);
                const uint64_t bh = sw128_desc(zh + kk * 32);
                const uint64_t bl = sw128_desc(zh + kTileBytes + kk * 32);
                mma_tf32(tmem, ah, bh, (it | kk) ? 1u : 0u);
                mma_tf32(tmem, ah, bl, 1u);
                mma_tf32(tmem, al, bh, 1u);
            }
            mma_commit(zempty0 + 8 * st);
            any = true;
        }
        if (any)
            mma_commit(done1);
        else
            mbar_arrive(done1);
    }
    __syncwarp();
    __syncthreads();
    ok = mbar_wait(done1, 0, err) && ok;
    ok = __syncthreads_and(ok && !*aborted) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // L1, split, into the freed ring: hi boxes at 0, lo boxes at 4 tiles (128 rows
    // x 32 columns each, 128B-swizzled: the TMA box and the MMA operand layout)
    const int r = warp * 32 + lane;
    if (ok) {
        for (int b = 0; b < 4; b++) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(32 * b), v);
            uint8_t* row_hi = smem + b * kTileBytes + r * 128;
            uint8_t* row_lo = smem + 4 * kTileBytes + b * kTileBytes + r * 128;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int pq = (q ^ (r & 7)) * 16;
                float4 h, l;
                split(v[4 * q], h.x, l.x);
                split(v[4 * q + 1], h.y, l.y);
                split(v[4 * q + 2], h.z, l.z);
                split(v[4 * q + 3], h.w, l.w);
                *reinterpret_cast<float4*>(row_hi + pq) = h;
                *reinterpret_cast<float4*>(row_lo + pq) = l;
            }
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok && threadIdx.x == 0) {
        for (int b = 0; b < 4; b++) {
            tma_store_2d(&l_hi, smem_u32(smem + b * kTileBytes), j0 + 32 * b, r1);
            tma_store_2d(&l_lo, smem_u32(smem + 4 * kTileBytes + b * kTileBytes), j0 + 32 * b, r1);
        }
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    }
    // phase 2: L1 L1^T into TMEM columns 128 .. 255, both operands the staged L1
    if (ok && warp == 1 && lane == 0) {
        const uint32_t d2 = tmem + (uint32_t)kTmemCols;
        for (int b = 0; b < 4; b++) {
            const uint32_t hb = smem_u32(smem + b * kTileBytes);
            const uint32_t lb = smem_u32(smem + 4 * kTileBytes + b * kTileBytes);
#pragma unroll
            for (int kk = 0; kk < kBK / 8; kk++) {
                const uint64_t h = sw128_desc(hb + kk * 32);
                const uint64_t l = sw128_desc(lb + kk * 32);
                mma_tf32(d2, h, h, (b | kk) ? 1u : 0u);
                mma_tf32(d2, h, l, 1u);
                mma_tf32(d2, l, h, 1u);
            }
        }
        mma_commit(done2);
    } else if (!ok && threadIdx.x == 32) {
        mbar_arrive(done2);
    }
    __syncwarp();
    bool ok2 = mbar_wait(done2, 0, err);
    ok2 = __syncthreads_and(ok2 && ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok2) {
        // -L1 L1^T staged after the L1 boxes, then reduce-added into D
        uint8_t* stage = smem + 8 * kTileBytes;
        for (int b = 0; b < 4; b++) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(kTmemCols + 32 * b), v);
            uint8_t* row = stage + b * kTileBytes + r * 128;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int pq = (q ^ (r & 7)) * 16;
                *reinterpret_cast<float4*>(row + pq) =
                    make_float4(-v[4 * q], -v[4 * q + 1], -v[4 * q + 2], -v[4 * q + 3]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        if (ok2) {
            for (int b = 0; b < 4; b++)
                tma_reduce_add_2d(&d_map, smem_u32(smem + 8 * kTileBytes + b * kTileBytes),
                                  r1 + 32 * b, r1);
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(2 * kTmemCols)
                     : "memory");
}

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

bool encode(CUtensorMap* map, float* base, int32_t rows, int32_t cols, int32_t ld) {
    auto enc = encoder();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)kBM};
    cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() { return encoder(); }

bool make_maps(SplitMat& m) {
    m.maps_ok = false;
    if (!m.hi || m.rows <= 0 || m.cols <= 0 || m.ld % 32 != 0 || m.cols > m.ld) return false;
    if (((uintptr_t)m.hi | (uintptr_t)m.lo) & 127) return false;
    if (!encode(&m.map_hi, m.hi, m.rows, m.cols, m.ld)) return false;
    if (m.lo && !encode(&m.map_lo, m.lo, m.rows, m.cols, m.ld)) return false;
    if (!m.lo) m.map_lo = m.map_hi;
    m.maps_ok = true;
    return true;
}

cudaError_t chain_tile(const SplitMat& L, const SplitMat& Z, const SplitMat& D, int32_t j0,
                       int32_t* err, cudaStream_t stream) {
    if (!L.maps_ok || !Z.maps_ok || !D.maps_ok || !L.lo || !Z.lo || D.lo || j0 < 0 || (j0 % kBM) != 0 ||
        j0 + 2 * kBM > L.rows || j0 + kBM > L.cols || j0 + kBM > Z.rows || j0 + kBM > Z.cols ||
        j0 + 2 * kBM > D.rows || j0 + 2 * kBM > D.cols)
        return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(chain_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kSmemBytes);
    if (e != cudaSuccess) return e;
    chain_tile_kernel<<<1, 128, kSmemBytes, stream>>>(L.map_hi, L.map_lo, Z.map_hi, Z.map_lo,
                                                     D.map_hi, j0, err);
    return cudaGetLastError();
}

cudaError_t gemm_nt(const SplitMat& A, const SplitMat& B, SplitMat& C, const GemmArgs& g,
                    int32_t* err, cudaStream_t stream, int32_t max_ctas, int32_t* tile_ctr) {
    if (g.M <= 0 || g.N <= 0 || g.nbatch <= 0) return cudaSuccess;
    // TMA x coordinates must be multiples of 4 FP32 elements (16 bytes); whole
    // K stages only (callers pad to 128).
    if (g.K < 0 || g.K % kBK != 0 || ((g.a_c0 | g.a_zc | g.b_c0 | g.b_zc) & 3) != 0 ||
        g.a_c0 < 0 || g.a_r0 < 0 || g.b_c0 < 0 || g.b_r0 < 0 || g.a_zc < 0 || g.a_zr < 0 ||
        g.b_zc < 0 || g.b_zr < 0 || !C.hi)
        return cudaErrorInvalidValue;
    // every element the epilogue writes lies inside C
    const int64_t last_r = (int64_t)g.c_r0 + (int64_t)(g.nbatch - 1) * g.c_zr + g.M;
    const int64_t last_c = (int64_t)g.c_c0 + (int64_t)(g.nbatch - 1) * g.c_zc + g.N;
    if (g.c_r0 < 0 || g.c_c0 < 0 || g.c_zr < 0 || g.c_zc < 0 || last_r > C.rows || last_c > C.cols)
        return cudaErrorInvalidValue;
    const int tm = (g.M + kBM - 1) / kBM, tn = (g.N + kBN - 1) / kBN;
    dim3 grid;
    if (g.mode & kLowerTiles) {
        if (tm != tn) return cudaErrorInvalidValue;
        grid = dim3((unsigned)(tm * (tm + 1) / 2), 1, (unsigned)g.nbatch);
    } else {
        grid = dim3((unsigned)tn, (unsigned)tm, (unsigned)g.nbatch);
    }
    cudaError_t e = cudaFuncSetAttribute(gemm_nt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kSmemBytes);
    if (e != cudaSuccess) return e;
    KParams P;
    P.g = g;
    P.c_hi = C.hi;
    P.c_lo = C.lo;
    P.ldc = C.ld;
    P.err = err;
    // TMA epilogue for whole tiles: a store when beta == 0, a reduce-add into a
    // plain C when beta == 1; anything else takes the register epilogue.
    P.tma_epi = 0;
    if (C.maps_ok && g.M % kBM == 0 && g.N % kBN == 0 && ((g.c_c0 | g.c_zc) & 3) == 0) {
        if (g.beta == 0.0f)
            P.tma_epi = 1;
        else if (g.beta == 1.0f && !C.lo)
            P.tma_epi = 2;
    }
    const int64_t ntiles = (int64_t)grid.x * grid.y * grid.z;
    const bool persist = max_ctas > 0 && P.tma_epi != 0 && ntiles > 1 && ntiles < (1LL << 30);
    if (g.tile_skip != 0 && (!persist || g.tile_skip < 0 || g.tile_skip >= ntiles))
        return cudaErrorInvalidValue;
    if (persist) {
        e = cudaFuncSetAttribute(gemm_nt_persist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kPSmemBytes);
        if (e != cudaSuccess) return e;
        const unsigned nb = (unsigned)std::min<int64_t>(ntiles - g.tile_skip, max_ctas);
        gemm_nt_persist_kernel<<<nb, kPThreads, kPSmemBytes, stream>>>(
            A.map_hi, A.map_lo, B.map_hi, B.map_lo, C.map_hi, C.map_lo, P, tm, tn, (int32_t)ntiles,
            tile_ctr);
        return cudaGetLastError();
    }
    gemm_nt_kernel<<<grid, 128, kSmemBytes, stream>>>(A.map_hi, A.map_lo, B.map_hi, B.map_lo,
                                                      C.map_hi, C.map_lo, P);
    return cudaGetLastError();
}

}  // namespace tc
}  // namespace tpe
