// Tensor-core (tcgen05, kind::tf32) building blocks of the mixed-precision
// factorization. Matrices are FP32 held as a "split" pair: hi = x rounded to
// TF32 (low 13 mantissa bits zero) and lo = x - hi, exact in FP32, so hi + lo
// reproduces x bit for bit. One product of two split operands is evaluated as
// the three TF32 tensor-core products hi*hi + hi*lo + lo*hi, accumulated in
// FP32 in tensor memory (3xTF32): FP32-level accuracy at tensor-core rate.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tpe {
namespace tc {

constexpr int kBM = 128;  // output tile rows (MMA M, TMEM lanes)
constexpr int kBN = 128;  // output tile columns (MMA N, TMEM columns)
constexpr int kBK = 32;   // K elements per pipeline stage (128 bytes of FP32: one 128B swizzle row)

// Row-major split-FP32 matrix view. ld is a multiple of 32 elements (TMA rows
// start on 16-byte boundaries); rows x cols is the logical extent the tensor
// maps cover (reads outside it return 0).
struct SplitMat {
    float* hi = nullptr;
    float* lo = nullptr;  // null for a plain FP32 output matrix (gemm_nt's C only)
    int32_t rows = 0, cols = 0, ld = 0;
    CUtensorMap map_hi, map_lo;  // 128 x 32 boxes, 128B swizzle
    bool maps_ok = false;
};

// The driver's cuTensorMapEncodeTiled (resolved once; null when unavailable).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// Encodes the tensor maps of m (host only; hi only when lo is null). Returns
// false on failure.
bool make_maps(SplitMat& m);

enum : int32_t {
    kLowerTiles = 1,  // only output tiles with tile column <= tile row (1-D grid)
    kAUpper = 2,      // A[i][k] = 0 for k < i: K range of tile row t starts at t*kBM
    kALower = 4,      // A[i][k] = 0 for k >= i+1: K range of tile row t ends at (t+1)*kBM
};

// C[c_r0+i][c_c0+j] = alpha * sum_{k<K} A[a_r0+i][k0+k] * B[b_r0+j][b_c0+k]
//                     + beta * C[c_r0+i][c_c0+j]      (i < M, j < N)
// for every batch z < nbatch, with all six origins shifted by z * (shift_r, shift_c)
// of their operand. beta == 0 never reads C, so C may alias the A tile a CTA
// reads (each CTA loads its whole A tile before it writes). A C without lo is
// read and written as plain FP32. err (device, may
// be null) is set to 1 when a pipeline wait gives up (no result then).
struct GemmArgs {
    int32_t a_r0 = 0, a_c0 = 0, b_r0 = 0, b_c0 = 0, c_r0 = 0, c_c0 = 0;
    int32_t a_zr = 0, a_zc = 0, b_zr = 0, b_zc = 0, c_zr = 0, c_zc = 0;
    int32_t M = 0, N = 0, K = 0;
    int32_t mode = 0;
    int32_t nbatch = 1;
    float alpha = 1.0f, beta = 0.0f;
    // persistent form only: the first tile_skip output tiles in tile order
    // (packed lower tiles with kLowerTiles, else row-major, batch last) are left out
    int32_t tile_skip = 0;
};

// max_ctas > 0 selects the persistent form (at most max_ctas CTAs, one per SM,
// each walking many tiles) for whole-tile TMA epilogues; tile_ctr (device, may be
// null) is then a zeroed counter the CTAs take tiles from, else tiles go
// round-robin.
// For the diagonal block at row/column j0 (a multiple of 128) of a Cholesky in
// progress on a plain FP32 D: L1 = D[j0+128.., j0..] Z[j0.., j0..]^T, written
// split into L, then D[j0+128.., j0+128..] -= L1 L1^T, by one CTA.
cudaError_t chain_tile(const SplitMat& L, const SplitMat& Z, const SplitMat& D, int32_t j0,
                       int32_t* err, cudaStream_t stream);

cudaError_t gemm_nt(const SplitMat& A, const SplitMat& B, SplitMat& C, const GemmArgs& g,
                    int32_t* err, cudaStream_t stream, int32_t max_ctas = 0,
                    int32_t* tile_ctr = nullptr);

}  // namespace tc
}  // namespace tpe
