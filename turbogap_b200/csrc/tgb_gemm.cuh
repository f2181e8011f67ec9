// tgb_gemm.cuh -- tcgen05/TMA GEMM for the GAP kernel (interfaces).
#pragma once

#include "tgb_common.cuh"

#include <cuda.h>

namespace tgb {

// C[M x N] = A[M x K] . B[N x K]^T, A and B bf16 K-major (row-major, K
// contiguous), fp32 accumulation in tensor memory, fused epilogue:
//   EPI_GAP_KERNEL  (GEMM 1 on centred operands, C = (q - mu).(q_s - mu)):
//       K = C + aoff[s] + qoff[row]                          (FP64; the exact rank-1 terms)
//       epart[row][e] = sum_s alpha_s K^zeta                 (FP64)
//       kdsum[row][e] = sum_s kd_s                           (FP64)
//       kd[row][s + t*Mpad] = split(kd_s - kcoef_s) (t = 0: hi, t = 1: lo), kd_s = kcoef_s K^(zeta-1),
//                             kcoef_s = c0 alpha_s, c0 = zeta delta^2 (the K = 1
//                             value is carried exactly by the caller)
//     The partial sums e run over the gemm_n_etiles(Mpad) column slices of
//     kGemmBN / kGemmEpiGroups sparse points; the consumer adds them up.
//   EPI_STORE_F32   (GEMM 2, sum_s (kd_s - kcoef_s)(q_s - mu)): out[row][col] = C
//   EPI_MLP_L1   z = C + p0[col]: bf16(silu z) at column col and bf16(silu' z) at
//                column x2 + col of the store map
//   EPI_MLP_L2   z = C + p0[col]: bf16(p1[col] silu' z) through the store map and the
//                row sums of p1[col] silu z into rowpart[row * rowpart_ld + tile * groups + group]
//                (groups = kGemmMlpEpiGroups)
//   EPI_MLP_L2B  bf16(C * in_b[row][col]) through the store map
//   EPI_MLP_L1B  out[row][col] = scale C - p0[col] (p0 may be null), fp32, cols < cols,
//                through the fp32 store map C (make_tma_store_f32 over out)
enum EpiMode {
    EPI_GAP_KERNEL = 0, EPI_STORE_F32 = 1, EPI_MLP_L1 = 2, EPI_MLP_L2 = 3, EPI_MLP_L2B = 4,
    EPI_MLP_L1B = 5
};

struct GemmEpi {
    int mode;
    int rows;             // valid rows of C (and the rows the launch is sized for)
    const int *rows_dev;  // optional: the valid rows are min(rows, *rows_dev), read on the device
    int bd_block;         // > 0: block-diagonal product; output columns [j b, (j+1) b) use A's
                          // K range [j b, j b + K) (b a multiple of kGemmBN)
    int a_krep;           // > 0: A's logical K column k >= a_krep is read from column k - a_krep
                          // (GEMM 2's [hi | hi | lo] operand stored as [hi | lo])
    int cols;             // valid columns of C
    // EPI_GAP_KERNEL
    const double *alpha;  // [Mpad]
    double c0;            // zeta delta^2
    int zeta_int;         // > 0: integer power; 0: use zeta_f
    double zeta_f;
    double *epart;        // [rows][gemm_n_etiles(Mpad)]
    double *kdsum;        // [rows][gemm_n_etiles(Mpad)]
    const double *aoff;   // [Mpad]: mu . q_s
    const double *qoff;   // [rows]: (q - mu) . mu
    __nv_bfloat16 *kd;    // [rows][K2]
    int K2, Mpad, nsplit;
    // EPI_STORE_F32, EPI_MLP_L1B
    float *out;
    int ldo;
    // EPI_MLP_*
    const float *p0, *p1;           // per-column parameters
    __nv_bfloat16 *out_b0, *out_b1; // bf16 outputs, row stride ldb (unused with a store map)
    int ldb;
    int x2;                         // EPI_MLP_L1: column offset of silu'(z) in the store map
    const __nv_bfloat16 *in_b;      // bf16 elementwise factor, row stride ldi
    int ldi;
    float scale;
    float *rowpart;                 // fp32 row partial sums (EPI_MLP_L2)
    int rowpart_ld;
    // failure test only (tgx_gemm_stall_probe): nonzero makes the producer issue
    // no loads, so the MMA issuer's first bounded wait runs out and every role
    // leaves with DEV_ERR_TIMEOUT_* set; zero in every production launch
    int stall_test;
};

constexpr int kGemmBM = 128;
constexpr int kGemmBN = 256;
constexpr int kGemmBK = 64;
constexpr int kGemmStages = 4;
constexpr int kGemmEpiGroups = 2;   // epilogue warps per TMEM lane quarter (column groups)
constexpr int kGemmMlpEpiGroups = 4;   // the same for the MLP epilogues (EPI_MLP_*)

struct TmaMap {
    alignas(64) CUtensorMap map;
};

// 2-D bf16 tensor map over a row-major [rows x cols] matrix (row stride ld
// elements), box [box_rows x 64], 128-byte swizzle, zero fill out of range.
int make_tma_bf16(TmaMap *m, const void *base, int64_t rows, int64_t cols, int64_t ld,
                  int box_rows);

// 2-D bf16 tensor map for TMA stores of 32 x 32 blocks (64-byte swizzle): the
// GAP epilogue's kd scratch.
int make_tma_store_bf16(TmaMap *m, const void *base, int64_t rows, int64_t cols, int64_t ld);
// fp32 store map: 32 x 32 boxes, 128-byte swizzle (the EPI_MLP_L1B output)
int make_tma_store_f32(TmaMap *m, const void *base, int64_t rows, int64_t cols, int64_t ld);

// C (map for the GAP epilogue's kd stores) is required in EPI_GAP_KERNEL mode.
// Blast, optional: a second map over B whose box is gemm_last_box_rows(N) rows
// tall; the last column tile of an N that is not a multiple of kGemmBN then
// loads and multiplies only those rows instead of a full kGemmBN-row box.
int launch_gemm_tn(const TmaMap &A, const TmaMap &B, int M, int N, int K, const GemmEpi &ep,
                   unsigned *err, cudaStream_t st, const TmaMap *C = nullptr,
                   const TmaMap *Blast = nullptr);

inline int gemm_n_tiles(int N) { return (N + kGemmBN - 1) / kGemmBN; }
// Rows of the last column tile, rounded up to the MMA's N step of 16; 0 when N
// is a multiple of kGemmBN (no short tile).
inline int gemm_last_box_rows(int N) {
    const int r = N % kGemmBN;
    return r == 0 ? 0 : (r + 15) / 16 * 16;
}
// Number of column slices the energy partials are split into.
inline int gemm_n_etiles(int N) { return gemm_n_tiles(N) * kGemmEpiGroups; }

}  // namespace tgb
