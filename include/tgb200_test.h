/*
 * tgb200_test.h -- test-only entry points of libtgb200.so.
 *
 * These expose single kernels of the backend so the GPU tests can check them in
 * isolation. They have no counterpart in the reference (TurboGAP has no GPU
 * kernels in its tree) and are not part of the drop-in seam declared in tgb200.h.
 */
#ifndef TGB200_TEST_H
#define TGB200_TEST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C[M x N] (fp32, row-major) = A[M x K] . B[N x K]^T with A, B bf16 (raw uint16
 * bit patterns, row-major, K contiguous) through the tcgen05/TMA GEMM kernel.
 * K must be a multiple of 64. Host pointers. */
int tgx_gemm_bf16_tn(int32_t M, int32_t N, int32_t K, const uint16_t *A, const uint16_t *B,
                     float *C);

#ifdef __cplusplus
}
#endif
#endif
