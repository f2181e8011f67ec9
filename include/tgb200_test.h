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

/* Failure test: the same GEMM with its TMA producer silenced (zero operands,
 * nothing loaded). The MMA issuer's bounded mbarrier wait runs out after 2 s,
 * the kernel sets its timeout bits and returns, TMEM freed, no fault. Returns
 * TG_ERR_TIMEOUT (and the device error word in *err_word). */
int tgx_gemm_stall_probe(int32_t M, int32_t N, int32_t K, uint32_t *err_word);

/* Failure test, host code only: NCCL communicator initialisation over the id
 * (from tg_nccl_unique_id), one grouped all-reduce without data, destruction.
 * Each step is polled with the deadline of TGB_NCCL_TIMEOUT_S: TG_ERR_TIMEOUT
 * when a rank never arrives. TGB_NCCL_LIBRARY selects the NCCL build. */
int tgx_comm_probe(const void *id128, int32_t n_ranks, int32_t rank);

struct tg_mlp;
/* Loss and parameter gradients of one member on one batch of B normalised
 * samples (x (B, dim), y (B), gref (B, dim) fp32), without updating it. grads
 * uses the flat parameter layout of tgx_mlp_layout; E (B) and G (B, Dp) receive
 * the forward energies and input gradients. */
int tgx_mlp_batch_grads(struct tg_mlp *m, int32_t member, int32_t B, const float *x,
                        const float *y, const float *gref, double lam, double *grads,
                        double *loss, float *E, float *G);
/* offsets[9] = {D, Dp, H, offset of W1, b1, W2, b2, w3, b3} in the flat layout. */
int tgx_mlp_layout(struct tg_mlp *m, int64_t *offsets);

#ifdef __cplusplus
}
#endif
#endif
