// tgb_mlp.cuh -- per-atom energy surrogate of one SOAP block (interfaces).
//
// Network (per ensemble member), on x = (q - mu) / sigma_x:
//   z1 = W1 x + b1, h1 = silu(z1); z2 = W2 h1 + b2, h2 = silu(z2); E = w3 . h2 + b3
// trained on normalised (x, E, dE/dx) triples with the loss
//   L = 1/B sum (E - y)^2 + lam/(B D) sum |dE/dx - Gref|^2
// (second-order back-propagation for the dE/dx term). Every matrix product is a
// tcgen05 GEMM (bf16 operands, fp32 accumulation); the elementwise stages are
// fp32; master weights and Adam moments are fp32.
#pragma once

#include "tgb_gemm.cuh"

#include <vector>

namespace tgb {

struct MlpLayout {
    int D = 0, Dp = 0, H = 0;
    // offsets (floats) of the parameters in a member's flat vector
    size_t oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, ow3 = 0, ob3 = 0, n = 0;
    void set(int d, int h) {
        D = d;
        Dp = (d + 63) / 64 * 64;
        H = h;
        oW1 = 0;
        ob1 = oW1 + (size_t)H * Dp;
        oW2 = ob1 + H;
        ob2 = oW2 + (size_t)H * H;
        ow3 = ob2 + H;
        ob3 = ow3 + H;
        n = (ob3 + 1 + 63) / 64 * 64;
    }
};

struct MlpTrainWork;   // batch buffers and GEMM plans (tgb_mlp.cu)
struct MlpInferWork;   // inference buffers for up to a given number of rows

struct Mlp {
    MlpLayout L;
    int n_members = 0;
    unsigned *err = nullptr;          // device error word of the GEMMs
    // per member (device): fp32 params, grads, Adam moments; bf16 operand copies
    std::vector<float *> P, Gr, Am, Av;
    std::vector<__nv_bfloat16 *> W1b, W1Tb, W2b, W2Tb;
    std::vector<long long> adam_t;
    // normalisation: x = delta / sx, y = (E - muE) / sE
    double sx = 0.0, muE = 0.0, sE = 0.0;
    // data set (device): delta rows [N][D] fp32, energies [N], dE/d(delta) rows [N][D] fp32
    float *dx = nullptr, *dg = nullptr;
    double *de = nullptr;
    long long n_data = 0, cap_data = 0;
    // inference weights of all members (refreshed after training / set)
    __nv_bfloat16 *W1cat = nullptr, *W1Tcat = nullptr;   // [nm H][Dp], [Dp][nm H]
    __nv_bfloat16 *W2cat = nullptr, *W2Tcat = nullptr;   // [nm H][H]: W2, W2^T of member k at row k H
    // [nm H][nm H] block-diagonal W2 and W2^T (zero off the members' blocks), for
    // ensembles whose hidden layers fit one GEMM column tile (mlp_dense_l2)
    __nv_bfloat16 *W2d = nullptr, *W2Td = nullptr;
    float *b1cat = nullptr, *b2cat = nullptr, *w3cat = nullptr, *b3cat = nullptr;
    bool infer_ready = false;
    MlpTrainWork *tw = nullptr;
};

int mlp_create(int dim, int hidden, int n_members, unsigned long long seed, Mlp **out);
void mlp_destroy(Mlp *m);
int mlp_set_member(Mlp &m, int k, const double *W1, const double *b1, const double *W2,
                   const double *b2, const double *w3, double b3);
int mlp_get_member(Mlp &m, int k, double *W1, double *b1, double *W2, double *b2, double *w3,
                   double *b3);
// Append samples already on the device (fp32 delta rows with row stride ldx, FP64
// energies, fp32 dE/d(delta) rows with row stride ldg).
int mlp_append_device(Mlp &m, int n, const float *x, int ldx, const double *e, const float *g,
                      int ldg, cudaStream_t st);
int mlp_train(Mlp &m, int epochs, int batch, double lr, double lam, unsigned long long seed,
              double *loss_per_epoch, cudaStream_t st);
// Loss and gradients (flat layout, FP64 on the host) of one normalised batch for
// one member, without updating it.
int mlp_batch_grads(Mlp &m, int member, int B, const float *x, const float *y, const float *gref,
                    double lam, double *grads, double *loss, float *E, float *G, cudaStream_t st);
// Inference buffers and GEMM plans of one caller (an engine block, a predict
// call): a captured CUDA graph keeps pointing at them, so callers never share.
MlpInferWork *mlp_infer_work_new();
void mlp_infer_work_delete(MlpInferWork *w);
// Inference on bf16 rows X (row stride ldx >= Dp; entries D..Dp-1 are ignored)
// for all members: energy mean and spread (eV) per row, and the member-mean
// dE/d(delta) minus g_sub (per column, may be null) as fp32 rows of length D
// (row stride ldg, a multiple of 4). Every stage is a fused GEMM epilogue.
int mlp_infer(Mlp &m, MlpInferWork &w, int n, const __nv_bfloat16 *X, int ldx, double *e_mean,
              double *e_std, float *g_mean, int ldg, const float *g_sub, cudaStream_t st);
int mlp_check_err(Mlp &m, cudaStream_t st);

}  // namespace tgb
