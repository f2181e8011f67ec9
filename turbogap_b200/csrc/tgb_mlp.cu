// tgb_mlp.cu -- training and inference of the per-atom energy surrogate.
//
// Every product is the persistent tcgen05 GEMM of tgb_gemm.cu in its "TN" form
// (C = A . B^T, both operands K-major bf16, fp32 out). Back-propagation needs
// products over the batch index, so the elementwise stages also write the
// transposed bf16 copies those products take as operands. Member weights keep
// an fp32 master copy (flat vector, MlpLayout) and bf16 copies W1, W1^T, W2,
// W2^T refreshed after each Adam step.

#include "tgb_mlp.cuh"
#include "tgb_neighbors.cuh"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>

namespace tgb {

namespace {

using bf16 = __nv_bfloat16;

template <class T>
struct Buf {
    T *p = nullptr;
    size_t n = 0;
    int ensure(size_t m) {
        if (m <= n && p) return TG_OK;
        dev_free(p);
        n = 0;
        TGB_TRY(dev_alloc(&p, m));
        n = m;
        return TG_OK;
    }
    ~Buf() { dev_free(p); }
};

inline unsigned blocks_for(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ float sigm(float z) { return 1.f / (1.f + expf(-z)); }
__device__ __forceinline__ float silu_f(float z, float s) { return z * s; }
__device__ __forceinline__ float dsilu_f(float z, float s) { return s * (1.f + z * (1.f - s)); }
__device__ __forceinline__ float d2silu_f(float z, float s) {
    return s * (1.f - s) * (2.f + z * (1.f - 2.f * s));
}

// ---------------------------------------------------------------- data
// Batch b takes sample idx[b]: x = delta * inv_sx (bf16, zero-padded to Dp),
// y = (E - muE) * inv_sE, Gref = dE/d(delta) * gscale (fp32, zero-padded).
__global__ void k_gather(int B, int D, int Dp, const int64_t *__restrict__ idx,
                         const float *__restrict__ X, const double *__restrict__ E,
                         const float *__restrict__ G, float inv_sx, double muE, double inv_sE,
                         float gscale, bf16 *__restrict__ Xb, float *__restrict__ y,
                         float *__restrict__ Gref) {
    const int b = blockIdx.x;
    if (b >= B) return;
    const int64_t s = idx[b];
    for (int d = threadIdx.x; d < Dp; d += blockDim.x) {
        float x = 0.f, g = 0.f;
        if (d < D) {
            x = X[s * D + d] * inv_sx;
            g = G[s * D + d] * gscale;
        }
        Xb[(size_t)b * Dp + d] = __float2bfloat16_rn(x);
        Gref[(size_t)b * Dp + d] = g;
    }
    if (threadIdx.x == 0) y[b] = (float)((E[s] - muE) * inv_sE);
}

// out[c][r] = in[r][c] for an R x C bf16 block (32 x 32 tiles through shared memory)
__global__ void k_transpose(int R, int C, const bf16 *__restrict__ in, int ldi, bf16 *__restrict__ out,
                            int ldo) {
    __shared__ bf16 t[32][34];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < R && c < C) t[k][threadIdx.x] = in[(size_t)r * ldi + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < R && c < C) out[(size_t)c * ldo + r] = t[threadIdx.x][k];
    }
}

// ---------------------------------------------------------------- training stages
__global__ void k_act1(int n, int H, const float *__restrict__ Z1, const float *__restrict__ b1,
                       bf16 *__restrict__ H1, float *__restrict__ S1, float *__restrict__ T1) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * H) return;
    const float z = Z1[i] + b1[i % H], s = sigm(z);
    H1[i] = __float2bfloat16_rn(silu_f(z, s));
    S1[i] = dsilu_f(z, s);
    T1[i] = d2silu_f(z, s);
}

// one warp per row: h2, silu', silu'', u2 = w3 silu'(z2) (bf16) and E = w3.h2 + b3
__global__ void k_act2(int B, int H, const float *__restrict__ Z2, const float *__restrict__ b2,
                       const float *__restrict__ w3, const float *__restrict__ b3,
                       float *__restrict__ H2, float *__restrict__ S2, float *__restrict__ T2,
                       bf16 *__restrict__ U2, float *__restrict__ E) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= B) return;
    float acc = 0.f;
    for (int j = lane; j < H; j += 32) {
        const size_t i = (size_t)row * H + j;
        const float z = Z2[i] + b2[j], s = sigm(z), h = silu_f(z, s), sp = dsilu_f(z, s);
        H2[i] = h;
        S2[i] = sp;
        T2[i] = d2silu_f(z, s);
        U2[i] = __float2bfloat16_rn(sp * w3[j]);
        acc += h * w3[j];
    }
    acc = warp_sum(acc);
    if (lane == 0) E[row] = acc + b3[0];
}

__global__ void k_mul_bf16(int64_t n, const float *__restrict__ a, const float *__restrict__ b,
                           bf16 *__restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = __float2bfloat16_rn(a[i] * b[i]);
}

// one warp per row: R = 2 lam (G - Gref) / (B D) (bf16, zero beyond D), e = 2 (E - y) / B,
// loss parts accumulated in FP64
__global__ void k_loss(int B, int D, int Dp, const float *__restrict__ G,
                       const float *__restrict__ Gref, const float *__restrict__ E,
                       const float *__restrict__ y, float lam, bf16 *__restrict__ R,
                       float *__restrict__ e, double *__restrict__ loss2) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= B) return;
    const float scale = 2.f * lam / ((float)B * (float)D);
    double acc = 0.0;
    for (int d = lane; d < Dp; d += 32) {
        float r = 0.f;
        if (d < D) {
            const float df = G[(size_t)row * Dp + d] - Gref[(size_t)row * Dp + d];
            acc += (double)df * df;
            r = scale * df;
        }
        R[(size_t)row * Dp + d] = __float2bfloat16_rn(r);
    }
    acc = warp_sum(acc);
    if (lane == 0) {
        const float de = E[row] - y[row];
        e[row] = 2.f * de / (float)B;
        atomicAdd(&loss2[0], (double)de * de / B);
        atomicAdd(&loss2[1], (double)lam * acc / ((double)B * D));
    }
}

__global__ void k_bw1(int64_t n, const float *__restrict__ A1, const float *__restrict__ S1,
                      const float *__restrict__ V1, const float *__restrict__ T1,
                      bf16 *__restrict__ dV1, float *__restrict__ dZ1p) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float a = A1[i];
    dV1[i] = __float2bfloat16_rn(a * S1[i]);
    dZ1p[i] = a * V1[i] * T1[i];
}

constexpr int kRowsPerBlock = 32;

// thread j owns column j over kRowsPerBlock rows: dz2 (bf16) and the column sums
// of dw3, db2 (db3 from thread 0), accumulated into the fp32 gradient vector
__global__ void k_bw2(int B, int H, const float *__restrict__ dU2, const float *__restrict__ S2,
                      const float *__restrict__ T2, const float *__restrict__ H2,
                      const float *__restrict__ w3, const float *__restrict__ e,
                      bf16 *__restrict__ dZ2, float *__restrict__ gw3, float *__restrict__ gb2,
                      float *__restrict__ gb3) {
    const int j = threadIdx.x;
    const int r0 = blockIdx.x * kRowsPerBlock, r1 = min(B, r0 + kRowsPerBlock);
    if (j < H) {
        const float w = w3[j];
        float aw = 0.f, ab = 0.f;
        for (int b = r0; b < r1; ++b) {
            const size_t i = (size_t)b * H + j;
            const float du = dU2[i], s = S2[i], eb = e[b];
            const float dz = du * w * T2[i] + eb * w * s;
            dZ2[i] = __float2bfloat16_rn(dz);
            aw += du * s + eb * H2[i];
            ab += dz;
        }
        atomicAdd(gw3 + j, aw);
        atomicAdd(gb2 + j, ab);
    }
    if (j == 0) {
        float s = 0.f;
        for (int b = r0; b < r1; ++b) s += e[b];
        atomicAdd(gb3, s);
    }
}

__global__ void k_bw3(int B, int H, const float *__restrict__ dH1, const float *__restrict__ S1,
                      const float *__restrict__ dZ1p, bf16 *__restrict__ dZ1,
                      float *__restrict__ gb1) {
    const int j = threadIdx.x;
    if (j >= H) return;
    const int r0 = blockIdx.x * kRowsPerBlock, r1 = min(B, r0 + kRowsPerBlock);
    float ab = 0.f;
    for (int b = r0; b < r1; ++b) {
        const size_t i = (size_t)b * H + j;
        const float dz = dH1[i] * S1[i] + dZ1p[i];
        dZ1[i] = __float2bfloat16_rn(dz);
        ab += dz;
    }
    atomicAdd(gb1 + j, ab);
}

__global__ void k_adam(int64_t n, float *__restrict__ p, const float *__restrict__ g,
                       float *__restrict__ m, float *__restrict__ v, float lr, float b1, float b2,
                       float bc1, float bc2, float eps) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// bf16 operand copies of one member: W1 [H][Dp], W1^T [Dp][H], W2 [H][H], W2^T [H][H]
__global__ void k_refresh(const float *__restrict__ P, MlpLayout L, bf16 *__restrict__ W1b,
                          bf16 *__restrict__ W1Tb, bf16 *__restrict__ W2b, bf16 *__restrict__ W2Tb) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t n1 = (int64_t)L.H * L.Dp, n2 = (int64_t)L.H * L.H;
    if (i < n1) {
        const int r = (int)(i / L.Dp), c = (int)(i % L.Dp);
        const bf16 v = __float2bfloat16_rn(P[L.oW1 + i]);
        W1b[i] = v;
        W1Tb[(size_t)c * L.H + r] = v;
    } else if (i < n1 + n2) {
        const int64_t k = i - n1;
        const int r = (int)(k / L.H), c = (int)(k % L.H);
        const bf16 v = __float2bfloat16_rn(P[L.oW2 + k]);
        W2b[k] = v;
        W2Tb[(size_t)c * L.H + r] = v;
    }
}

// inference copy of member k: W1 / sx into rows k H .. of W1cat and columns of
// W1Tcat; W2 and W2^T into rows k H .. of W2cat, W2Tcat; biases; w3 sE; b3 sE + muE
__global__ void k_refresh_infer(const float *__restrict__ P, MlpLayout L, int k, int nm, float inv_sx,
                                float sE, float muE, bf16 *__restrict__ W1cat,
                                bf16 *__restrict__ W1Tcat, bf16 *__restrict__ W2cat,
                                bf16 *__restrict__ W2Tcat, float *__restrict__ b1cat,
                                float *__restrict__ b2cat, float *__restrict__ w3cat,
                                float *__restrict__ b3cat, bf16 *__restrict__ W2d,
                                bf16 *__restrict__ W2Td) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t n1 = (int64_t)L.H * L.Dp, n2 = (int64_t)L.H * L.H;
    const int HH = nm * L.H;
    if (i >= n1 + L.H && i < n1 + L.H + n2) {
        const int64_t q = i - n1 - L.H;
        const int r = (int)(q / L.H), c = (int)(q % L.H);
        const bf16 v = __float2bfloat16_rn(P[L.oW2 + q]);
        W2cat[((size_t)k * L.H + r) * L.H + c] = v;
        W2Tcat[((size_t)k * L.H + c) * L.H + r] = v;
        if (W2d) {   // member k's diagonal block; the rest was zeroed
            W2d[((size_t)k * L.H + r) * HH + k * L.H + c] = v;
            W2Td[((size_t)k * L.H + c) * HH + k * L.H + r] = v;
        }
    } else if (i < n1) {
        const int r = (int)(i / L.Dp), c = (int)(i % L.Dp);
        const bf16 v = __float2bfloat16_rn(c < L.D ? P[L.oW1 + i] * inv_sx : 0.f);
        W1cat[(size_t)(k * L.H + r) * L.Dp + c] = v;
        W1Tcat[(size_t)c * HH + k * L.H + r] = v;
    } else if (i < n1 + L.H) {
        const int j = (int)(i - n1);
        b1cat[k * L.H + j] = P[L.ob1 + j];
        b2cat[k * L.H + j] = P[L.ob2 + j];
        w3cat[k * L.H + j] = P[L.ow3 + j] * sE;
        if (j == 0) b3cat[k] = P[L.ob3] * sE + muE;
    }
}

// ---------------------------------------------------------------- inference stages
// One thread per row: member energies from the layer-2 epilogue's row partials
// (E_k = sum_t part[row][k][t] + b3_k), their mean and spread (FP64).
__global__ void k_i_energy(int n, int nm, int npart, const float *__restrict__ part,
                           const float *__restrict__ b3, double *__restrict__ e_mean,
                           double *__restrict__ e_std) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    double Ek[8], s = 0.0;
    for (int k = 0; k < nm; ++k) {
        double e = b3[k];
        for (int t = 0; t < npart; ++t) e += part[((size_t)row * nm + k) * npart + t];
        Ek[k] = e;
        s += e;
    }
    const double mean = s / nm;
    double s2 = 0.0;
    for (int k = 0; k < nm; ++k) s2 += (Ek[k] - mean) * (Ek[k] - mean);
    e_mean[row] = mean;
    if (e_std) e_std[row] = sqrt(s2 / nm);
}

// moments of the data set for the normalisation: sum x^2 (all entries), sum E, sum E^2
__global__ void k_moments(int64_t nx, const float *__restrict__ x, int64_t ne,
                          const double *__restrict__ e, double *__restrict__ out3) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nx;
         i += (int64_t)gridDim.x * blockDim.x)
        a += (double)x[i] * x[i];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ne;
         i += (int64_t)gridDim.x * blockDim.x) {
        b += e[i];
        c += e[i] * e[i];
    }
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out3, a);
        atomicAdd(out3 + 1, b);
        atomicAdd(out3 + 2, c);
    }
}

__global__ void k_copy_rows(int n, int D, const float *__restrict__ x, int ldx, float *__restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * D) return;
    const int64_t r = i / D;
    out[i] = x[r * ldx + (i - r * D)];
}

// ---------------------------------------------------------------- GEMM plans
struct Plan {
    TmaMap a{}, b{}, c{};   // c: store map of the staged bf16 epilogues
    bool has_c = false;
    int M = 0, N = 0, K = 0;
    GemmEpi ep{};
};

// C[M x N] = A . B^T (K-major bf16, row strides lda / ldb); fp32 store epilogue
// into out (row stride ldo) unless the caller replaces p.ep afterwards.
int plan(Plan &p, const bf16 *A, int M, int lda, const bf16 *Bm, int N, int ldb, int K, float *out,
         int ldo) {
    TGB_TRY(make_tma_bf16(&p.a, A, M, K, lda, kGemmBM));
    TGB_TRY(make_tma_bf16(&p.b, Bm, N, K, ldb, kGemmBN));
    p.M = M;
    p.N = N;
    p.K = K;
    p.ep = GemmEpi{};
    p.ep.mode = EPI_STORE_F32;
    p.ep.rows = M;
    p.ep.cols = N;
    p.ep.out = out;
    p.ep.ldo = ldo;
    return TG_OK;
}

int run(const Plan &p, unsigned *err, cudaStream_t st) {
    return launch_gemm_tn(p.a, p.b, p.M, p.N, p.K, p.ep, err, st, p.has_c ? &p.c : nullptr);
}

// bf16 output of a staged epilogue: rows x cols at base, row stride ld
int plan_store(Plan &p, const bf16 *base, int rows, int cols, int ld) {
    TGB_TRY(make_tma_store_bf16(&p.c, base, rows, cols, ld));
    p.has_c = true;
    return TG_OK;
}

int transpose(int R, int C, const bf16 *in, int ldi, bf16 *out, int ldo, cudaStream_t st) {
    dim3 g((C + 31) / 32, (R + 31) / 32), b(32, 8);
    k_transpose<<<g, b, 0, st>>>(R, C, in, ldi, out, ldo);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

}  // namespace

// Batch buffers of one training step (shared by the members, which run in turn)
// and the GEMM plans of every member.
struct MlpTrainWork {
    int B = 0;
    Buf<int64_t> idx;
    Buf<bf16> Xb, H1, U2, U1, R, dV1, dZ2, dZ1, AW2, BW2, AW1, BW1;
    Buf<float> y, Gref, Z1, S1, T1, Z2, H2, S2, T2, E, V1, G, A1, dZ1p, dU2, dH1, e;
    Buf<double> loss2;
    std::vector<Plan> pZ1, pZ2, pV1, pG, pA1, pdU2, pdH1, pdW2, pdW1;

    int ensure(Mlp &m, int b) {
        if (B == b) return TG_OK;
        const int H = m.L.H, Dp = m.L.Dp;
        const size_t bh = (size_t)b * H, bd = (size_t)b * Dp;
        TGB_TRY(idx.ensure(b));
        TGB_TRY(Xb.ensure(bd)); TGB_TRY(H1.ensure(bh)); TGB_TRY(U2.ensure(bh));
        TGB_TRY(U1.ensure(bh)); TGB_TRY(R.ensure(bd)); TGB_TRY(dV1.ensure(bh));
        TGB_TRY(dZ2.ensure(bh)); TGB_TRY(dZ1.ensure(bh));
        TGB_TRY(AW2.ensure((size_t)H * 2 * b)); TGB_TRY(BW2.ensure((size_t)H * 2 * b));
        TGB_TRY(AW1.ensure((size_t)H * 2 * b)); TGB_TRY(BW1.ensure((size_t)Dp * 2 * b));
        TGB_TRY(y.ensure(b)); TGB_TRY(Gref.ensure(bd)); TGB_TRY(Z1.ensure(bh));
        TGB_TRY(S1.ensure(bh)); TGB_TRY(T1.ensure(bh)); TGB_TRY(Z2.ensure(bh));
        TGB_TRY(H2.ensure(bh)); TGB_TRY(S2.ensure(bh)); TGB_TRY(T2.ensure(bh));
        TGB_TRY(E.ensure(b)); TGB_TRY(V1.ensure(bh)); TGB_TRY(G.ensure(bd));
        TGB_TRY(A1.ensure(bh)); TGB_TRY(dZ1p.ensure(bh)); TGB_TRY(dU2.ensure(bh));
        TGB_TRY(dH1.ensure(bh)); TGB_TRY(e.ensure(b)); TGB_TRY(loss2.ensure(2));
        const int nm = m.n_members;
        for (auto *v : {&pZ1, &pZ2, &pV1, &pG, &pA1, &pdU2, &pdH1, &pdW2, &pdW1}) v->assign(nm, Plan{});
        for (int k = 0; k < nm; ++k) {
            float *gr = m.Gr[k];
            TGB_TRY(plan(pZ1[k], Xb.p, b, Dp, m.W1b[k], H, Dp, Dp, Z1.p, H));
            TGB_TRY(plan(pZ2[k], H1.p, b, H, m.W2b[k], H, H, H, Z2.p, H));
            TGB_TRY(plan(pV1[k], U2.p, b, H, m.W2Tb[k], H, H, H, V1.p, H));
            TGB_TRY(plan(pG[k], U1.p, b, H, m.W1Tb[k], Dp, H, H, G.p, Dp));
            TGB_TRY(plan(pA1[k], R.p, b, Dp, m.W1b[k], H, Dp, Dp, A1.p, H));
            TGB_TRY(plan(pdU2[k], dV1.p, b, H, m.W2b[k], H, H, H, dU2.p, H));
            TGB_TRY(plan(pdH1[k], dZ2.p, b, H, m.W2Tb[k], H, H, H, dH1.p, H));
            TGB_TRY(plan(pdW2[k], AW2.p, H, 2 * b, BW2.p, H, 2 * b, 2 * b, gr + m.L.oW2, H));
            TGB_TRY(plan(pdW1[k], AW1.p, H, 2 * b, BW1.p, Dp, 2 * b, 2 * b, gr + m.L.oW1, Dp));
        }
        B = b;
        return TG_OK;
    }
};

// Layer 2 and its adjoint as one GEMM each over a dense block-diagonal weight
// (every member's hidden columns in one column tile) when the members' columns
// are not whole tiles but all of them fit one: one launch instead of one per
// member, and every epilogue warp busy. The layer-2 epilogue's row partials then
// come one per 64-column group, H / 64 of them per member.
static bool mlp_dense_l2(const Mlp &m) {
    const int HH = m.n_members * m.L.H;
    return m.L.H % kGemmBN != 0 && HH <= kGemmBN && m.L.H % (kGemmBN / kGemmMlpEpiGroups) == 0;
}

struct MlpInferWork {
    int cap = 0;
    // binding of the current plans
    const bf16 *X = nullptr;
    int n = 0, ldx = 0, ldg = 0;
    float *g = nullptr;
    const float *sub = nullptr;
    Buf<bf16> HS, U2, U1;   // HS: [rows][2 HH] = h1 | silu'(z1)
    Buf<float> part;
    Plan p1, p4;
    std::vector<Plan> p2, p3;

    int npart(const Mlp &m) const {
        return mlp_dense_l2(m) ? m.L.H / (kGemmBN / kGemmMlpEpiGroups)
                               : gemm_n_tiles(m.L.H) * kGemmMlpEpiGroups;
    }

    int ensure(Mlp &m, int rows) {
        if (rows > cap) {
            const size_t hh = (size_t)m.n_members * m.L.H;
            TGB_TRY(HS.ensure(rows * 2 * hh));
            TGB_TRY(U2.ensure(rows * hh)); TGB_TRY(U1.ensure(rows * hh));
            TGB_TRY(part.ensure((size_t)rows * m.n_members * npart(m)));
            cap = rows;
            X = nullptr;
        }
        return TG_OK;
    }
    // GEMM plans with their fused epilogues for input rows X and output rows g
    int bind(Mlp &m, const bf16 *x, int rows, int ld, float *gout, int ldgo, const float *s) {
        if (x == X && rows == n && ld == ldx && gout == g && ldgo == ldg && s == sub) return TG_OK;
        const int H = m.L.H, Dp = m.L.Dp, nm = m.n_members, HH = nm * H, np = npart(m);
        TGB_TRY(plan(p1, x, rows, ld, m.W1cat, HH, Dp, Dp, nullptr, 0));
        p1.ep.mode = EPI_MLP_L1;
        p1.ep.p0 = m.b1cat;
        p1.ep.x2 = HH;
        TGB_TRY(plan_store(p1, HS.p, rows, 2 * HH, 2 * HH));
        // layer 2 and its adjoint: one block-diagonal launch over all members when a
        // member's columns are whole tiles, else one launch per member
        const bool bd = H % kGemmBN == 0, dense = mlp_dense_l2(m);
        const int nl = (bd || dense) ? 1 : nm;
        p2.assign(nl, Plan{});
        p3.assign(nl, Plan{});
        if (dense) {
            TGB_TRY(plan(p2[0], HS.p, rows, 2 * HH, m.W2d, HH, HH, HH, nullptr, 0));
            p2[0].ep.mode = EPI_MLP_L2;
            p2[0].ep.p0 = m.b2cat;
            p2[0].ep.p1 = m.w3cat;
            p2[0].ep.rowpart = part.p;
            p2[0].ep.rowpart_ld = nm * np;
            TGB_TRY(plan_store(p2[0], U2.p, rows, HH, HH));
            TGB_TRY(plan(p3[0], U2.p, rows, HH, m.W2Td, HH, HH, HH, nullptr, 0));
            p3[0].ep.mode = EPI_MLP_L2B;
            p3[0].ep.in_b = HS.p + HH;
            p3[0].ep.ldi = 2 * HH;
            TGB_TRY(plan_store(p3[0], U1.p, rows, HH, HH));
        } else if (bd) {
            // the A maps span every member's columns: tile column j reads K range [j H, j H + H)
            TGB_TRY(plan(p2[0], HS.p, rows, 2 * HH, m.W2cat, HH, H, H, nullptr, 0));
            TGB_TRY(make_tma_bf16(&p2[0].a, HS.p, rows, HH, 2 * HH, kGemmBM));
            p2[0].ep.mode = EPI_MLP_L2;
            p2[0].ep.bd_block = H;
            p2[0].ep.p0 = m.b2cat;
            p2[0].ep.p1 = m.w3cat;
            p2[0].ep.rowpart = part.p;
            p2[0].ep.rowpart_ld = nm * np;
            TGB_TRY(plan_store(p2[0], U2.p, rows, HH, HH));
            TGB_TRY(plan(p3[0], U2.p, rows, HH, m.W2Tcat, HH, H, H, nullptr, 0));
            TGB_TRY(make_tma_bf16(&p3[0].a, U2.p, rows, HH, HH, kGemmBM));
            p3[0].ep.mode = EPI_MLP_L2B;
            p3[0].ep.bd_block = H;
            p3[0].ep.in_b = HS.p + HH;
            p3[0].ep.ldi = 2 * HH;
            TGB_TRY(plan_store(p3[0], U1.p, rows, HH, HH));
        }
        for (int k = 0; k < nm && !bd && !dense; ++k) {
            TGB_TRY(plan(p2[k], HS.p + k * H, rows, 2 * HH, m.W2b[k], H, H, H, nullptr, 0));
            p2[k].ep.mode = EPI_MLP_L2;
            p2[k].ep.p0 = m.b2cat + k * H;
            p2[k].ep.p1 = m.w3cat + k * H;
            p2[k].ep.rowpart = part.p + (size_t)k * np;
            p2[k].ep.rowpart_ld = nm * np;
            TGB_TRY(plan_store(p2[k], U2.p + k * H, rows, H, HH));
            TGB_TRY(plan(p3[k], U2.p + k * H, rows, HH, m.W2Tb[k], H, H, H, nullptr, 0));
            p3[k].ep.mode = EPI_MLP_L2B;
            p3[k].ep.in_b = HS.p + HH + k * H;
            p3[k].ep.ldi = 2 * HH;
            TGB_TRY(plan_store(p3[k], U1.p + k * H, rows, H, HH));
        }
        TGB_TRY(plan(p4, U1.p, rows, HH, m.W1Tcat, m.L.D, HH, HH, gout, ldgo));
        p4.ep.mode = EPI_MLP_L1B;
        p4.ep.scale = 1.f / (float)nm;
        p4.ep.p0 = s;
        TGB_TRY(make_tma_store_f32(&p4.c, gout, rows, m.L.D, ldgo));
        p4.has_c = true;
        X = x;
        n = rows;
        ldx = ld;
        g = gout;
        ldg = ldgo;
        sub = s;
        return TG_OK;
    }
};

// ---------------------------------------------------------------- host API
int mlp_create(int dim, int hidden, int n_members, unsigned long long seed, Mlp **out) {
    TGB_CHECK(out, TG_ERR_ARG, "null output");
    *out = nullptr;
    TGB_CHECK(dim >= 1 && hidden >= 64 && hidden % 64 == 0 && hidden <= 1024, TG_ERR_ARG,
              "MLP sizes: dim >= 1, hidden a multiple of 64 up to 1024 (got %d, %d)", dim, hidden);
    TGB_CHECK(n_members >= 1 && n_members <= 8, TG_ERR_ARG, "1..8 ensemble members (got %d)",
              n_members);
    auto *m = new Mlp();
    m->L.set(dim, hidden);
    m->n_members = n_members;
    const MlpLayout &L = m->L;
    int rc = dev_alloc(&m->err, 1);
    if (rc == TG_OK) rc = cudaMemset(m->err, 0, sizeof(unsigned)) == cudaSuccess ? TG_OK : TG_ERR_CUDA;
    for (int k = 0; k < n_members && rc == TG_OK; ++k) {
        float *p = nullptr, *g = nullptr, *a = nullptr, *v = nullptr;
        bf16 *w1 = nullptr, *w1t = nullptr, *w2 = nullptr, *w2t = nullptr;
        rc = dev_alloc(&p, L.n);
        if (rc == TG_OK) rc = dev_alloc(&g, L.n);
        if (rc == TG_OK) rc = dev_alloc(&a, L.n);
        if (rc == TG_OK) rc = dev_alloc(&v, L.n);
        if (rc == TG_OK) rc = dev_alloc(&w1, (size_t)L.H * L.Dp);
        if (rc == TG_OK) rc = dev_alloc(&w1t, (size_t)L.H * L.Dp);
        if (rc == TG_OK) rc = dev_alloc(&w2, (size_t)L.H * L.H);
        if (rc == TG_OK) rc = dev_alloc(&w2t, (size_t)L.H * L.H);
        m->P.push_back(p); m->Gr.push_back(g); m->Am.push_back(a); m->Av.push_back(v);
        m->W1b.push_back(w1); m->W1Tb.push_back(w1t); m->W2b.push_back(w2); m->W2Tb.push_back(w2t);
        m->adam_t.push_back(0);
    }
    const size_t HH = (size_t)n_members * L.H;
    if (rc == TG_OK) rc = dev_alloc(&m->W1cat, HH * L.Dp);
    if (rc == TG_OK) rc = dev_alloc(&m->W1Tcat, HH * L.Dp);
    if (rc == TG_OK) rc = dev_alloc(&m->W2cat, HH * L.H);
    if (rc == TG_OK) rc = dev_alloc(&m->W2Tcat, HH * L.H);
    if (rc == TG_OK && mlp_dense_l2(*m)) rc = dev_alloc(&m->W2d, HH * HH);
    if (rc == TG_OK && mlp_dense_l2(*m)) rc = dev_alloc(&m->W2Td, HH * HH);
    if (rc == TG_OK) rc = dev_alloc(&m->b1cat, HH);
    if (rc == TG_OK) rc = dev_alloc(&m->b2cat, HH);
    if (rc == TG_OK) rc = dev_alloc(&m->w3cat, HH);
    if (rc == TG_OK) rc = dev_alloc(&m->b3cat, (size_t)n_members);
    if (rc != TG_OK) {
        mlp_destroy(m);
        return rc;
    }
    // He-style initialisation, one seeded stream per member
    std::vector<double> W1((size_t)L.H * L.D), b1(L.H), W2((size_t)L.H * L.H), b2(L.H), w3(L.H);
    for (int k = 0; k < n_members; ++k) {
        std::mt19937_64 gen(seed * 1000003ull + (unsigned long long)k * 7919ull + 17ull);
        std::normal_distribution<double> nd(0.0, 1.0);
        const double s1 = std::sqrt(1.0 / L.D), s2 = std::sqrt(1.0 / L.H);
        for (auto &x : W1) x = s1 * nd(gen);
        for (auto &x : b1) x = 0.1 * nd(gen);
        for (auto &x : W2) x = s2 * nd(gen);
        for (auto &x : b2) x = 0.1 * nd(gen);
        for (auto &x : w3) x = s2 * nd(gen);
        rc = mlp_set_member(*m, k, W1.data(), b1.data(), W2.data(), b2.data(), w3.data(), 0.0);
        if (rc != TG_OK) {
            mlp_destroy(m);
            return rc;
        }
    }
    *out = m;
    return TG_OK;
}

void mlp_destroy(Mlp *m) {
    if (!m) return;
    cudaDeviceSynchronize();
    for (auto *v : {&m->P, &m->Gr, &m->Am, &m->Av})
        for (auto &p : *v) dev_free(p);
    for (auto *v : {&m->W1b, &m->W1Tb, &m->W2b, &m->W2Tb})
        for (auto &p : *v) dev_free(p);
    dev_free(m->W1cat); dev_free(m->W1Tcat); dev_free(m->W2cat); dev_free(m->W2Tcat);
    dev_free(m->W2d); dev_free(m->W2Td);
    dev_free(m->b1cat); dev_free(m->b2cat);
    dev_free(m->w3cat); dev_free(m->b3cat); dev_free(m->dx); dev_free(m->dg); dev_free(m->de);
    dev_free(m->err);
    delete m->tw;
    delete m;
}

static int refresh_member(Mlp &m, int k, cudaStream_t st) {
    const MlpLayout &L = m.L;
    const int64_t n = (int64_t)L.H * L.Dp + (int64_t)L.H * L.H;
    k_refresh<<<blocks_for(n), 256, 0, st>>>(m.P[k], L, m.W1b[k], m.W1Tb[k], m.W2b[k], m.W2Tb[k]);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

// inference weights of every member from the current normalisation
static int refresh_infer(Mlp &m, cudaStream_t st) {
    const MlpLayout &L = m.L;
    const double sx = m.sx > 0 ? m.sx : 1.0, sE = m.sE > 0 ? m.sE : 1.0;
    const int64_t n = (int64_t)L.H * L.Dp + L.H + (int64_t)L.H * L.H;
    if (m.W2d) {
        const size_t hh = (size_t)m.n_members * L.H;
        TGB_CUDA(cudaMemsetAsync(m.W2d, 0, sizeof(bf16) * hh * hh, st));
        TGB_CUDA(cudaMemsetAsync(m.W2Td, 0, sizeof(bf16) * hh * hh, st));
    }
    for (int k = 0; k < m.n_members; ++k) {
        k_refresh_infer<<<blocks_for(n), 256, 0, st>>>(m.P[k], L, k, m.n_members, (float)(1.0 / sx),
                                                       (float)sE, (float)m.muE, m.W1cat, m.W1Tcat,
                                                       m.W2cat, m.W2Tcat, m.b1cat, m.b2cat,
                                                       m.w3cat, m.b3cat, m.W2d, m.W2Td);
        TGB_CUDA(cudaGetLastError());
    }
    m.infer_ready = true;
    return TG_OK;
}

int mlp_set_member(Mlp &m, int k, const double *W1, const double *b1, const double *W2,
                   const double *b2, const double *w3, double b3) {
    TGB_CHECK(k >= 0 && k < m.n_members, TG_ERR_ARG, "member %d out of range", k);
    TGB_CHECK(W1 && b1 && W2 && b2 && w3, TG_ERR_ARG, "null weights");
    const MlpLayout &L = m.L;
    std::vector<float> h(L.n, 0.f);
    for (int i = 0; i < L.H; ++i)
        for (int d = 0; d < L.D; ++d) h[L.oW1 + (size_t)i * L.Dp + d] = (float)W1[(size_t)i * L.D + d];
    for (int i = 0; i < L.H; ++i) {
        h[L.ob1 + i] = (float)b1[i];
        h[L.ob2 + i] = (float)b2[i];
        h[L.ow3 + i] = (float)w3[i];
    }
    for (size_t i = 0; i < (size_t)L.H * L.H; ++i) h[L.oW2 + i] = (float)W2[i];
    h[L.ob3] = (float)b3;
    TGB_CUDA(cudaMemcpy(m.P[k], h.data(), sizeof(float) * L.n, cudaMemcpyHostToDevice));
    TGB_CUDA(cudaMemset(m.Am[k], 0, sizeof(float) * L.n));
    TGB_CUDA(cudaMemset(m.Av[k], 0, sizeof(float) * L.n));
    m.adam_t[k] = 0;
    TGB_TRY(refresh_member(m, k, 0));
    TGB_TRY(refresh_infer(m, 0));
    TGB_CUDA(cudaDeviceSynchronize());
    return TG_OK;
}

int mlp_get_member(Mlp &m, int k, double *W1, double *b1, double *W2, double *b2, double *w3,
                   double *b3) {
    TGB_CHECK(k >= 0 && k < m.n_members, TG_ERR_ARG, "member %d out of range", k);
    const MlpLayout &L = m.L;
    std::vector<float> h(L.n);
    TGB_CUDA(cudaDeviceSynchronize());
    TGB_CUDA(cudaMemcpy(h.data(), m.P[k], sizeof(float) * L.n, cudaMemcpyDeviceToHost));
    if (W1)
        for (int i = 0; i < L.H; ++i)
            for (int d = 0; d < L.D; ++d) W1[(size_t)i * L.D + d] = h[L.oW1 + (size_t)i * L.Dp + d];
    for (int i = 0; i < L.H; ++i) {
        if (b1) b1[i] = h[L.ob1 + i];
        if (b2) b2[i] = h[L.ob2 + i];
        if (w3) w3[i] = h[L.ow3 + i];
    }
    if (W2)
        for (size_t i = 0; i < (size_t)L.H * L.H; ++i) W2[i] = h[L.oW2 + i];
    if (b3) *b3 = h[L.ob3];
    return TG_OK;
}

int mlp_append_device(Mlp &m, int n, const float *x, int ldx, const double *e, const float *g,
                      int ldg, cudaStream_t st) {
    if (n <= 0) return TG_OK;
    const int D = m.L.D;
    const long long need = m.n_data + n;
    if (need > m.cap_data) {
        long long cap = std::max<long long>(need, std::max<long long>(4096, m.cap_data * 2));
        float *nx = nullptr, *ng = nullptr;
        double *ne = nullptr;
        TGB_TRY(dev_alloc(&nx, (size_t)cap * D));
        int rc = dev_alloc(&ng, (size_t)cap * D);
        if (rc == TG_OK) rc = dev_alloc(&ne, (size_t)cap);
        if (rc != TG_OK) {
            dev_free(nx); dev_free(ng); dev_free(ne);
            return rc;
        }
        if (m.n_data > 0) {
            TGB_CUDA(cudaMemcpyAsync(nx, m.dx, sizeof(float) * m.n_data * D, cudaMemcpyDeviceToDevice, st));
            TGB_CUDA(cudaMemcpyAsync(ng, m.dg, sizeof(float) * m.n_data * D, cudaMemcpyDeviceToDevice, st));
            TGB_CUDA(cudaMemcpyAsync(ne, m.de, sizeof(double) * m.n_data, cudaMemcpyDeviceToDevice, st));
        }
        TGB_CUDA(cudaStreamSynchronize(st));
        dev_free(m.dx); dev_free(m.dg); dev_free(m.de);
        m.dx = nx; m.dg = ng; m.de = ne;
        m.cap_data = cap;
    }
    const int64_t tot = (int64_t)n * D;
    k_copy_rows<<<blocks_for(tot), 256, 0, st>>>(n, D, x, ldx, m.dx + m.n_data * D);
    k_copy_rows<<<blocks_for(tot), 256, 0, st>>>(n, D, g, ldg, m.dg + m.n_data * D);
    TGB_CUDA(cudaGetLastError());
    TGB_CUDA(cudaMemcpyAsync(m.de + m.n_data, e, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    m.n_data += n;
    return TG_OK;
}

int mlp_check_err(Mlp &m, cudaStream_t st) {
    unsigned e = 0;
    TGB_CUDA(cudaMemcpyAsync(&e, m.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaStreamSynchronize(st));
    if (e) {
        cudaMemsetAsync(m.err, 0, sizeof(unsigned), st);
        set_error("device error word 0x%x in an MLP GEMM", e);
        return (e & (DEV_ERR_TIMEOUT_TMA | DEV_ERR_TIMEOUT_MMA | DEV_ERR_TIMEOUT_EPI)) ? TG_ERR_TIMEOUT
                                                                                       : TG_ERR_DEVICE;
    }
    return TG_OK;
}

// Forward and backward of member k on the gathered batch in w; gradients into m.Gr[k].
static int member_step(Mlp &m, MlpTrainWork &w, int k, double lam, cudaStream_t st) {
    const int B = w.B, H = m.L.H, Dp = m.L.Dp, D = m.L.D;
    const MlpLayout &L = m.L;
    const float *P = m.P[k];
    float *gr = m.Gr[k];
    const int64_t bh = (int64_t)B * H;
    const unsigned wb = blocks_for((size_t)B * 32);   // one warp per row
    TGB_CUDA(cudaMemsetAsync(gr, 0, sizeof(float) * L.n, st));
    // forward
    TGB_TRY(run(w.pZ1[k], m.err, st));
    k_act1<<<blocks_for(bh), 256, 0, st>>>(B, H, w.Z1.p, P + L.ob1, w.H1.p, w.S1.p, w.T1.p);
    TGB_TRY(run(w.pZ2[k], m.err, st));
    k_act2<<<wb, 256, 0, st>>>(B, H, w.Z2.p, P + L.ob2, P + L.ow3, P + L.ob3, w.H2.p, w.S2.p,
                               w.T2.p, w.U2.p, w.E.p);
    TGB_TRY(run(w.pV1[k], m.err, st));
    k_mul_bf16<<<blocks_for(bh), 256, 0, st>>>(bh, w.V1.p, w.S1.p, w.U1.p);
    TGB_TRY(run(w.pG[k], m.err, st));
    // loss
    k_loss<<<wb, 256, 0, st>>>(B, D, Dp, w.G.p, w.Gref.p, w.E.p, w.y.p, (float)lam, w.R.p, w.e.p,
                               w.loss2.p);
    // backward
    TGB_TRY(run(w.pA1[k], m.err, st));
    k_bw1<<<blocks_for(bh), 256, 0, st>>>(bh, w.A1.p, w.S1.p, w.V1.p, w.T1.p, w.dV1.p, w.dZ1p.p);
    TGB_TRY(run(w.pdU2[k], m.err, st));
    const unsigned rb = (unsigned)((B + kRowsPerBlock - 1) / kRowsPerBlock);
    k_bw2<<<rb, H, 0, st>>>(B, H, w.dU2.p, w.S2.p, w.T2.p, w.H2.p, P + L.ow3, w.e.p, w.dZ2.p,
                            gr + L.ow3, gr + L.ob2, gr + L.ob3);
    TGB_TRY(run(w.pdH1[k], m.err, st));
    k_bw3<<<rb, H, 0, st>>>(B, H, w.dH1.p, w.S1.p, w.dZ1p.p, w.dZ1.p, gr + L.ob1);
    TGB_CUDA(cudaGetLastError());
    // weight gradients: dW2 = [dZ2 | U2]^T [H1 | dV1], dW1 = [dZ1 | U1]^T [X | R]
    TGB_TRY(transpose(B, H, w.dZ2.p, H, w.AW2.p, 2 * B, st));
    TGB_TRY(transpose(B, H, w.U2.p, H, w.AW2.p + B, 2 * B, st));
    TGB_TRY(transpose(B, H, w.H1.p, H, w.BW2.p, 2 * B, st));
    TGB_TRY(transpose(B, H, w.dV1.p, H, w.BW2.p + B, 2 * B, st));
    TGB_TRY(transpose(B, H, w.dZ1.p, H, w.AW1.p, 2 * B, st));
    TGB_TRY(transpose(B, H, w.U1.p, H, w.AW1.p + B, 2 * B, st));
    TGB_TRY(transpose(B, Dp, w.R.p, Dp, w.BW1.p + B, 2 * B, st));
    TGB_TRY(run(w.pdW2[k], m.err, st));
    TGB_TRY(run(w.pdW1[k], m.err, st));
    return TG_OK;
}

static int adam_member(Mlp &m, int k, double lr, cudaStream_t st) {
    const double b1 = 0.9, b2 = 0.999;
    const long long t = ++m.adam_t[k];
    const double bc1 = 1.0 - std::pow(b1, (double)t), bc2 = 1.0 - std::pow(b2, (double)t);
    k_adam<<<blocks_for(m.L.n), 256, 0, st>>>((int64_t)m.L.n, m.P[k], m.Gr[k], m.Am[k], m.Av[k],
                                              (float)lr, (float)b1, (float)b2, (float)bc1,
                                              (float)bc2, 1e-8f);
    TGB_CUDA(cudaGetLastError());
    return refresh_member(m, k, st);
}

int mlp_batch_grads(Mlp &m, int member, int B, const float *x, const float *y, const float *gref,
                    double lam, double *grads, double *loss, float *E, float *G, cudaStream_t st) {
    TGB_CHECK(member >= 0 && member < m.n_members, TG_ERR_ARG, "member %d out of range", member);
    TGB_CHECK(B >= 32 && B % 32 == 0, TG_ERR_ARG, "batch %d must be a positive multiple of 32", B);
    if (!m.tw) m.tw = new MlpTrainWork();
    MlpTrainWork &w = *m.tw;
    TGB_TRY(w.ensure(m, B));
    const int D = m.L.D, Dp = m.L.Dp;
    Buf<float> tx, tg;
    Buf<double> te;
    TGB_TRY(tx.ensure((size_t)B * D));
    TGB_TRY(tg.ensure((size_t)B * D));
    TGB_TRY(te.ensure(B));
    std::vector<double> yd(y, y + B);
    std::vector<int64_t> id(B);
    std::iota(id.begin(), id.end(), 0);
    TGB_CUDA(cudaMemcpyAsync(tx.p, x, sizeof(float) * B * D, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(tg.p, gref, sizeof(float) * B * D, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(te.p, yd.data(), sizeof(double) * B, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(w.idx.p, id.data(), sizeof(int64_t) * B, cudaMemcpyHostToDevice, st));
    k_gather<<<B, 128, 0, st>>>(B, D, Dp, w.idx.p, tx.p, te.p, tg.p, 1.f, 0.0, 1.0, 1.f, w.Xb.p,
                                w.y.p, w.Gref.p);
    TGB_CUDA(cudaGetLastError());
    TGB_TRY(transpose(B, Dp, w.Xb.p, Dp, w.BW1.p, 2 * B, st));
    TGB_CUDA(cudaMemsetAsync(w.loss2.p, 0, 2 * sizeof(double), st));
    TGB_TRY(member_step(m, w, member, lam, st));
    std::vector<float> h(m.L.n);
    double l2[2];
    TGB_CUDA(cudaMemcpyAsync(h.data(), m.Gr[member], sizeof(float) * m.L.n, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaMemcpyAsync(l2, w.loss2.p, sizeof(l2), cudaMemcpyDeviceToHost, st));
    if (E) TGB_CUDA(cudaMemcpyAsync(E, w.E.p, sizeof(float) * B, cudaMemcpyDeviceToHost, st));
    if (G) TGB_CUDA(cudaMemcpyAsync(G, w.G.p, sizeof(float) * B * Dp, cudaMemcpyDeviceToHost, st));
    TGB_TRY(mlp_check_err(m, st));
    if (grads)
        for (size_t i = 0; i < m.L.n; ++i) grads[i] = h[i];
    if (loss) *loss = l2[0] + l2[1];
    return TG_OK;
}

int mlp_train(Mlp &m, int epochs, int batch, double lr, double lam, unsigned long long seed,
              double *loss_per_epoch, cudaStream_t st) {
    TGB_CHECK(batch >= 32 && batch % 32 == 0, TG_ERR_ARG, "batch %d must be a positive multiple of 32",
              batch);
    TGB_CHECK(m.n_data >= batch, TG_ERR_STATE, "%lld samples, fewer than one batch of %d",
              (long long)m.n_data, batch);
    TGB_CHECK(epochs >= 0, TG_ERR_ARG, "negative epochs");
    const int D = m.L.D, Dp = m.L.Dp;
    if (!(m.sx > 0.0) || !(m.sE > 0.0)) {   // normalisation from the data set
        Buf<double> mo;
        TGB_TRY(mo.ensure(3));
        TGB_CUDA(cudaMemsetAsync(mo.p, 0, 3 * sizeof(double), st));
        k_moments<<<296, 256, 0, st>>>((int64_t)m.n_data * D, m.dx, (int64_t)m.n_data, m.de, mo.p);
        TGB_CUDA(cudaGetLastError());
        double h[3];
        TGB_CUDA(cudaMemcpyAsync(h, mo.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        TGB_CUDA(cudaStreamSynchronize(st));
        const double N = (double)m.n_data;
        m.sx = std::sqrt(h[0] / (N * D));
        m.muE = h[1] / N;
        m.sE = std::sqrt(std::max(h[2] / N - m.muE * m.muE, 0.0));
        if (!(m.sx > 0.0)) m.sx = 1.0;
        if (!(m.sE > 1e-12)) m.sE = 1.0;
    }
    if (!m.tw) m.tw = new MlpTrainWork();
    MlpTrainWork &w = *m.tw;
    TGB_TRY(w.ensure(m, batch));
    const long long nb = m.n_data / batch;
    std::vector<int64_t> order(m.n_data);
    std::iota(order.begin(), order.end(), 0);
    std::mt19937_64 gen(seed);
    Buf<int64_t> ord;
    TGB_TRY(ord.ensure(order.size()));
    const float inv_sx = (float)(1.0 / m.sx), gscale = (float)(m.sx / m.sE);
    const double inv_sE = 1.0 / m.sE;
    for (int ep = 0; ep < epochs; ++ep) {
        // cosine decay of the step size from lr to lr / 20 over the epochs
        const double lr_ep =
            epochs > 1 ? lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(3.141592653589793 * ep / (epochs - 1))))
                       : lr;
        std::shuffle(order.begin(), order.end(), gen);
        TGB_CUDA(cudaMemcpyAsync(ord.p, order.data(), sizeof(int64_t) * order.size(),
                                 cudaMemcpyHostToDevice, st));
        TGB_CUDA(cudaMemsetAsync(w.loss2.p, 0, 2 * sizeof(double), st));
        for (long long b = 0; b < nb; ++b) {
            k_gather<<<batch, 128, 0, st>>>(batch, D, Dp, ord.p + b * batch, m.dx, m.de, m.dg,
                                            inv_sx, m.muE, inv_sE, gscale, w.Xb.p, w.y.p, w.Gref.p);
            TGB_CUDA(cudaGetLastError());
            TGB_TRY(transpose(batch, Dp, w.Xb.p, Dp, w.BW1.p, 2 * batch, st));
            for (int k = 0; k < m.n_members; ++k) {
                TGB_TRY(member_step(m, w, k, lam, st));
                TGB_TRY(adam_member(m, k, lr_ep, st));
            }
        }
        double l2[2];
        TGB_CUDA(cudaMemcpyAsync(l2, w.loss2.p, sizeof(l2), cudaMemcpyDeviceToHost, st));
        TGB_TRY(mlp_check_err(m, st));
        if (loss_per_epoch) loss_per_epoch[ep] = (l2[0] + l2[1]) / ((double)nb * m.n_members);
    }
    TGB_TRY(refresh_infer(m, st));
    TGB_CUDA(cudaStreamSynchronize(st));
    return TG_OK;
}

MlpInferWork *mlp_infer_work_new() { return new MlpInferWork(); }
void mlp_infer_work_delete(MlpInferWork *w) { delete w; }

int mlp_infer(Mlp &m, MlpInferWork &w, int n, const bf16 *X, int ldx, double *e_mean,
              double *e_std, float *g_mean, int ldg, const float *g_sub, cudaStream_t st) {
    if (n <= 0) return TG_OK;
    TGB_CHECK(m.infer_ready, TG_ERR_STATE, "MLP has no inference weights");
    TGB_CHECK(ldx >= m.L.Dp && ldx % 8 == 0, TG_ERR_ARG, "input row stride %d < %d or not a multiple of 8",
              ldx, m.L.Dp);
    TGB_CHECK(g_mean && ldg >= m.L.D && ldg % 4 == 0, TG_ERR_ARG,
              "dE/d(delta) rows need a stride >= %d and a multiple of 4", m.L.D);
    TGB_TRY(w.ensure(m, n));
    TGB_TRY(w.bind(m, X, n, ldx, g_mean, ldg, g_sub));
    const int nm = m.n_members;
    TGB_TRY(run(w.p1, m.err, st));
    for (const Plan &q : w.p2) TGB_TRY(run(q, m.err, st));
    for (const Plan &q : w.p3) TGB_TRY(run(q, m.err, st));
    TGB_TRY(run(w.p4, m.err, st));
    k_i_energy<<<blocks_for((size_t)n), 256, 0, st>>>(n, nm, w.npart(m), w.part.p, m.b3cat, e_mean,
                                                       e_std);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

}  // namespace tgb
