// tgb_soap.cu -- SOAP descriptor (expansion, power spectrum, normalisation)
// and the fused adjoint force/virial kernel for one soap_turbo block.
//
// The descriptor follows the published method (Caro, PRB 100, 024112 (2019);
// Bartok et al., PRB 87, 184115 (2013)) in the form restated by the FP64 oracle:
//   c_{n,lm}(i) = sum_j w(r) R_n(r) a_l(r) Y_lm(u)   (real Y_lm, u = r_ij/r)
//   p_{nn'l}    = mu_{nn'} sum_m c_{n,lm} c_{n',lm}, mu = sqrt2 off-diagonal
//   q           = p / |p|
// R_n (poly3, orthonormalised by the FP64 Jacobi matrix) and a_l (smeared
// angular factor 4 pi e^{-k} i_l(k)) are tabulated per species in FP64 on the
// GPU and interpolated in FP32 (cubic Hermite). Forces contract dE/dq through
// the normalisation and the power spectrum back to dE/dc on chip; the per-pair
// Cartesian derivative of q is never formed.

#include "tgb_soap.cuh"

#include <algorithm>
#include <cstring>
#include <cmath>
#include <vector>

namespace tgb {

constexpr int kMaxL = 12;
__constant__ float cYn[kMaxL + 1][kMaxL + 1];   // N_l0, sqrt2 N_lm (m > 0)
__constant__ float cRa[kMaxL + 1][kMaxL + 1];   // (2l-1)/(l-m)
__constant__ float cRb[kMaxL + 1][kMaxL + 1];   // (l+m-1)/(l-m)
__constant__ float cDf[kMaxL + 2];              // (2m-1)!!

// ---- column order of the tensor-core pair contraction (l_max = 8) ----------
// G_lm = sum_n Gamma_{n,lm} R_n(r_pair) is an MMA whose 96 accumulator columns
// hold the 81 lm of Gamma. A lane with t = lane % 4 owns columns 8k + 2t and
// 8k + 2t + 1 of every n-tile k: at step k they hold the (cos, sin) pair of one
// (l, m), and the steps of a lane walk whole m-chains (l = m .. 8 at fixed m), so
// the lane evaluates Y_lm and its gradient with the Legendre recurrence in l.
// Chains per lane group: t = 0: m = 0, 7, 8 (the m = 0 sin column is empty);
// t = 1: m = 1, 6; t = 2: m = 2, 5; t = 3: m = 3, 4 (the last step is empty).
constexpr int kMmaSteps = 12, kMmaCols = 8 * kMmaSteps;
// step record: qa = Aa z qa1 - Ba qa2 + Ca (Q_l^m), qb likewise (Q_l^{m+1}),
// f = the Y_lm normalisation, m; an empty step has f = 0
struct MmaStep {
    float Aa, Ba, Ca, Ab, Bb, Cb, f, m;
};
__constant__ MmaStep cStep[kMmaSteps][4];
__constant__ signed char cStepL[kMmaSteps][4];   // l of the step, -1 when empty
__constant__ unsigned char cLm2Col[81];          // accumulator column of lm

static int init_mma_steps(const float yn[kMaxL + 1][kMaxL + 1], const float ra[kMaxL + 1][kMaxL + 1],
                          const float rb[kMaxL + 1][kMaxL + 1], const float *df) {
    const int chains[4][3] = {{0, 7, 8}, {1, 6, -1}, {2, 5, -1}, {3, 4, -1}};
    MmaStep st[kMmaSteps][4] = {};
    signed char sl[kMmaSteps][4];
    unsigned char lm2col[81];
    std::memset(sl, -1, sizeof(sl));
    std::memset(lm2col, 0xff, sizeof(lm2col));
    for (int t = 0; t < 4; ++t) {
        int k = 0;
        for (int c = 0; c < 3; ++c) {
            const int m = chains[t][c];
            if (m < 0) continue;
            for (int l = m; l <= 8; ++l, ++k) {
                MmaStep &r = st[k][t];
                if (l == m) { r.Aa = 0.f; r.Ba = 0.f; r.Ca = df[m]; }
                else if (l == m + 1) { r.Aa = (float)(2 * m + 1); r.Ba = 0.f; r.Ca = 0.f; }
                else { r.Aa = ra[l][m]; r.Ba = rb[l][m]; r.Ca = 0.f; }
                if (l == m) { r.Ab = 0.f; r.Bb = 0.f; r.Cb = 0.f; }
                else if (l == m + 1) { r.Ab = 0.f; r.Bb = 0.f; r.Cb = df[m + 1]; }
                else if (l == m + 2) { r.Ab = (float)(2 * m + 3); r.Bb = 0.f; r.Cb = 0.f; }
                else { r.Ab = ra[l][m + 1]; r.Bb = rb[l][m + 1]; r.Cb = 0.f; }
                r.f = yn[l][m];
                r.m = (float)m;
                sl[k][t] = (signed char)l;
                lm2col[l * l + l + m] = (unsigned char)(8 * k + 2 * t);
                if (m > 0) lm2col[l * l + l - m] = (unsigned char)(8 * k + 2 * t + 1);
            }
        }
        if (k > kMmaSteps) {
            set_error("tensor-core step plan overflows (%d steps)", k);
            return TG_ERR_STATE;
        }
    }
    for (int lm = 0; lm < 81; ++lm)
        if (lm2col[lm] == 0xff) {
            set_error("tensor-core step plan misses lm %d", lm);
            return TG_ERR_STATE;
        }
    TGB_CUDA(cudaMemcpyToSymbol(cStep, st, sizeof(st)));
    TGB_CUDA(cudaMemcpyToSymbol(cStepL, sl, sizeof(sl)));
    TGB_CUDA(cudaMemcpyToSymbol(cLm2Col, lm2col, sizeof(lm2col)));
    return TG_OK;
}

int init_soap_constants() {
    float yn[kMaxL + 1][kMaxL + 1] = {}, ra[kMaxL + 1][kMaxL + 1] = {},
          rb[kMaxL + 1][kMaxL + 1] = {}, df[kMaxL + 2] = {};
    for (int l = 0; l <= kMaxL; ++l)
        for (int m = 0; m <= l; ++m) {
            double ratio = 1.0;
            for (int k = l - m + 1; k <= l + m; ++k) ratio /= (double)k;
            const double N = std::sqrt((2.0 * l + 1.0) / (4.0 * kPi) * ratio);
            yn[l][m] = (float)(m == 0 ? N : std::sqrt(2.0) * N);
            if (l >= m + 2) {
                ra[l][m] = (float)((2.0 * l - 1.0) / (double)(l - m));
                rb[l][m] = (float)((double)(l + m - 1) / (double)(l - m));
            }
        }
    for (int m = 0; m <= kMaxL + 1; ++m) {
        double d = 1.0;
        for (int k = 1; k <= 2 * m - 1; k += 2) d *= k;
        df[m] = (float)d;
    }
    TGB_CUDA(cudaMemcpyToSymbol(cYn, yn, sizeof(yn)));
    TGB_CUDA(cudaMemcpyToSymbol(cRa, ra, sizeof(ra)));
    TGB_CUDA(cudaMemcpyToSymbol(cRb, rb, sizeof(rb)));
    TGB_CUDA(cudaMemcpyToSymbol(cDf, df, sizeof(df)));
    return init_mma_steps(yn, ra, rb, df);
}

// ===================== FP64 table construction ==============================

namespace {

struct TableHyper {
    double rh, rs, nf, gs, sr, srs, st, sts, A, cw;
    int amax, lmax, re;
};

__device__ void d_scaled_moments(double tr, double s, int kmax, double *m) {
    const double g1 = exp(-(1.0 - tr) * (1.0 - tr) / (2.0 * s * s));
    const double g0 = exp(-tr * tr / (2.0 * s * s));
    m[0] = s * sqrt(kPi / 2.0) * (erf((1.0 - tr) / (sqrt(2.0) * s)) + erf(tr / (sqrt(2.0) * s)));
    for (int k = 0; k < kmax; ++k)
        m[k + 1] = tr * m[k] + s * s * ((k > 0 ? k * m[k - 1] : 0.0) - g1 + (k == 0 ? g0 : 0.0));
}

__device__ double d_e_of(const double *m, int k, int re) {
    if (re == 0) return m[k];
    if (re == 1) return m[k] - m[k + 1];
    return m[k] - 2.0 * m[k + 1] + m[k + 2];
}

// R_n(r) (without the neighbour weight) and dR_n/dr for n < amax.
__device__ void d_radial_basis(const TableHyper &h, const double *W, double r, double *R,
                               double *dR) {
    const int amax = h.amax, re = h.re;
    const double sig = h.sr * (1.0 + h.srs * r), dsig = h.sr * h.srs;
    const double tr = (h.rh - r) / h.rh, sc = sig / h.rh;
    const int kmax = amax + 2 + re + 2;
    double m[32], dm[32];
    d_scaled_moments(tr, sc, kmax, m);
    for (int k = 0; k + 2 <= kmax; ++k) {
        const double j1 = m[k + 1] - tr * m[k];
        const double j2 = m[k + 2] - 2.0 * tr * m[k + 1] + tr * tr * m[k];
        dm[k] = (-1.0 / h.rh) * j1 / (sc * sc) + (dsig / h.rh) * j2 / (sc * sc * sc);
    }
    const double pre = pow(h.rh, 0.5 + re);
    for (int n = 0; n < amax; ++n) {
        double v = 0.0, dv = 0.0;
        for (int j = 0; j < amax; ++j) {
            const double c = W[n * amax + j];
            if (c == 0.0) continue;
            v += c * d_e_of(m, j + 3, re);
            dv += c * d_e_of(dm, j + 3, re);
        }
        R[n] = v * pre;
        dR[n] = dv * pre;
    }
}

__device__ void d_weight(const TableHyper &h, double r, double *w, double *dw) {
    if (r >= h.rh) { *w = 0.0; *dw = 0.0; return; }
    double fa = 1.0, dfa = 0.0;
    if (h.A != 0.0) {
        const double x = r / h.rh;
        const double P = 1.0 - 3.0 * x * x + 2.0 * x * x * x;
        const double dP = (-6.0 * x + 6.0 * x * x) / h.rh;
        fa = pow(P, h.A);
        dfa = h.A * pow(P, h.A - 1.0) * dP;
    }
    double fc = 1.0, dfc = 0.0;
    if (h.rs < h.rh && r > h.rs) {
        const double wd = h.rh - h.rs;
        const double t = (r - h.rs) / wd;
        const double den = 1.0 - t * t;
        fc = exp(-h.nf * t * t / den);
        dfc = fc * (-h.nf) * (2.0 * t / (den * den)) / wd;
    }
    *w = h.gs * fa * fc;
    *dw = h.gs * (dfa * fc + fa * dfc);
}

// e^{-k} i_l(k) for l = 0..lmax+1 (power series; positive terms only).
__device__ void d_scaled_msbessel(double k, int lmax1, double *out) {
    const double ek = exp(-k);
    double pref = 1.0;
    const double x = 0.5 * k * k;
    for (int l = 0; l <= lmax1; ++l) {
        if (l > 0) pref *= k / (double)(2 * l + 1);
        double term = 1.0, sum = 1.0;
        for (int j = 1; j < 400; ++j) {
            term *= x / ((double)j * (double)(2 * l + 2 * j + 1));
            sum += term;
            if (term < 1e-18 * sum) break;
        }
        out[l] = ek * pref * sum;
    }
}

// Neighbour functions of one species at r: R~_n = w R_n and a_l, with d/dr.
__device__ void d_functions(const TableHyper &h, const double *W, double r, double *R, double *dR,
                            double *a, double *da) {
    double Rb[16], dRb[16], w, dw;
    d_weight(h, r, &w, &dw);
    d_radial_basis(h, W, r, Rb, dRb);
    for (int n = 0; n < h.amax; ++n) {
        R[n] = w * Rb[n];
        dR[n] = dw * Rb[n] + w * dRb[n];
    }
    const double st = h.st * (1.0 + h.sts * r), dst = h.st * h.sts;
    const double kk = r * r / (st * st);
    const double dk = 2.0 * r / (st * st) - 2.0 * r * r * dst / (st * st * st);
    double ei[kMaxL + 3];
    d_scaled_msbessel(kk, h.lmax + 1, ei);
    for (int l = 0; l <= h.lmax; ++l) {
        const double dil =
            (l == 0) ? ei[1] : ((double)l * ei[l - 1] + (double)(l + 1) * ei[l + 1]) / (2.0 * l + 1.0);
        a[l] = 4.0 * kPi * ei[l];
        da[l] = 4.0 * kPi * (dil - ei[l]) * dk;
    }
}

// One node per thread. Per node and function (R~_0..R~_{A-1}, a_0..a_lmax) one
// float4 (f, f', f'', 0). Values and first derivatives are analytic (FP64);
// second derivatives are the central difference of the analytic first
// derivative (FP64, step 1e-5 A), used only to interpolate the first derivative
// as a cubic Hermite function of its own (O(h^4) instead of the O(h^3) of the
// differentiated value interpolant).
__global__ void k_build_table(TableHyper h, const double *__restrict__ W, float4 *__restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > kTableIntervals) return;
    const double r = h.rh * (double)k / (double)kTableIntervals;
    const double eps = 1e-5;
    double R[16], dR[16], a[kMaxL + 1], da[kMaxL + 1];
    double Rp[16], dRp[16], ap[kMaxL + 1], dap[kMaxL + 1];
    double Rm[16], dRm[16], am[kMaxL + 1], dam[kMaxL + 1];
    d_functions(h, W, r, R, dR, a, da);
    d_functions(h, W, r + eps, Rp, dRp, ap, dap);
    d_functions(h, W, r - eps, Rm, dRm, am, dam);
    const int A = h.amax, nl = h.lmax + 1;
    float4 *o = out + (size_t)k * (A + nl);
    for (int n = 0; n < A; ++n)
        o[n] = make_float4((float)R[n], (float)dR[n], (float)((dRp[n] - dRm[n]) / (2.0 * eps)), 0.f);
    for (int l = 0; l < nl; ++l)
        o[A + l] = make_float4((float)a[l], (float)da[l],
                               (float)((dap[l] - dam[l]) / (2.0 * eps)), 0.f);
}

// Central atom: weight global_scaling * central_weight, Gaussian at r = 0,
// a_0(0) = 4 pi and Y_00 = 1/sqrt(4 pi) folded in.
__global__ void k_build_self(TableHyper h, const double *__restrict__ W, float *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double R[16], dR[16];
    d_radial_basis(h, W, 0.0, R, dR);
    for (int n = 0; n < h.amax; ++n)
        out[n] = (float)(h.gs * h.cw * R[n] * 4.0 * kPi / sqrt(4.0 * kPi));
}

}  // namespace

// Orthonormal poly3 basis: Gram-Schmidt of (rc - x)^(alpha+2) on [0, rc], which is
// t^3 P_n^{(0,6)}(2t - 1), t = (rc - x)/rc, normalised by sqrt(2n + 7). W[n][j]
// is sqrt(2n+7) times the integer coefficient of t^j in P_n^{(0,6)}(2t - 1).
static void poly3_jacobi_W(int amax, double *W) {
    auto binom = [](int n, int k) -> long long {
        if (k < 0 || k > n) return 0;
        long long r = 1;
        for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
        return r;
    };
    for (int n = 0; n < amax; ++n) {
        std::vector<long long> coef(amax, 0);
        for (int s = 0; s <= n; ++s) {
            const long long base = binom(n, n - s) * binom(n + 6, s);
            for (int i = 0; i <= s; ++i) coef[n - s + i] += base * binom(s, i) * (((s - i) % 2) ? -1 : 1);
        }
        const double nrm = std::sqrt((double)(2 * n + 7));
        for (int j = 0; j < amax; ++j) W[n * amax + j] = nrm * (double)coef[j];
    }
}

int table_width(int amax, int lmax) { return 4 * (amax + lmax + 1); }

int descriptor_ref_index(int d_internal, int nt, int nl) {
    const int np = nt * (nt + 1) / 2;
    const int l = d_internal / np, pi = d_internal - l * np;
    int n = 0, n2 = 0;
    internal_pair(pi, nt, n, n2);
    const int pi_ref = n * nt - n * (n - 1) / 2 + (n2 - n);   // row-major n <= n2
    return pi_ref * nl + l;
}

// (f, f') at both ends of every interval and function, (f_k, f'_k, f_k+1, f'_k+1),
// interval-major: the descriptor's Hermite value is one 16-byte gather per
// function instead of two 8-byte ones
__global__ void k_table_fd(int nf, const float4 *__restrict__ T, float4 *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf * kTableIntervals) return;
    const float4 a = T[i], b = T[i + nf];   // node k and node k + 1 of function j
    out[i] = make_float4(a.x, a.y, b.x, b.y);
}

int build_soap_tables(const SoapHostHypers &h, float *table, float *self_R, cudaStream_t st,
                      float4 *table_fd) {
    const int amax = h.alpha_max[0];
    const int tw = table_width(amax, h.lmax);
    std::vector<double> W(amax * amax);
    poly3_jacobi_W(amax, W.data());
    double *dW = nullptr;
    TGB_CUDA(cudaMalloc(&dW, sizeof(double) * W.size()));
    TGB_CUDA(cudaMemcpyAsync(dW, W.data(), sizeof(double) * W.size(), cudaMemcpyHostToDevice, st));
    for (int s = 0; s < h.ns; ++s) {
        TableHyper th{h.rcut_hard[s], h.rcut_soft[s], h.nf[s], h.global_scaling[s], h.sigma_r[s],
                      h.sigma_r_scaling[s], h.sigma_t[s], h.sigma_t_scaling[s],
                      h.amplitude_scaling[s], h.central_weight[s], amax, h.lmax,
                      h.radial_enhancement};
        k_build_table<<<(kTableIntervals + 1 + 127) / 128, 128, 0, st>>>(
            th, dW, reinterpret_cast<float4 *>(table + (size_t)s * (kTableIntervals + 1) * tw));
        k_build_self<<<1, 32, 0, st>>>(th, dW, self_R + s * amax);
        if (table_fd) {
            const int nf = amax + h.lmax + 1, nodes = kTableIntervals + 1;
            k_table_fd<<<(nf * kTableIntervals + 255) / 256, 256, 0, st>>>(
                nf, reinterpret_cast<const float4 *>(table + (size_t)s * nodes * tw),
                table_fd + (size_t)s * nf * kTableIntervals);
        }
    }
    cudaError_t e = cudaGetLastError();
    cudaError_t e2 = cudaStreamSynchronize(st);
    cudaFree(dW);
    TGB_CUDA(e);
    TGB_CUDA(e2);
    return TG_OK;
}

// ===================== FP32 device math ======================================

namespace {

// Cubic Hermite weights at fractional position t in a node interval of width h;
// the derivative-carrying weights h10, h11 include the factor h.
struct Hermite {
    int k;
    float h00, h10, h01, h11;
    __device__ __forceinline__ Hermite(float r, float h, float inv_h) {
        const float x = r * inv_h;
        int kk = (int)x;
        kk = kk > kTableIntervals - 1 ? kTableIntervals - 1 : (kk < 0 ? 0 : kk);
        k = kk;
        const float t = x - (float)kk, t2 = t * t, t3 = t2 * t;
        h00 = 2.f * t3 - 3.f * t2 + 1.f;
        h10 = (t3 - 2.f * t2 + t) * h;
        h01 = -2.f * t3 + 3.f * t2;
        h11 = (t3 - t2) * h;
    }
    // value from the interval table (f_k, f'_k, f_k+1, f'_k+1) of function j
    __device__ __forceinline__ float value_fd(const float4 *T, int nf, int j) const {
        const float4 a = __ldg(T + (size_t)k * nf + j);
        return h00 * a.x + h10 * a.y + h01 * a.z + h11 * a.w;
    }
    // value from (f, f') and, when wanted, first derivative from (f', f'') of function j
    __device__ __forceinline__ float value(const float4 *T, int nf, int j) const {
        const float4 a = __ldg(T + (size_t)k * nf + j), b = __ldg(T + (size_t)(k + 1) * nf + j);
        return h00 * a.x + h10 * a.y + h01 * b.x + h11 * b.y;
    }
    __device__ __forceinline__ void value_deriv(const float4 *T, int nf, int j, float &v,
                                                float &d) const {
        const float4 a = __ldg(T + (size_t)k * nf + j), b = __ldg(T + (size_t)(k + 1) * nf + j);
        v = h00 * a.x + h10 * a.y + h01 * b.x + h11 * b.y;
        d = h00 * a.y + h10 * a.z + h01 * b.y + h11 * b.z;
    }
};

__device__ __forceinline__ int fold_index(int j, int n) {
    return j < n ? j : j % n;
}

// Bulk prefetch of [p, p + bytes) into L2 (a hint; nothing is written). The range
// shrinks to whole 16-byte units inside it, so it never leaves the buffer.
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes) {
    const uintptr_t a = ((uintptr_t)p + 15) & ~(uintptr_t)15;
    const uintptr_t e = ((uintptr_t)p + bytes) & ~(uintptr_t)15;
    if (e > a)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(e - a))
                     : "memory");
}

// The rows a site's force pass reads (g, q, c) and its pair records, prefetched
// into L2 by the warp that runs `ahead` sites earlier: sites run in about index
// order, so when the site's own warp starts, its rows come from L2, not DRAM.
// RAW (compressed blocks): g is dE/dp in rows of DIM, and q (rows of the
// compressed dim) is not read.
template <int DIM, int NT, int NLM, bool RAW>
__device__ __forceinline__ void prefetch_force_site(const SiteArgs &S, const ForceIn &I, int site,
                                                    int lane) {
    const int fs = site + I.ahead;
    if (I.ahead <= 0 || fs >= S.n_sites || lane >= 4) return;
    if (lane == 0) prefetch_l2(I.g + (size_t)fs * DIM, sizeof(float) * DIM);
    else if (lane == 1) {
        if (!RAW) prefetch_l2(I.q + (size_t)fs * DIM, sizeof(float) * DIM);
    }
    else if (lane == 2) prefetch_l2(I.c + (size_t)fs * NT * NLM, sizeof(float) * NT * NLM);
    else {
        const int row = S.site_row[fs];
        const int64_t p0 = S.pstart[row], p1 = S.pstart[row + 1];
        prefetch_l2(S.xyz + 3 * p0, sizeof(double) * 3 * (size_t)(p1 - p0));
        prefetch_l2(S.nbr + p0, sizeof(int) * (size_t)(p1 - p0));
    }
}

// Descriptor species of a global species id (its first match, or with inst 1
// its second), -1 when the block does not see it.
__device__ __forceinline__ int zlookup(const SoapParams &P, int z, int inst = 0) {
    if (z < 0 || z >= kMaxZ) return -1;
    return inst == 0 ? (int)P.zmap[z] : (int)P.zmap2[z];
}

// Under species multiplicity a site's list is walked once per match as one run
// of virtual pairs 1 .. n_inst (np - 1): virtual pair v >= np is list pair
// v - np + 1 of the second match. Returns the list position and sets inst.
__device__ __forceinline__ int virtual_pair(int v, int np, int &inst) {
    inst = v >= np;
    return inst ? v - np + 1 : v;
}

// Real spherical harmonics of unit u into Y[l*l + l + m] (m = -l..l), by the
// running Legendre recurrence in l for each m (Q_l^m = d^m P_l/dz^m) and the
// running (x + iy)^m: a handful of live registers.
template <int LMAX>
__device__ __forceinline__ void real_ylm(float x, float y, float z, float *Y) {
    float cm = 1.f, sm = 0.f;
#pragma unroll
    for (int m = 0; m <= LMAX; ++m) {
        float q2 = 0.f, q1 = 0.f;
#pragma unroll
        for (int l = m; l <= LMAX; ++l) {
            float q;
            if (l == m) q = cDf[m];
            else if (l == m + 1) q = (float)(2 * m + 1) * z * q1;
            else q = cRa[l][m] * z * q1 - cRb[l][m] * q2;
            const float f = cYn[l][m] * q;
            if (m == 0) {
                Y[l * l + l] = f;
            } else {
                Y[l * l + l + m] = f * cm;
                Y[l * l + l - m] = f * sm;
            }
            q2 = q1;
            q1 = q;
        }
        const float c2 = x * cm - y * sm;
        sm = x * sm + y * cm;
        cm = c2;
    }
}

}  // namespace

// ===================== expansion + power spectrum ===========================

// CTA tiles of the descriptor and force passes that the autotuner picks from:
// tile v runs soap_tile_warps(v) central sites (warps) per CTA with at least
// soap_tile_minb(v) CTAs resident per SM (the register budget follows).
template <int NS, int AMAX, int LMAX, int TILE = 0>
struct DescShape {
    static constexpr int NL = LMAX + 1;
    static constexpr int NLM = NL * NL;
    static constexpr int NT = NS * AMAX;
    static constexpr int NF = AMAX + NL;          // tabulated functions per node
    static constexpr int DIM = NT * (NT + 1) / 2 * NL;
    static constexpr int SLOTS = (NLM + 31) / 32;
    static constexpr int CHUNK = 32;
    static constexpr int WARPS = soap_tile_warps(TILE);
    // per-warp shared memory (floats): Y rows (odd stride NLM), R rows (stride
    // AMAX, read as broadcast float4), a rows (odd stride NL), pair species.
    // The FP64 coefficients of the power-spectrum phase reuse the same area.
    static constexpr int YS = CHUNK * NLM;
    static constexpr int RS = CHUNK * AMAX;
    static constexpr int AS = CHUNK * NL;
    static constexpr int STAGE = YS + RS + AS + CHUNK;
    // FP64 c rows for the power spectrum: stride CS = 4 mod 16 doubles, so an
    // 8 x 4 DMMA fragment load (rows lane/4, columns lane%4) is two wavefronts
    static constexpr int CS = (NLM + 11) / 16 * 16 + 4;
    static constexpr int CWORDS = 2 * NT * CS;
    static constexpr int WARP_FLOATS = ((STAGE > CWORDS ? STAGE : CWORDS) + 3) / 4 * 4;
    static_assert(AMAX % 4 == 0, "float4 reads of R rows need alpha_max % 4 == 0");
    static_assert(YS % 4 == 0 && RS % 4 == 0, "R rows must stay 16-byte aligned");
};

// One warp per central atom. Lanes evaluate 32 pairs at a time (table
// interpolation, Y_lm) into shared memory; then each lane owns (l, m) slots and
// accumulates c_{n,lm} over the chunk's pairs in FP32. The central atom's
// constant contribution to c_{n,00} is added in FP64 afterwards (it dominates
// c_{n,00}, and FP32 sums on top of it were the main descriptor error).
// Power spectrum and |p| in FP64. RAW (compressed blocks, P.raw): the power
// spectrum goes to O.praw in FP64 for the compression pass, and the kernel stops
// there; a separate instantiation, so the uncompressed kernels keep their code.
// MULT: the block has species multiplicity (P.n_inst = 2); its own
// instantiation, so blocks without it keep their code and registers.
template <int NS, int AMAX, int LMAX, int TILE, bool RAW = false, bool MULT = false>
__global__ void __launch_bounds__(32 * soap_tile_warps(TILE), soap_tile_minb(TILE))
    k_soap_expand(SoapParams P, SiteArgs S, DescOut O) {
    using Sh = DescShape<NS, AMAX, LMAX, TILE>;
    constexpr int NL = Sh::NL, NLM = Sh::NLM, NT = Sh::NT, NF = Sh::NF, DIM = Sh::DIM;
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *Ys = smem + warp * Sh::WARP_FLOATS;
    float *Rs = Ys + Sh::YS;
    float *As = Rs + Sh::RS;
    int *pspec = reinterpret_cast<int *>(As + Sh::AS);
    __shared__ unsigned char pair_n[NT * (NT + 1) / 2], pair_n2[NT * (NT + 1) / 2];
    for (int t = threadIdx.x; t < NT * (NT + 1) / 2; t += blockDim.x) {
        int n = 0, n2 = 0;
        internal_pair(t, NT, n, n2);
        pair_n[t] = (unsigned char)n;
        pair_n2[t] = (unsigned char)n2;
    }
    __syncthreads();
    const int site = blockIdx.x * Sh::WARPS + warp;
    if (site >= S.n_sites) return;
    if (lane == 0 && S.ahead > 0 && site + S.ahead < S.n_sites) {
        // the pair records of the site `ahead` sites on, into L2 for its warp
        const int fr = S.site_row[site + S.ahead];
        const int64_t f0 = S.pstart[fr], f1 = S.pstart[fr + 1];
        prefetch_l2(S.xyz + 3 * f0, sizeof(double) * 3 * (size_t)(f1 - f0));
        prefetch_l2(S.nbr + f0, sizeof(int) * (size_t)(f1 - f0));
    }
    const int row = S.site_row[site];
    const int catom = S.site_atom[site];
    const int64_t p0 = S.pstart[row];
    const int np = (int)(S.pstart[row + 1] - p0);
    const int scen = zlookup(P, S.species[catom]);   // central atom's descriptor species

    int lmk[Sh::SLOTS], lk[Sh::SLOTS];
#pragma unroll
    for (int k = 0; k < Sh::SLOTS; ++k) {
        lmk[k] = lane + 32 * k;
        int l = 0;
        while ((l + 1) * (l + 1) <= lmk[k]) ++l;
        lk[k] = l;
    }
    float acc[NT][Sh::SLOTS];
#pragma unroll
    for (int n = 0; n < NT; ++n)
#pragma unroll
        for (int k = 0; k < Sh::SLOTS; ++k) acc[n][k] = 0.f;

    // the self pair (first of the list) is not part of the chunks; under species
    // multiplicity the list is walked once per match (virtual pairs)
    const int npv = MULT ? 2 * np - 1 : np;
    for (int base = 1; base < npv; base += Sh::CHUNK) {
        const int t = lane;
        int s = -1;
        if (base + t < npv) {
            int inst = 0;
            int64_t p = p0 + base + t;
            if constexpr (MULT) p = p0 + virtual_pair(base + t, np, inst);
            s = zlookup(P, S.nsp ? (int)S.nsp[p] : S.species[fold_index(S.nbr[p], P.n_atoms)],
                        inst);
            const float x = (float)S.xyz[3 * p], y = (float)S.xyz[3 * p + 1],
                        z = (float)S.xyz[3 * p + 2];
            const float r = sqrtf(x * x + y * y + z * z);
            if (s >= 0 && r < P.rcut[s] && r > 0.f) {
                const float4 *Tf = P.table_fd + (size_t)s * NF * kTableIntervals;
                const Hermite hm(r, P.tab_h[s], P.tab_inv_h[s]);
                float rv[AMAX];
#pragma unroll
                for (int n = 0; n < AMAX; ++n) rv[n] = hm.value_fd(Tf, NF, n);
                float4 *r4 = reinterpret_cast<float4 *>(Rs + t * AMAX);
#pragma unroll
                for (int q = 0; q < AMAX / 4; ++q)
                    r4[q] = make_float4(rv[4 * q], rv[4 * q + 1], rv[4 * q + 2], rv[4 * q + 3]);
#pragma unroll
                for (int l = 0; l < NL; ++l)
                    As[t * NL + l] = hm.value_fd(Tf, NF, AMAX + l);
                const float ir = 1.f / r;
                real_ylm<LMAX>(x * ir, y * ir, z * ir, Ys + t * NLM);
            } else {
                s = -1;
            }
        }
        pspec[t] = s;
        __syncwarp();
        const int cnt = min(Sh::CHUNK, npv - base);
        for (int tt = 0; tt < cnt; ++tt) {
            const int ss = pspec[tt];
            if (ss < 0) continue;
            float rv[AMAX];
            const float4 *r4 = reinterpret_cast<const float4 *>(Rs + tt * AMAX);
#pragma unroll
            for (int q = 0; q < AMAX / 4; ++q) {
                const float4 v = r4[q];
                rv[4 * q] = v.x; rv[4 * q + 1] = v.y; rv[4 * q + 2] = v.z; rv[4 * q + 3] = v.w;
            }
            const float *Yr = Ys + tt * NLM;
            const float *Ar = As + tt * NL;
#pragma unroll
            for (int k = 0; k < Sh::SLOTS; ++k) {
                if (lmk[k] < NLM) {
                    const float ya = Yr[lmk[k]] * Ar[lk[k]];
#pragma unroll
                    for (int sp = 0; sp < NS; ++sp) {
                        if (ss == sp) {
#pragma unroll
                            for (int n = 0; n < AMAX; ++n) acc[sp * AMAX + n][k] += rv[n] * ya;
                        }
                    }
                }
            }
        }
        __syncwarp();
    }
    // c to shared (FP64, layout [n][lm]) with the central term, and to global (fp32);
    // (under multiplicity the central atom's second descriptor species too)
    const int scen2 = MULT ? zlookup(P, S.species[catom], 1) : -1;
    double *cs = reinterpret_cast<double *>(Ys);
#pragma unroll
    for (int n = 0; n < NT; ++n)
#pragma unroll
        for (int k = 0; k < Sh::SLOTS; ++k)
            if (lmk[k] < NLM) {
                double v = (double)acc[n][k];
                if (lmk[k] == 0 && (n / AMAX == scen || n / AMAX == scen2))
                    v += (double)P.self_R[n];   // [ns][amax]: species n / AMAX, radial n % AMAX
                cs[n * Sh::CS + lmk[k]] = v;
                O.c[((size_t)site * NT + n) * NLM + lmk[k]] = (float)v;
            }
    __syncwarp();
    // Power spectrum in the internal order u = l * NP + pi. For each l the NP
    // channel pairs (n <= n2) run across lanes, so one warp-wide load reads
    // c_{n,lm} of at most NT distinct n: distinct bank pairs (the row stride NLM
    // is odd), one shared-memory wavefront per load and no divergence in m.
    constexpr int NP = NT * (NT + 1) / 2;
    auto power = [&](int l, int pi) -> double {
        const int n = pair_n[pi], n2 = pair_n2[pi];
        const double *c1 = cs + n * Sh::CS + l * l, *c2 = cs + n2 * Sh::CS + l * l;
        double v = 0.0;
#pragma unroll
        for (int m = 0; m < 2 * l + 1; ++m) v += c1[m] * c2[m];
        return n != n2 ? v * 1.4142135623730951 : v;
    };
    const int K1 = P.K1;
    __nv_bfloat16 *qs = O.qsplit + (size_t)site * K1;
    float *qrow = O.q + (size_t)site * DIM;
    auto emit = [&](int u, double v, double invv, double &offv) {
        const double mu = P.mu[u];
        const double dl = v * invv - mu;
        offv += dl * mu;
        const float df = (float)dl;
        qrow[u] = df;
        __nv_bfloat16 hi, lo;
        bf16_split(df, hi, lo);
        qs[u] = hi;
        if (P.nsplit == 3) {
            qs[DIM + u] = hi;
            qs[2 * DIM + u] = lo;
        }
    };
    double nrm2 = 0.0, off = 0.0, inv = 0.0;
    if constexpr (NT % 8 == 0) {
        // FP64 tensor cores: per l, the Gram blocks G_ab = C_a C_b^T of the 8-channel
        // blocks a <= b (C_a = c[8a .. 8a+7][l^2 .. l^2+2l]), k-steps of 4 m values
        // (zero-padded). Lane (g = lane/4, t = lane%4) holds G_ab[g][2t], G_ab[g][2t+1].
        constexpr int NB = NT / 8;
        const int g8 = lane >> 2, t4 = lane & 3;
        auto gram = [&](int l, int a, int b, double &d0, double &d1) {
            d0 = 0.0;
            d1 = 0.0;
            const double *ra = cs + (8 * a + g8) * Sh::CS + l * l;
            const double *rb = cs + (8 * b + g8) * Sh::CS + l * l;
            const int M = 2 * l + 1;
#pragma unroll
            for (int kb = 0; kb < M; kb += 4) {
                const int m = kb + t4;
                const double va = m < M ? ra[m] : 0.0;
                const double vb = a == b ? va : (m < M ? rb[m] : 0.0);
                asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                    : "+d"(d0), "+d"(d1)
                    : "d"(va), "d"(vb));
            }
        };
        // pass 1: p and |p|. Each Gram block is computed once; p goes to the q row in
        // fp32 at its internal position (an off-diagonal block's entries in lane order
        // (2 lane + e), a diagonal block's upper triangle row by row), |p|^2 in FP64.
#pragma unroll
        for (int l = 0; l < NL; ++l)
#pragma unroll
            for (int a = 0; a < NB; ++a)
#pragma unroll
                for (int b = a; b < NB; ++b) {
                    double d[2];
                    gram(l, a, b, d[0], d[1]);
                    const int base = l * NP + gram_block_start(a, b, NB);
                    if (a != b) {
                        const double v0 = d[0] * 1.4142135623730951, v1 = d[1] * 1.4142135623730951;
                        nrm2 += v0 * v0 + v1 * v1;
                        if constexpr (RAW)
                            *reinterpret_cast<double2 *>(O.praw + (size_t)site * DIM + base +
                                                         2 * lane) = make_double2(v0, v1);
                        else
                            *reinterpret_cast<float2 *>(qrow + base + 2 * lane) =
                                make_float2((float)v0, (float)v1);
                    } else {
#pragma unroll
                        for (int e = 0; e < 2; ++e) {
                            const int j = 2 * t4 + e;
                            if (g8 > j) continue;
                            const double v = g8 != j ? d[e] * 1.4142135623730951 : d[e];
                            nrm2 += v * v;
                            const int u = base + g8 * 8 - (g8 * (g8 - 1)) / 2 + (j - g8);
                            if constexpr (RAW) O.praw[(size_t)site * DIM + u] = v;
                            else qrow[u] = (float)v;
                        }
                    }
                }
        if constexpr (RAW) return;
        nrm2 = warp_sum(nrm2);
        inv = nrm2 > 0.0 ? 1.0 / sqrt(nrm2) : 0.0;
        __syncwarp();   // the warp's p entries are visible to every lane
        // pass 2, streaming: q = p/|p|, delta = q - mu (fp32 row and bf16 split), delta . mu
        static_assert(DIM % 4 == 0, "four descriptor entries per lane step");
        for (int u = 4 * lane; u < DIM; u += 128) {
            const float4 pv = *reinterpret_cast<const float4 *>(qrow + u);
            const double2 m0 = __ldg(reinterpret_cast<const double2 *>(P.mu + u));
            const double2 m1 = __ldg(reinterpret_cast<const double2 *>(P.mu + u + 2));
            const double dl0 = (double)pv.x * inv - m0.x, dl1 = (double)pv.y * inv - m0.y;
            const double dl2 = (double)pv.z * inv - m1.x, dl3 = (double)pv.w * inv - m1.y;
            off += (dl0 * m0.x + dl1 * m0.y) + (dl2 * m1.x + dl3 * m1.y);
            const float f0 = (float)dl0, f1 = (float)dl1, f2 = (float)dl2, f3 = (float)dl3;
            *reinterpret_cast<float4 *>(qrow + u) = make_float4(f0, f1, f2, f3);
            __nv_bfloat16 h0, l0, h1, l1, h2, l2, h3, l3;
            bf16_split(f0, h0, l0);
            bf16_split(f1, h1, l1);
            bf16_split(f2, h2, l2);
            bf16_split(f3, h3, l3);
            __nv_bfloat162 hh[2] = {__halves2bfloat162(h0, h1), __halves2bfloat162(h2, h3)};
            *reinterpret_cast<uint2 *>(qs + u) = *reinterpret_cast<const uint2 *>(hh);
            if (P.nsplit == 3) {
                __nv_bfloat162 ll[2] = {__halves2bfloat162(l0, l1), __halves2bfloat162(l2, l3)};
                *reinterpret_cast<uint2 *>(qs + DIM + u) = *reinterpret_cast<const uint2 *>(hh);
                *reinterpret_cast<uint2 *>(qs + 2 * DIM + u) = *reinterpret_cast<const uint2 *>(ll);
            }
        }
    } else {
        if constexpr (RAW) {
#pragma unroll
            for (int l = 0; l < NL; ++l)
                for (int pi = lane; pi < NP; pi += 32)
                    O.praw[(size_t)site * DIM + l * NP + pi] = power(l, pi);
            return;
        }
        // pass 1: |p| (FP64)
#pragma unroll
        for (int l = 0; l < NL; ++l)
            for (int pi = lane; pi < NP; pi += 32) {
                const double v = power(l, pi);
                nrm2 += v * v;
            }
        nrm2 = warp_sum(nrm2);
        inv = nrm2 > 0.0 ? 1.0 / sqrt(nrm2) : 0.0;
        // pass 2: q = p/|p|, delta = q - mu, delta . mu; operand rows hold split(delta)
#pragma unroll
        for (int l = 0; l < NL; ++l)
            for (int pi = lane; pi < NP; pi += 32) emit(l * NP + pi, power(l, pi), inv, off);
    }
    const double nrm = sqrt(nrm2);
    off = warp_sum(off);
    const int fill = P.fill_to > 0 ? P.fill_to : K1;
    for (int d = P.nsplit * DIM + lane; d < fill; d += 32) qs[d] = __float2bfloat16_rn(0.f);
    if (lane == 0) {
        O.pnorm[site] = nrm;
        O.qoff[site] = off;
    }
}

// ===================== adjoint force / virial ================================

template <int NS, int AMAX, int LMAX, int TILE = 0>
struct ForceShape {
    static constexpr int NL = LMAX + 1;
    static constexpr int NLM = NL * NL;
    static constexpr int NT = NS * AMAX;
    static constexpr int NF = AMAX + NL;
    static constexpr int DIM = NT * (NT + 1) / 2 * NL;
    static constexpr int SLOTS = (NLM + 31) / 32;
    static constexpr int WARPS = soap_tile_warps(TILE);
    static constexpr int BROW = NT + 4;            // row stride of B_l: rows read as float4, the
                                                   // transposed writes spread over the banks
    static constexpr int BSTRIDE = NT * BROW + 4;  // per-l stride (multiple of 4, 4 mod 32)
    static constexpr int BAREA = (NL * BSTRIDE + 3) / 4 * 4;   // keeps gam 16-byte aligned
    // Gamma rows [lm][n] with stride GS = NT + 4: a lane's four consecutive n go in
    // one float4 store, and 8 lanes' stores hit 8 distinct 16-byte bank groups
    static constexpr int GS = NT + 4;
    // Gamma is computed into registers and then written over the B area, which is
    // dead by then: the warp's area is the larger of the two
    static constexpr int GAREA = NLM * GS;
    static constexpr int WARP_FLOATS = BAREA > GAREA ? BAREA : GAREA;
    // Gamma rows of slot k (lm 32k .. 32k + 31) may be stored as soon as slot k is
    // done when they end below the first B_l that slot k + 1 reads
    // (l = floor(sqrt(32 (k + 1)))); true for every shape compiled here.
    static constexpr int isqrt(int v) { int r = 0; while ((r + 1) * (r + 1) <= v) ++r; return r; }
    static constexpr bool gamma_over_b_ok() {
        for (int k = 0; k + 1 < SLOTS; ++k)
            if ((32 * (k + 1)) * GS > isqrt(32 * (k + 1)) * BSTRIDE) return false;
        return true;
    }
    static constexpr bool GAMMA_EARLY = gamma_over_b_ok();
    static_assert(AMAX % 4 == 0, "float4 reads of Gamma need alpha_max % 4 == 0");
};

// One warp per central atom: dE/dq -> dE/dp (normalisation, FP64) -> B_l -> Gamma =
// dE/dc (shared memory), then one lane per pair contracts Gamma with d(c)/d(r_j)
// on the fly: F_j -= dE_i/dr_j, F_i += dE_i/dr_j, virial += 1/2 (f x + x f).
// RAW (compressed blocks, P.raw): I.g already holds dE/dp, from the compression's
// adjoint; a separate instantiation, so the uncompressed kernels keep their code.
// MULT: species multiplicity, as in k_soap_expand.
template <int NS, int AMAX, int LMAX, int TILE, bool RAW = false, bool MULT = false>
__global__ void __launch_bounds__(32 * soap_tile_warps(TILE), soap_tile_minb(TILE))
    k_soap_force(SoapParams P, SiteArgs S, ForceIn I, ForceOut O) {
    using Sh = ForceShape<NS, AMAX, LMAX, TILE>;
    constexpr int NL = Sh::NL, NLM = Sh::NLM, NT = Sh::NT, NF = Sh::NF, DIM = Sh::DIM;
    extern __shared__ __align__(16) float smem[];
    __shared__ double vred[Sh::WARPS][6];
    __shared__ unsigned char pair_n[NT * (NT + 1) / 2], pair_n2[NT * (NT + 1) / 2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = threadIdx.x; t < NT * (NT + 1) / 2; t += blockDim.x) {
        int n = 0, n2 = 0;
        internal_pair(t, NT, n, n2);
        pair_n[t] = (unsigned char)n;
        pair_n2[t] = (unsigned char)n2;
    }
    if (lane < 6) vred[warp][lane] = 0.0;
    __syncthreads();
    float *Bm = smem + warp * Sh::WARP_FLOATS;   // [l][n][n2] (stride BSTRIDE per l)
    float *gam = Bm;                             // [lm][n], over B once Gamma is computed
    const int site = blockIdx.x * Sh::WARPS + warp;
    double vir[6] = {0, 0, 0, 0, 0, 0};
    if (site < S.n_sites) {
        prefetch_force_site<DIM, NT, NLM, RAW>(S, I, site, lane);
        const int row = S.site_row[site];
        const int catom = S.site_atom[site];
        const int64_t p0 = S.pstart[row];
        const int np = (int)(S.pstart[row + 1] - p0);
        // the c row is read after the dE/dp phase: request its lines into L1 now
        for (int o = 32 * lane; o < NT * NLM; o += 32 * 32)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(I.c + (size_t)site * NT * NLM + o));
        // dE/dq = G = ksum mu + g0 + g: ksum = sum_s kd_s (FP64, GEMM-1 epilogue),
        // g0 = sum_s kcoef_s (q_s - mu) (per block), g from GEMM 2; q = mu + delta.
        // dE/dp = (G - (G . q) q) / |p| = (a mu + g0 + g - dot delta) / |p| with
        // dot = G . q and a = ksum - dot. The large parts, ksum mu . mu against dot,
        // cancel only in the FP64 scalars dot = ksum (mu . mu + delta . mu) + g0 . mu
        // + sum (g0 delta + g q) and a; the per-entry terms are all small and run in
        // fp32.
        const float *g = I.g + (size_t)site * DIM;
        const float *q = I.q + (size_t)site * DIM;
        // per-slice partial sums: lanes load in parallel, a butterfly adds them
        double ksum = 0.0, esum = 0.0;
        for (int t = lane; t < I.n_etiles; t += 32) {
            ksum += I.kdsum[(size_t)site * I.n_etiles + t];
            esum += I.epart[(size_t)site * I.n_etiles + t];
        }
        ksum = warp_sum(ksum);
        esum = warp_sum(esum);
        // descriptor entries in the internal order d = l * NP + pi
        constexpr int NP = NT * (NT + 1) / 2;
        // Four consecutive entries per lane and 16-byte loads; a group of four never
        // crosses an l boundary because NP % 4 == 0.
        constexpr bool VEC = (DIM % 4 == 0) && (NP % 4 == 0);
        auto put_b = [&](int d, float h) {
            const int l = d / NP, pi = d - l * NP;
            float *Bl = Bm + l * Sh::BSTRIDE;
            const int n = pair_n[pi], n2 = pair_n2[pi];
            if (n == n2) {
                Bl[n * Sh::BROW + n] = 2.f * h;
            } else {
                const float v = 1.41421356237309515f * h;
                Bl[n * Sh::BROW + n2] = v;
                Bl[n2 * Sh::BROW + n] = v;
            }
        };
        if constexpr (RAW) {
            for (int d = lane; d < DIM; d += 32) put_b(d, g[d]);
        } else {
            float sp = 0.f;   // sum (g0 delta + g q), a small sum
            if constexpr (VEC) {
                // the site's g and q rows go to registers in one round trip and are
                // read once; mu and g0 (per block, L1-resident) are read twice
                constexpr int NV4 = DIM / 4, NV = (NV4 + 31) / 32;
                const float4 *g4 = reinterpret_cast<const float4 *>(g);
                const float4 *q4 = reinterpret_cast<const float4 *>(q);
                const float4 *m4 = reinterpret_cast<const float4 *>(P.muf);
                const float4 *z4 = reinterpret_cast<const float4 *>(P.g0f);
                float4 gr[NV], qr[NV];
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    const int i4 = lane + 32 * k;
                    gr[k] = i4 < NV4 ? g4[i4] : make_float4(0.f, 0.f, 0.f, 0.f);
                    qr[k] = i4 < NV4 ? q4[i4] : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    const int i4 = lane + 32 * k;
                    if (i4 >= NV4) continue;
                    const float4 m = __ldg(m4 + i4), z = __ldg(z4 + i4);
                    const float4 gv = gr[k], qv = qr[k];
                    sp += z.x * qv.x + gv.x * (m.x + qv.x);
                    sp += z.y * qv.y + gv.y * (m.y + qv.y);
                    sp += z.z * qv.z + gv.z * (m.z + qv.z);
                    sp += z.w * qv.w + gv.w * (m.w + qv.w);
                }
                const double dot = ksum * (P.mu2 + I.qoff[site]) + P.g0mu + warp_sum((double)sp);
                const double nrm = I.pnorm[site];
                const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
                const float fa = (float)((ksum - dot) * inv), fi = (float)inv,
                            fd = (float)(dot * inv);
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    const int i4 = lane + 32 * k;
                    if (i4 >= NV4) continue;
                    const float4 m = __ldg(m4 + i4), z = __ldg(z4 + i4);
                    const float4 gv = gr[k], qv = qr[k];
                    const int d0 = 4 * i4;
                    put_b(d0, fa * m.x + fi * (z.x + gv.x) - fd * qv.x);
                    put_b(d0 + 1, fa * m.y + fi * (z.y + gv.y) - fd * qv.y);
                    put_b(d0 + 2, fa * m.z + fi * (z.z + gv.z) - fd * qv.z);
                    put_b(d0 + 3, fa * m.w + fi * (z.w + gv.w) - fd * qv.w);
                }
            } else {
                for (int d = lane; d < DIM; d += 32)
                    sp += P.g0f[d] * q[d] + g[d] * (P.muf[d] + q[d]);
                const double dot = ksum * (P.mu2 + I.qoff[site]) + P.g0mu + warp_sum((double)sp);
                const double nrm = I.pnorm[site];
                const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
                const float fa = (float)((ksum - dot) * inv), fi = (float)inv,
                            fd = (float)(dot * inv);
                for (int d = lane; d < DIM; d += 32)
                    put_b(d, fa * P.muf[d] + fi * (P.g0f[d] + g[d]) - fd * q[d]);
            }
        }
        __syncwarp();
        // Gamma_{n,lm} = dE/dc_{n,lm} = sum_n2 B_l(n, n2) c_{n2,lm}
        int lmk[Sh::SLOTS], lk[Sh::SLOTS];
#pragma unroll
        for (int k = 0; k < Sh::SLOTS; ++k) {
            lmk[k] = lane + 32 * k;
            int l = 0;
            while ((l + 1) * (l + 1) <= lmk[k]) ++l;
            lk[k] = l;
        }
        const float *cg = I.c + (size_t)site * NT * NLM;
        // One slot (32 lm) at a time, 16 live accumulators per lane: a slot's Gamma
        // rows go over the B_l of the smallest l, which no later slot reads, once
        // the whole warp has finished reading B for the slot (gamma_over_b_ok).
        auto slot_gamma = [&](int k, float (&gv)[NT]) {
            float cr[NT];
#pragma unroll
            for (int n2 = 0; n2 < NT; ++n2) cr[n2] = cg[n2 * NLM + lmk[k]];
            const float *Bl = Bm + lk[k] * Sh::BSTRIDE;
#pragma unroll
            for (int n = 0; n < NT; ++n) {
                const float4 *Bn = reinterpret_cast<const float4 *>(Bl + n * Sh::BROW);
                float v = 0.f;
#pragma unroll
                for (int j = 0; j < NT / 4; ++j) {
                    const float4 b = Bn[j];
                    v += b.x * cr[4 * j] + b.y * cr[4 * j + 1] + b.z * cr[4 * j + 2] +
                         b.w * cr[4 * j + 3];
                }
                gv[n] = v;
            }
        };
        auto store_gamma = [&](int k, const float (&gv)[NT]) {
#pragma unroll
            for (int n0 = 0; n0 < NT; n0 += 4)
                *reinterpret_cast<float4 *>(gam + lmk[k] * Sh::GS + n0) =
                    make_float4(gv[n0], gv[n0 + 1], gv[n0 + 2], gv[n0 + 3]);
        };
        if constexpr (Sh::GAMMA_EARLY) {
#pragma unroll
            for (int k = 0; k < Sh::SLOTS; ++k) {
                float gv[NT];
                if (lmk[k] < NLM) slot_gamma(k, gv);
                __syncwarp();   // the warp is done with this slot's B_l
                if (lmk[k] < NLM) store_gamma(k, gv);
            }
        } else {
            float gv[Sh::SLOTS][NT];
#pragma unroll
            for (int k = 0; k < Sh::SLOTS; ++k)
                if (lmk[k] < NLM) slot_gamma(k, gv[k]);
            __syncwarp();   // every lane is done with B: Gamma goes over it
#pragma unroll
            for (int k = 0; k < Sh::SLOTS; ++k)
                if (lmk[k] < NLM) store_gamma(k, gv[k]);
        }
        __syncwarp();
        // pairs: lane per pair (the self pair, first in the list, is the -sum),
        // once per species match
        double fs[3] = {0, 0, 0};
        const int npv = MULT ? 2 * np - 1 : np;   // virtual pairs: once per species match
        for (int pv = 1 + lane; pv < npv; pv += 32) {
            int inst = 0;
            int64_t p = p0 + pv;
            if constexpr (MULT) p = p0 + virtual_pair(pv, np, inst);
            const int ja = fold_index(S.nbr[p], P.n_atoms);
            const int s = zlookup(P, S.nsp ? (int)S.nsp[p] : S.species[ja], inst);
            const double X = S.xyz[3 * p], Yy = S.xyz[3 * p + 1], Z = S.xyz[3 * p + 2];
            const float x = (float)X, y = (float)Yy, z = (float)Z;
            const float r = sqrtf(x * x + y * y + z * z);
            if (s < 0 || !(r < P.rcut[s]) || !(r > 0.f)) continue;
            const float4 *T = reinterpret_cast<const float4 *>(
                P.table + (size_t)s * (kTableIntervals + 1) * (4 * NF));
            const Hermite hm(r, P.tab_h[s], P.tab_inv_h[s]);
            float R[AMAX], dR[AMAX], al[NL], dal[NL];
#pragma unroll
            for (int n = 0; n < AMAX; ++n) hm.value_deriv(T, NF, n, R[n], dR[n]);
#pragma unroll
            for (int l = 0; l < NL; ++l) hm.value_deriv(T, NF, AMAX + l, al[l], dal[l]);
            const float ir = 1.f / r;
            const float u0 = x * ir, u1 = y * ir, u2 = z * ir;
            float T1 = 0.f, T2x = 0.f, T2y = 0.f, T2z = 0.f;
            const int ch = s * AMAX;
            // m outer, l inner: Q_l^m and Q_l^{m+1} by running recurrences in l;
            // (C_m, S_m) = (x + iy)^m and (C_{m-1}, S_{m-1}) running in m.
            float cm = 1.f, sm = 0.f, cm1 = 0.f, sm1 = 0.f;
#pragma unroll
            for (int m = 0; m <= LMAX; ++m) {
                float qa2 = 0.f, qa1 = 0.f, qb2 = 0.f, qb1 = 0.f;
#pragma unroll
                for (int l = m; l <= LMAX; ++l) {
                    float qa, qb;
                    if (l == m) qa = cDf[m];
                    else if (l == m + 1) qa = (float)(2 * m + 1) * u2 * qa1;
                    else qa = cRa[l][m] * u2 * qa1 - cRb[l][m] * qa2;
                    if (l == m) qb = 0.f;
                    else if (l == m + 1) qb = cDf[m + 1];
                    else if (l == m + 2) qb = (float)(2 * m + 3) * u2 * qb1;
                    else qb = cRa[l][m + 1] * u2 * qb1 - cRb[l][m + 1] * qb2;
                    qa2 = qa1; qa1 = qa;
                    qb2 = qb1; qb1 = qb;
                    // G = sum_n Gamma R_n, G' = sum_n Gamma R_n' for +m (C) and -m (S)
                    const int lmp = l * l + l + m;
                    float Gp = 0.f, dGp = 0.f;
                    const float4 *gp = reinterpret_cast<const float4 *>(gam + lmp * Sh::GS + ch);
#pragma unroll
                    for (int qd = 0; qd < AMAX / 4; ++qd) {
                        const float4 v = gp[qd];
                        Gp += v.x * R[4 * qd] + v.y * R[4 * qd + 1] + v.z * R[4 * qd + 2] +
                              v.w * R[4 * qd + 3];
                        dGp += v.x * dR[4 * qd] + v.y * dR[4 * qd + 1] + v.z * dR[4 * qd + 2] +
                               v.w * dR[4 * qd + 3];
                    }
                    const float f = cYn[l][m];
                    const float a = al[l], da = dal[l];
                    if (m == 0) {
                        T1 += f * qa * (a * dGp + da * Gp);
                        T2z += a * Gp * f * qb;
                    } else {
                        const int lmn = l * l + l - m;
                        float Gn = 0.f, dGn = 0.f;
                        const float4 *gn = reinterpret_cast<const float4 *>(gam + lmn * Sh::GS + ch);
#pragma unroll
                        for (int qd = 0; qd < AMAX / 4; ++qd) {
                            const float4 v = gn[qd];
                            Gn += v.x * R[4 * qd] + v.y * R[4 * qd + 1] + v.z * R[4 * qd + 2] +
                                  v.w * R[4 * qd + 3];
                            dGn += v.x * dR[4 * qd] + v.y * dR[4 * qd + 1] +
                                   v.z * dR[4 * qd + 2] + v.w * dR[4 * qd + 3];
                        }
                        const float yc = f * qa * cm, ys = f * qa * sm;
                        T1 += yc * (a * dGp + da * Gp) + ys * (a * dGn + da * Gn);
                        const float wc = a * Gp, wsn = a * Gn;
                        const float fm = f * qa * (float)m;
                        // grad of sqrt2 N Q C_m: (m C_{m-1}, -m S_{m-1}, Q' C_m); S_m likewise
                        T2x += wc * fm * cm1 + wsn * fm * sm1;
                        T2y += -wc * fm * sm1 + wsn * fm * cm1;
                        T2z += (wc * cm + wsn * sm) * f * qb;
                    }
                }
                cm1 = cm;
                sm1 = sm;
                const float c2 = u0 * cm - u1 * sm;
                sm = u0 * sm + u1 * cm;
                cm = c2;
            }
            const float ut2 = u0 * T2x + u1 * T2y + u2 * T2z;
            // f_pair = -dE_i/dr_j = -(T1 u + (T2 - (u.T2) u)/r)
            const float fx = -(T1 * u0 + (T2x - ut2 * u0) * ir);
            const float fy = -(T1 * u1 + (T2y - ut2 * u1) * ir);
            const float fz = -(T1 * u2 + (T2z - ut2 * u2) * ir);
            atomicAdd(&O.forces[3 * (size_t)ja], (double)fx);
            atomicAdd(&O.forces[3 * (size_t)ja + 1], (double)fy);
            atomicAdd(&O.forces[3 * (size_t)ja + 2], (double)fz);
            if (O.pair_grad) {   // d E_i / d r_j = -f_pair (summed over species matches)
                if constexpr (MULT) {
                    O.pair_grad[3 * p] -= (double)fx;
                    O.pair_grad[3 * p + 1] -= (double)fy;
                    O.pair_grad[3 * p + 2] -= (double)fz;
                } else {
                    O.pair_grad[3 * p] = -(double)fx;
                    O.pair_grad[3 * p + 1] = -(double)fy;
                    O.pair_grad[3 * p + 2] = -(double)fz;
                }
            }
            fs[0] -= fx; fs[1] -= fy; fs[2] -= fz;
            // virial += 1/2 (f x + x f), packed xx yy zz xy xz yz
            vir[0] += (double)fx * X;
            vir[1] += (double)fy * Yy;
            vir[2] += (double)fz * Z;
            vir[3] += 0.5 * ((double)fx * Yy + (double)fy * X);
            vir[4] += 0.5 * ((double)fx * Z + (double)fz * X);
            vir[5] += 0.5 * ((double)fy * Z + (double)fz * Yy);
        }
#pragma unroll
        for (int qd = 0; qd < 3; ++qd) fs[qd] = warp_sum(fs[qd]);
        if (lane == 0 && O.pair_grad)   // the self pair: d E_i / d r_i = -sum_j d E_i / d r_j
            for (int qd = 0; qd < 3; ++qd) O.pair_grad[3 * p0 + qd] = -fs[qd];
        if (lane == 0) {
            atomicAdd(&O.forces[3 * (size_t)catom], fs[0]);
            atomicAdd(&O.forces[3 * (size_t)catom + 1], fs[1]);
            atomicAdd(&O.forces[3 * (size_t)catom + 2], fs[2]);
            O.energies[catom] += I.delta2 * esum;
        }
    }
#pragma unroll
    for (int qd = 0; qd < 6; ++qd) vir[qd] = warp_sum(vir[qd]);
    if (lane == 0)
        for (int qd = 0; qd < 6; ++qd) vred[warp][qd] = vir[qd];
    if (O.vir_struct && lane == 0 && site < S.n_sites) {   // per-structure virial (batches)
        double *o = O.vir_struct + 9 * (size_t)O.atom_struct[S.site_atom[site]];
        atomicAdd(o + 0, vir[0]);
        atomicAdd(o + 4, vir[1]);
        atomicAdd(o + 8, vir[2]);
        atomicAdd(o + 1, vir[3]);
        atomicAdd(o + 3, vir[3]);
        atomicAdd(o + 2, vir[4]);
        atomicAdd(o + 6, vir[4]);
        atomicAdd(o + 5, vir[5]);
        atomicAdd(o + 7, vir[5]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double v[6] = {0, 0, 0, 0, 0, 0};
        for (int w = 0; w < Sh::WARPS; ++w)
            for (int qd = 0; qd < 6; ++qd) v[qd] += vred[w][qd];
        double *o = O.vpart + (size_t)blockIdx.x * 9;
        o[0] = v[0]; o[4] = v[1]; o[8] = v[2];
        o[1] = o[3] = v[3];
        o[2] = o[6] = v[4];
        o[5] = o[7] = v[5];
    }
}

// ===================== adjoint forces on the tensor cores =====================
//
// The same contraction as k_soap_force, with its two dense products on the
// tensor cores (mma.sync m16n8k8, TF32 operands, fp32 accumulation):
//   Gamma_l = B_l C_l              [NT x NT] . [NT x (2l+1)] per l,
//   G = R Gamma, G' = R' Gamma     [16 pairs x NT] . [NT x 96 columns] per 16 pairs,
// where row p of R (R') holds R~_n (R~'_n) of pair p in its species' channels.
// PREC 3 splits every operand into TF32 hi + lo and runs hi.hi + hi.lo + lo.hi
// (about fp32 accuracy: the plain form); PREC 1 runs hi.hi (the mixed form).
// The accumulators stay in registers: the lane owning columns (8k + 2t, +1)
// walks its m-chains over the steps k (see init_mma_steps) for the rows g and
// g + 8 of the tile and sums its part of T1 = sum Y (a G' + a' G) and
// T2 = sum a G grad Y; a quad shuffle adds the four lanes' parts.

template <int PREC>
__device__ __forceinline__ void tf32_split(float x, uint32_t &hi, uint32_t &lo) {
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
    if constexpr (PREC == 3) {
        const float r = x - __uint_as_float(hi);
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
    } else {
        lo = 0u;
    }
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
        "{%8, %9}, {%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// d += a . b with the TF32 split of both (PREC 3) or the leading parts only
template <int PREC>
__device__ __forceinline__ void mma_split(float (&d)[4], const uint32_t (&ah)[4],
                                          const uint32_t (&al)[4], uint32_t bh0, uint32_t bh1,
                                          uint32_t bl0, uint32_t bl1) {
    if constexpr (PREC == 3) {
        mma_tf32(d, al[0], al[1], al[2], al[3], bh0, bh1);
        mma_tf32(d, ah[0], ah[1], ah[2], ah[3], bl0, bl1);
    }
    mma_tf32(d, ah[0], ah[1], ah[2], ah[3], bh0, bh1);
}

template <int NS>
struct MmaForceShape {
    static constexpr int NT = NS * 8, NL = 9, NLM = 81;
    static constexpr int NP = NT * (NT + 1) / 2, DIM = NP * NL;
    static constexpr int BROW = NT + 4;               // B_l rows: A-fragment loads conflict-free
    static constexpr int BSTRIDE = NT * BROW + 4;
    static constexpr int BAREA = NL * BSTRIDE;
    static constexpr int CROW = 88;                   // staged c rows: B-fragment loads conflict-free
    static constexpr int CAREA = NT * CROW;
    static constexpr int AROW = NT + 4;               // pair rows of R~ and R~'
    static constexpr int AUX = 44;                    // a_l, a'_l, u, 1/r, (x+iy)^m per pair
    static constexpr int STAGE = 32 * (2 * AROW + AUX);
    static constexpr int XAREA = (BAREA + CAREA > STAGE ? BAREA + CAREA : STAGE);
    static constexpr int GROW = 104;                  // Gamma rows (96 columns), 8 mod 32
    static constexpr int GAREA = NT * GROW;
    static constexpr int WARP_FLOATS = (XAREA + GAREA + 3) / 4 * 4;
    static constexpr int WARPS = 4;
};

template <int NS, int PREC>
__global__ void __launch_bounds__(128, 2)
    k_soap_force_mma(SoapParams P, SiteArgs S, ForceIn I, ForceOut O) {
    using Sh = MmaForceShape<NS>;
    constexpr int NT = Sh::NT, NL = Sh::NL, NLM = Sh::NLM, NP = Sh::NP, DIM = Sh::DIM;
    constexpr int AMAX = 8, NF = AMAX + NL, KS = NT / 8;
    extern __shared__ __align__(16) float smem[];
    __shared__ double vred[Sh::WARPS][6];
    __shared__ unsigned char pair_n[NP], pair_n2[NP];
    __shared__ float4 stepc[kMmaSteps * 4 * 2];
    __shared__ int stepl[kMmaSteps * 4];
    __shared__ unsigned char lm2col[NLM];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    for (int i = threadIdx.x; i < NP; i += blockDim.x) {
        int n = 0, n2 = 0;
        internal_pair(i, NT, n, n2);
        pair_n[i] = (unsigned char)n;
        pair_n2[i] = (unsigned char)n2;
    }
    for (int i = threadIdx.x; i < kMmaSteps * 4; i += blockDim.x) {
        const MmaStep &r = cStep[i / 4][i % 4];
        stepc[2 * i] = make_float4(r.Aa, r.Ba, r.Ca, r.Ab);
        stepc[2 * i + 1] = make_float4(r.Bb, r.Cb, r.f, r.m);
        stepl[i] = cStepL[i / 4][i % 4];
    }
    for (int i = threadIdx.x; i < NLM; i += blockDim.x) lm2col[i] = cLm2Col[i];
    if (lane < 6) vred[warp][lane] = 0.0;
    float *X = smem + warp * Sh::WARP_FLOATS;
    float *Bm = X;                    // [l][n][n2], phases A and B
    float *cs = X + Sh::BAREA;        // [n][lm] (row CROW), phase B
    float *Ag = X;                    // [pair][n] R~ (row AROW), phase C
    float *Ad = X + 32 * Sh::AROW;    // [pair][n] R~'
    float *aux = X + 64 * Sh::AROW;   // [pair][AUX]
    float *Gs = X + Sh::XAREA;        // Gamma [n][column] (row GROW)
    // columns without an lm stay zero: zero the whole Gamma area once
    for (int i = lane; i < Sh::GAREA; i += 32) Gs[i] = 0.f;
    __syncthreads();
    const int site = blockIdx.x * Sh::WARPS + warp;
    double vir[6] = {0, 0, 0, 0, 0, 0};
    if (site < S.n_sites) {
        prefetch_force_site<DIM, NT, NLM, false>(S, I, site, lane);
        const int row = S.site_row[site];
        const int catom = S.site_atom[site];
        const int64_t p0 = S.pstart[row];
        const int np = (int)(S.pstart[row + 1] - p0);
        const float *g_row = I.g + (size_t)site * DIM;
        const float *q_row = I.q + (size_t)site * DIM;
        const float *c_row = I.c + (size_t)site * NT * NLM;
        // ---- every row of the site in one round trip: c (to shared memory), g and q
        constexpr int NV4 = DIM / 4, NV = (NV4 + 31) / 32;
        constexpr int NC4 = NT * NLM / 4, NCV = (NC4 + 31) / 32;
        static_assert(DIM % 4 == 0 && NP % 4 == 0 && (NT * NLM) % 4 == 0, "vector rows");
        float4 cv[NCV], gr[NV], qr[NV];
#pragma unroll
        for (int k = 0; k < NCV; ++k) {
            const int i4 = lane + 32 * k;
            cv[k] = i4 < NC4 ? reinterpret_cast<const float4 *>(c_row)[i4]
                             : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const int i4 = lane + 32 * k;
            gr[k] = i4 < NV4 ? reinterpret_cast<const float4 *>(g_row)[i4]
                             : make_float4(0.f, 0.f, 0.f, 0.f);
            qr[k] = i4 < NV4 ? reinterpret_cast<const float4 *>(q_row)[i4]
                             : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        double ksum = 0.0, esum = 0.0;
        for (int k = lane; k < I.n_etiles; k += 32) {
            ksum += I.kdsum[(size_t)site * I.n_etiles + k];
            esum += I.epart[(size_t)site * I.n_etiles + k];
        }
        ksum = warp_sum(ksum);
        esum = warp_sum(esum);
#pragma unroll
        for (int k = 0; k < NCV; ++k) {
            const int i4 = lane + 32 * k;
            if (i4 >= NC4) continue;
            const float v[4] = {cv[k].x, cv[k].y, cv[k].z, cv[k].w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = 4 * i4 + u, n2 = e / NLM;
                cs[n2 * Sh::CROW + (e - n2 * NLM)] = v[u];
            }
        }
        // ---- dE/dp, as in k_soap_force, into the symmetric B_l
        auto put_b = [&](int d, float h) {
            const int l = d / NP, pi = d - l * NP;
            float *Bl = Bm + l * Sh::BSTRIDE;
            const int n = pair_n[pi], n2 = pair_n2[pi];
            if (n == n2) {
                Bl[n * Sh::BROW + n] = 2.f * h;
            } else {
                const float v = 1.41421356237309515f * h;
                Bl[n * Sh::BROW + n2] = v;
                Bl[n2 * Sh::BROW + n] = v;
            }
        };
        {
            const float4 *m4 = reinterpret_cast<const float4 *>(P.muf);
            const float4 *z4 = reinterpret_cast<const float4 *>(P.g0f);
            float sp = 0.f;
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                const int i4 = lane + 32 * k;
                if (i4 >= NV4) continue;
                const float4 m = __ldg(m4 + i4), z = __ldg(z4 + i4);
                const float4 gv = gr[k], qv = qr[k];
                sp += z.x * qv.x + gv.x * (m.x + qv.x);
                sp += z.y * qv.y + gv.y * (m.y + qv.y);
                sp += z.z * qv.z + gv.z * (m.z + qv.z);
                sp += z.w * qv.w + gv.w * (m.w + qv.w);
            }
            const double dot = ksum * (P.mu2 + I.qoff[site]) + P.g0mu + warp_sum((double)sp);
            const double nrm = I.pnorm[site];
            const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
            const float fa = (float)((ksum - dot) * inv), fi = (float)inv, fd = (float)(dot * inv);
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                const int i4 = lane + 32 * k;
                if (i4 >= NV4) continue;
                const float4 m = __ldg(m4 + i4), z = __ldg(z4 + i4);
                const float4 gv = gr[k], qv = qr[k];
                const int d0 = 4 * i4;
                put_b(d0, fa * m.x + fi * (z.x + gv.x) - fd * qv.x);
                put_b(d0 + 1, fa * m.y + fi * (z.y + gv.y) - fd * qv.y);
                put_b(d0 + 2, fa * m.z + fi * (z.z + gv.z) - fd * qv.z);
                put_b(d0 + 3, fa * m.w + fi * (z.w + gv.w) - fd * qv.w);
            }
        }
        __syncwarp();
        // ---- Gamma_l = B_l C_l: rows n (g, g + 8), columns m-index (8 jj + 2t, +1)
#pragma unroll 1
        for (int l = 0; l < NL; ++l) {
            const float *Bl = Bm + l * Sh::BSTRIDE;
            uint32_t ah[KS][4], al[KS][4];
#pragma unroll
            for (int ks = 0; ks < KS; ++ks) {
                const int c0 = 8 * ks + t;
                if constexpr (NT == 16) {
                    tf32_split<PREC>(Bl[g * Sh::BROW + c0], ah[ks][0], al[ks][0]);
                    tf32_split<PREC>(Bl[(g + 8) * Sh::BROW + c0], ah[ks][1], al[ks][1]);
                    tf32_split<PREC>(Bl[g * Sh::BROW + c0 + 4], ah[ks][2], al[ks][2]);
                    tf32_split<PREC>(Bl[(g + 8) * Sh::BROW + c0 + 4], ah[ks][3], al[ks][3]);
                } else {   // 8 channels: rows 8..15 of the tile are zero
                    tf32_split<PREC>(Bl[g * Sh::BROW + c0], ah[ks][0], al[ks][0]);
                    tf32_split<PREC>(Bl[g * Sh::BROW + c0 + 4], ah[ks][2], al[ks][2]);
                    ah[ks][1] = al[ks][1] = ah[ks][3] = al[ks][3] = 0u;
                }
            }
            const int nm = 2 * l + 1;
            for (int jj = 0; 8 * jj < nm; ++jj) {
                float d[4] = {0.f, 0.f, 0.f, 0.f};
                const int col = 8 * jj + g;   // this lane's B-fragment column (m-index)
#pragma unroll
                for (int ks = 0; ks < KS; ++ks) {
                    const int k0 = 8 * ks + t;
                    const float b0 = col < nm ? cs[k0 * Sh::CROW + l * l + col] : 0.f;
                    const float b1 = col < nm ? cs[(k0 + 4) * Sh::CROW + l * l + col] : 0.f;
                    uint32_t bh0, bl0, bh1, bl1;
                    tf32_split<PREC>(b0, bh0, bl0);
                    tf32_split<PREC>(b1, bh1, bl1);
                    mma_split<PREC>(d, ah[ks], al[ks], bh0, bh1, bl0, bl1);
                }
                // d: rows n = g (d0, d1), g + 8 (d2, d3); m-index 8 jj + 2t (+1)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int mi = 8 * jj + 2 * t + e;
                    if (mi < nm) {
                        const int c = lm2col[l * l + mi];
                        Gs[g * Sh::GROW + c] = d[e];
                        if (NT == 16) Gs[(g + 8) * Sh::GROW + c] = d[2 + e];
                    }
                }
            }
        }
        __syncwarp();   // Gamma complete; B_l and c are dead: the pair staging goes over them
        // ---- pairs, 32 at a time: lane-per-pair set-up, then two 16-pair MMA tiles
        double fs[3] = {0, 0, 0};
        for (int base = 1; base < np; base += 32) {
            {
                const int pp = base + lane;
                float *ag = Ag + lane * Sh::AROW, *ad = Ad + lane * Sh::AROW, *ax = aux + lane * Sh::AUX;
#pragma unroll
                for (int n = 0; n < NT; ++n) { ag[n] = 0.f; ad[n] = 0.f; }
#pragma unroll
                for (int k = 0; k <= 40; ++k) ax[k] = 0.f;   // [40]: the valid flag
                if (pp < np) {
                    const int64_t p = p0 + pp;
                    const int s = zlookup(P, S.nsp ? (int)S.nsp[p]
                                                   : S.species[fold_index(S.nbr[p], P.n_atoms)]);
                    const float x = (float)S.xyz[3 * p], y = (float)S.xyz[3 * p + 1],
                                z = (float)S.xyz[3 * p + 2];
                    const float r = sqrtf(x * x + y * y + z * z);
                    if (s >= 0 && r < P.rcut[s] && r > 0.f) {
                        const float4 *T = reinterpret_cast<const float4 *>(
                            P.table + (size_t)s * (kTableIntervals + 1) * (4 * NF));
                        const Hermite hm(r, P.tab_h[s], P.tab_inv_h[s]);
#pragma unroll
                        for (int n = 0; n < AMAX; ++n)
                            hm.value_deriv(T, NF, n, ag[s * AMAX + n], ad[s * AMAX + n]);
#pragma unroll
                        for (int l = 0; l < NL; ++l) hm.value_deriv(T, NF, AMAX + l, ax[l], ax[9 + l]);
                        const float ir = 1.f / r, u0 = x * ir, u1 = y * ir, u2 = z * ir;
                        ax[18] = u0; ax[19] = u1; ax[20] = u2; ax[21] = ir;
                        float cm = 1.f, sm = 0.f;
#pragma unroll
                        for (int m = 0; m <= 8; ++m) {
                            ax[22 + m] = cm;
                            ax[31 + m] = sm;
                            const float c2 = u0 * cm - u1 * sm;
                            sm = u0 * sm + u1 * cm;
                            cm = c2;
                        }
                        ax[40] = 1.f;
                    }
                }
            }
            __syncwarp();
#pragma unroll 1
            for (int mt = 0; mt < 2; ++mt) {
                if (base + 16 * mt >= np) break;   // warp-uniform
                const int r0 = 16 * mt + g, r1 = r0 + 8;
                float accG[kMmaSteps][4], accD[kMmaSteps][4];
#pragma unroll
                for (int j = 0; j < kMmaSteps; ++j)
#pragma unroll
                    for (int e = 0; e < 4; ++e) accG[j][e] = accD[j][e] = 0.f;
#pragma unroll
                for (int ks = 0; ks < KS; ++ks) {
                    const int k0 = 8 * ks + t;
                    uint32_t gh[4], gl[4], dh[4], dl[4];
                    tf32_split<PREC>(Ag[r0 * Sh::AROW + k0], gh[0], gl[0]);
                    tf32_split<PREC>(Ag[r1 * Sh::AROW + k0], gh[1], gl[1]);
                    tf32_split<PREC>(Ag[r0 * Sh::AROW + k0 + 4], gh[2], gl[2]);
                    tf32_split<PREC>(Ag[r1 * Sh::AROW + k0 + 4], gh[3], gl[3]);
                    tf32_split<PREC>(Ad[r0 * Sh::AROW + k0], dh[0], dl[0]);
                    tf32_split<PREC>(Ad[r1 * Sh::AROW + k0], dh[1], dl[1]);
                    tf32_split<PREC>(Ad[r0 * Sh::AROW + k0 + 4], dh[2], dl[2]);
                    tf32_split<PREC>(Ad[r1 * Sh::AROW + k0 + 4], dh[3], dl[3]);
#pragma unroll
                    for (int j = 0; j < kMmaSteps; ++j) {
                        uint32_t bh0, bl0, bh1, bl1;
                        tf32_split<PREC>(Gs[k0 * Sh::GROW + 8 * j + g], bh0, bl0);
                        tf32_split<PREC>(Gs[(k0 + 4) * Sh::GROW + 8 * j + g], bh1, bl1);
                        mma_split<PREC>(accG[j], gh, gl, bh0, bh1, bl0, bl1);
                        mma_split<PREC>(accD[j], dh, dl, bh0, bh1, bl0, bl1);
                    }
                }
                // post-processing: rows r0 (accumulator elements 0, 1) and r1 (2, 3)
                float T[2][4];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const float *ax = aux + (h ? r1 : r0) * Sh::AUX;
                    const float z = ax[20];
                    float qa1 = 0.f, qa2 = 0.f, qb1 = 0.f, qb2 = 0.f;
                    float T1 = 0.f, T2x = 0.f, T2y = 0.f, T2z = 0.f;
#pragma unroll
                    for (int k = 0; k < kMmaSteps; ++k) {
                        const float4 c1 = stepc[2 * (4 * k + t)], c2 = stepc[2 * (4 * k + t) + 1];
                        const int l = stepl[4 * k + t];
                        const int m = (int)c2.w;
                        const float qa = c1.x * z * qa1 - c1.y * qa2 + c1.z;
                        const float qb = c1.w * z * qb1 - c2.x * qb2 + c2.y;
                        qa2 = qa1; qa1 = qa;
                        qb2 = qb1; qb1 = qb;
                        if (l < 0) continue;   // an empty step (lane-group uniform)
                        const float a = ax[l], da = ax[9 + l];
                        const float cm = ax[22 + m], sm = ax[31 + m];
                        const float cm1 = ax[22 + (m > 0 ? m - 1 : 0)], sm1 = ax[31 + (m > 0 ? m - 1 : 0)];
                        const float Gp = accG[k][2 * h], Gn = accG[k][2 * h + 1];
                        const float dGp = accD[k][2 * h], dGn = accD[k][2 * h + 1];
                        const float y = c2.z * qa;
                        T1 += y * (cm * (a * dGp + da * Gp) + sm * (a * dGn + da * Gn));
                        const float wc = a * Gp, ws = a * Gn, fm = y * c2.w;
                        T2x += fm * (wc * cm1 + ws * sm1);
                        T2y += fm * (ws * cm1 - wc * sm1);
                        T2z += c2.z * qb * (wc * cm + ws * sm);
                    }
                    T[h][0] = T1; T[h][1] = T2x; T[h][2] = T2y; T[h][3] = T2z;
                }
#pragma unroll
                for (int h = 0; h < 2; ++h)
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        T[h][c] += __shfl_xor_sync(0xffffffffu, T[h][c], 1);
                        T[h][c] += __shfl_xor_sync(0xffffffffu, T[h][c], 2);
                    }
                // lane t = 0 takes row r0's pair, t = 1 row r1's
                if (t < 2) {
                    const int rr = t == 0 ? r0 : r1;
                    const float *ax = aux + rr * Sh::AUX;
                    const int pp = base + rr;
                    if (pp < np && ax[40] != 0.f) {
                        const int64_t p = p0 + pp;
                        const int ja = fold_index(S.nbr[p], P.n_atoms);
                        const float u0 = ax[18], u1 = ax[19], u2 = ax[20], ir = ax[21];
                        const float T1 = T[t][0], T2x = T[t][1], T2y = T[t][2], T2z = T[t][3];
                        const float ut2 = u0 * T2x + u1 * T2y + u2 * T2z;
                        const float fx = -(T1 * u0 + (T2x - ut2 * u0) * ir);
                        const float fy = -(T1 * u1 + (T2y - ut2 * u1) * ir);
                        const float fz = -(T1 * u2 + (T2z - ut2 * u2) * ir);
                        const double X3 = S.xyz[3 * p], Y3 = S.xyz[3 * p + 1], Z3 = S.xyz[3 * p + 2];
                        atomicAdd(&O.forces[3 * (size_t)ja], (double)fx);
                        atomicAdd(&O.forces[3 * (size_t)ja + 1], (double)fy);
                        atomicAdd(&O.forces[3 * (size_t)ja + 2], (double)fz);
                        if (O.pair_grad) {
                            O.pair_grad[3 * p] = -(double)fx;
                            O.pair_grad[3 * p + 1] = -(double)fy;
                            O.pair_grad[3 * p + 2] = -(double)fz;
                        }
                        fs[0] -= fx; fs[1] -= fy; fs[2] -= fz;
                        vir[0] += (double)fx * X3;
                        vir[1] += (double)fy * Y3;
                        vir[2] += (double)fz * Z3;
                        vir[3] += 0.5 * ((double)fx * Y3 + (double)fy * X3);
                        vir[4] += 0.5 * ((double)fx * Z3 + (double)fz * X3);
                        vir[5] += 0.5 * ((double)fy * Z3 + (double)fz * Y3);
                    }
                }
            }
            __syncwarp();   // the next 32 pairs overwrite the staging
        }
#pragma unroll
        for (int qd = 0; qd < 3; ++qd) fs[qd] = warp_sum(fs[qd]);
        if (lane == 0 && O.pair_grad)
            for (int qd = 0; qd < 3; ++qd) O.pair_grad[3 * p0 + qd] = -fs[qd];
        if (lane == 0) {
            atomicAdd(&O.forces[3 * (size_t)catom], fs[0]);
            atomicAdd(&O.forces[3 * (size_t)catom + 1], fs[1]);
            atomicAdd(&O.forces[3 * (size_t)catom + 2], fs[2]);
            O.energies[catom] += I.delta2 * esum;
        }
    }
#pragma unroll
    for (int qd = 0; qd < 6; ++qd) vir[qd] = warp_sum(vir[qd]);
    if (lane == 0)
        for (int qd = 0; qd < 6; ++qd) vred[warp][qd] = vir[qd];
    if (O.vir_struct && lane == 0 && site < S.n_sites) {
        double *o = O.vir_struct + 9 * (size_t)O.atom_struct[S.site_atom[site]];
        atomicAdd(o + 0, vir[0]);
        atomicAdd(o + 4, vir[1]);
        atomicAdd(o + 8, vir[2]);
        atomicAdd(o + 1, vir[3]);
        atomicAdd(o + 3, vir[3]);
        atomicAdd(o + 2, vir[4]);
        atomicAdd(o + 6, vir[4]);
        atomicAdd(o + 5, vir[5]);
        atomicAdd(o + 7, vir[5]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double v[6] = {0, 0, 0, 0, 0, 0};
        for (int w = 0; w < Sh::WARPS; ++w)
            for (int qd = 0; qd < 6; ++qd) v[qd] += vred[w][qd];
        double *o = O.vpart + (size_t)blockIdx.x * 9;
        o[0] = v[0]; o[4] = v[1]; o[8] = v[2];
        o[1] = o[3] = v[3];
        o[2] = o[6] = v[4];
        o[5] = o[7] = v[5];
    }
}

// Grid-strided over the per-CTA partials; every block adds its sums into out
// (as do the reductions of other blocks' passes into the same virial).
__global__ void k_virial_reduce(const double *__restrict__ vpart, int nblk, double *out) {
    const int q = threadIdx.y;   // 9 components
    double s = 0.0;
    for (int b = blockIdx.x * 32 + threadIdx.x; b < nblk; b += 32 * gridDim.x)
        s += vpart[(size_t)b * 9 + q];
    s = warp_sum(s);
    if (threadIdx.x == 0) atomicAdd(out + q, s);
}

// ===================== SOAP compression =====================================

// Both compression kernels run one warp per site and stage a row of D FP64
// values per warp in shared memory; W warps per CTA with W * 8 * D bytes within
// the default 48 KB where D allows, else one warp with opt-in shared memory.

// v = C p (FP64, from a CSR copy of C by row), |v| in FP64, then q = v / |v|
// leaves as the uncompressed pass leaves it: delta = q - mu (fp32 row, bf16
// split rows) and delta . mu. Each lane reads back only the v entries it wrote.
__global__ void __launch_bounds__(256) k_compress_fwd(SoapParams P, CompressArgs C, int n_sites,
                                                      const double *__restrict__ praw, DescOut O) {
    extern __shared__ double vsh[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int site = blockIdx.x * (blockDim.x >> 5) + warp;
    if (site >= n_sites) return;
    const int D = P.dim;
    double *v = vsh + (size_t)warp * D;
    const double *p = praw + (size_t)site * C.dimf;
    double nrm2 = 0.0;
    for (int i = lane; i < D; i += 32) {
        double x = 0.0;
        for (int k = C.row_ptr[i]; k < C.row_ptr[i + 1]; ++k) x += C.row_val[k] * p[C.row_col[k]];
        v[i] = x;
        nrm2 += x * x;
    }
    nrm2 = warp_sum(nrm2);
    const double inv = nrm2 > 0.0 ? 1.0 / sqrt(nrm2) : 0.0;
    __nv_bfloat16 *qs = O.qsplit + (size_t)site * P.K1;
    float *qrow = O.q + (size_t)site * D;
    double off = 0.0;
    for (int i = lane; i < D; i += 32) {
        const double mu = P.mu[i];
        const double dl = v[i] * inv - mu;
        off += dl * mu;
        const float df = (float)dl;
        qrow[i] = df;
        __nv_bfloat16 hi, lo;
        bf16_split(df, hi, lo);
        qs[i] = hi;
        if (P.nsplit == 3) {
            qs[D + i] = hi;
            qs[2 * D + i] = lo;
        }
    }
    const int fill = P.fill_to > 0 ? P.fill_to : P.K1;
    for (int k = P.nsplit * D + lane; k < fill; k += 32) qs[k] = __float2bfloat16_rn(0.f);
    off = warp_sum(off);
    if (lane == 0) {
        O.pnorm[site] = sqrt(nrm2);
        O.qoff[site] = off;
    }
}

// dE/dq = ksum mu + g0 + g (as the force pass forms it), dE/dv = (dE/dq -
// (dE/dq . q) q) / |v| in FP64 into shared memory, then dE/dp = C^T dE/dv (fp32
// out): the row is zeroed, and the columns of C that have entries (a CSR copy of
// C by column) are written one per lane step.
__global__ void __launch_bounds__(256) k_compress_adj(SoapParams P, CompressArgs C, int n_sites,
                                                      ForceIn I, float *__restrict__ gfull) {
    extern __shared__ double hsh[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int site = blockIdx.x * (blockDim.x >> 5) + warp;
    if (site >= n_sites) return;
    const int D = P.dim;
    double *h = hsh + (size_t)warp * D;
    const float *g = I.g + (size_t)site * D;
    const float *q = I.q + (size_t)site * D;
    double ksum = 0.0;
    for (int t = lane; t < I.n_etiles; t += 32) ksum += I.kdsum[(size_t)site * I.n_etiles + t];
    ksum = warp_sum(ksum);
    double dot = 0.0;
    for (int i = lane; i < D; i += 32) {
        const double mu = P.mu[i];
        const double gi = ksum * mu + P.g0[i] + (double)g[i];
        h[i] = gi;
        dot += gi * (mu + (double)q[i]);
    }
    dot = warp_sum(dot);
    const double nrm = I.pnorm[site];
    const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
    for (int i = lane; i < D; i += 32) h[i] = (h[i] - dot * (P.mu[i] + (double)q[i])) * inv;
    __syncwarp();   // every lane reads every entry of h below
    float *out = gfull + (size_t)site * C.dimf;
    if ((C.dimf & 3) == 0) {
        float4 *o4 = reinterpret_cast<float4 *>(out);
        for (int j = lane; j < C.dimf / 4; j += 32) o4[j] = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
        for (int j = lane; j < C.dimf; j += 32) out[j] = 0.f;
    }
    __syncwarp();   // the zeros land before the columns below overwrite theirs
    for (int t = lane; t < C.ncols; t += 32) {
        double acc = 0.0;
        for (int k = C.col_ptr[t]; k < C.col_ptr[t + 1]; ++k) acc += C.col_val[k] * h[C.col_row[k]];
        out[C.col_idx[t]] = (float)acc;
    }
}

// Warps per CTA and shared bytes for the compression kernels at row length D.
static void compress_launch_shape(int D, int &warps, size_t &smem) {
    const size_t row = sizeof(double) * (size_t)D;
    warps = (int)std::max<size_t>(1, std::min<size_t>(8, (48 * 1024) / row));
    smem = row * warps;
}

template <typename K>
static int compress_smem_attr(K kernel, size_t smem) {
    if (smem > 48 * 1024)
        TGB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return TG_OK;
}

int launch_compress_forward(const SoapParams &P, const CompressArgs &C, int n_sites,
                            const double *praw, const DescOut &O, cudaStream_t st) {
    int w = 0;
    size_t smem = 0;
    compress_launch_shape(P.dim, w, smem);
    TGB_TRY(compress_smem_attr(k_compress_fwd, smem));
    if (n_sites > 0)
        k_compress_fwd<<<(n_sites + w - 1) / w, 32 * w, smem, st>>>(P, C, n_sites, praw, O);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

int launch_compress_adjoint(const SoapParams &P, const CompressArgs &C, int n_sites,
                            const ForceIn &I, float *gfull, cudaStream_t st) {
    int w = 0;
    size_t smem = 0;
    compress_launch_shape(P.dim, w, smem);
    TGB_TRY(compress_smem_attr(k_compress_adj, smem));
    if (n_sites > 0)
        k_compress_adj<<<(n_sites + w - 1) / w, 32 * w, smem, st>>>(P, C, n_sites, I, gfull);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

// ===================== launchers ============================================

#define TGB_SOAP_SHAPES(X) X(1, 8, 8) X(2, 8, 8) X(1, 8, 6) X(2, 8, 6) X(1, 4, 4) X(2, 4, 4)

bool soap_shape_supported(int ns, int amax, int lmax) {
#define X(a, b, c) if (ns == a && amax == b && lmax == c) return true;
    TGB_SOAP_SHAPES(X)
#undef X
    return false;
}

// Warps of a kernel resident on the whole GPU at once (one site per warp).
template <typename K>
static int resident_warps(K kernel, int threads, size_t smem, int *out) {
    int per_sm = 0, dev = 0, n_sm = 0;
    TGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    TGB_CUDA(cudaGetDevice(&dev));
    TGB_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    *out = std::max(1, per_sm * n_sm * (threads / 32));
    return TG_OK;
}

template <int NS, int AMAX, int LMAX, int TILE, bool RAW = false, bool MULT = false>
static int expand_impl(const SoapParams &P, const SiteArgs &S, const DescOut &O, cudaStream_t st) {
    using Sh = DescShape<NS, AMAX, LMAX, TILE>;
    const size_t smem = sizeof(float) * Sh::WARP_FLOATS * Sh::WARPS;
    static bool attr = false;
    if (!attr) {
        TGB_CUDA(cudaFuncSetAttribute(k_soap_expand<NS, AMAX, LMAX, TILE, RAW, MULT>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
    static int resident = 0;   // sites in flight at once: the L2 prefetch distance
    if (!resident)
        TGB_TRY(resident_warps(k_soap_expand<NS, AMAX, LMAX, TILE, RAW, MULT>, 32 * Sh::WARPS, smem,
                               &resident));
    SiteArgs S2 = S;
    S2.ahead = resident;
    const int grid = (S.n_sites + Sh::WARPS - 1) / Sh::WARPS;
    if (grid > 0)
        k_soap_expand<NS, AMAX, LMAX, TILE, RAW, MULT><<<grid, 32 * Sh::WARPS, smem, st>>>(P, S2, O);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

template <int NS, int AMAX, int LMAX, int TILE, bool RAW = false, bool MULT = false>
static int force_impl(const SoapParams &P, const SiteArgs &S, const ForceIn &I, const ForceOut &O,
                      int *nblk, cudaStream_t st) {
    using Sh = ForceShape<NS, AMAX, LMAX, TILE>;
    const size_t smem = sizeof(float) * Sh::WARP_FLOATS * Sh::WARPS;
    static bool attr = false;
    if (!attr) {
        TGB_CUDA(cudaFuncSetAttribute(k_soap_force<NS, AMAX, LMAX, TILE, RAW, MULT>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
    static int resident = 0;   // sites in flight at once
    if (!resident)
        TGB_TRY(resident_warps(k_soap_force<NS, AMAX, LMAX, TILE, RAW, MULT>, 32 * Sh::WARPS, smem,
                               &resident));
    ForceIn I2 = I;
    // the L2 prefetch distance: a quarter of the sites in flight ahead: the rows arrive in L2 in time and
    // stay there until used (measured: ch32k 0.552 -> 0.541 ms, ch1m unchanged)
    I2.ahead = std::max(1, resident / 4);
    const int grid = (S.n_sites + Sh::WARPS - 1) / Sh::WARPS;
    *nblk = grid;
    if (grid > 0)
        k_soap_force<NS, AMAX, LMAX, TILE, RAW, MULT><<<grid, 32 * Sh::WARPS, smem, st>>>(P, S, I2, O);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

template <int NS, int AMAX, int LMAX, bool RAW>
static int expand_tiles(const SoapParams &P, const SiteArgs &S, const DescOut &O, cudaStream_t st,
                        int tile) {
    switch (tile) {
        case 1: return expand_impl<NS, AMAX, LMAX, 1, RAW>(P, S, O, st);
        case 2: return expand_impl<NS, AMAX, LMAX, 2, RAW>(P, S, O, st);
        case 3: return expand_impl<NS, AMAX, LMAX, 3, RAW>(P, S, O, st);
        default: return expand_impl<NS, AMAX, LMAX, 0, RAW>(P, S, O, st);
    }
}

// A block with species multiplicity runs tile 0 whatever the tile asked for.
template <int NS, int AMAX, int LMAX>
static int expand_tile(const SoapParams &P, const SiteArgs &S, const DescOut &O, cudaStream_t st,
                       int tile) {
    TGB_CHECK(!P.raw || O.praw != nullptr, TG_ERR_ARG, "a compressed block needs DescOut::praw");
    if (P.n_inst > 1) {
        if constexpr (NS == 2)
            return P.raw ? expand_impl<NS, AMAX, LMAX, 0, true, true>(P, S, O, st)
                         : expand_impl<NS, AMAX, LMAX, 0, false, true>(P, S, O, st);
        set_error("species multiplicity needs two descriptor species");
        return TG_ERR_ARG;
    }
    if (P.raw) return expand_tiles<NS, AMAX, LMAX, true>(P, S, O, st, tile);
    return expand_tiles<NS, AMAX, LMAX, false>(P, S, O, st, tile);
}

template <int NS, int PREC>
static int force_mma_impl(const SoapParams &P, const SiteArgs &S, const ForceIn &I,
                          const ForceOut &O, int *nblk, cudaStream_t st) {
    using Sh = MmaForceShape<NS>;
    const size_t smem = sizeof(float) * Sh::WARP_FLOATS * Sh::WARPS;
    static bool attr = false;
    if (!attr) {
        TGB_CUDA(cudaFuncSetAttribute(k_soap_force_mma<NS, PREC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
    static int resident = 0;   // sites in flight at once: the L2 prefetch distance
    if (!resident)
        TGB_TRY(resident_warps(k_soap_force_mma<NS, PREC>, 32 * Sh::WARPS, smem, &resident));
    ForceIn I2 = I;
    I2.ahead = resident;
    const int grid = (S.n_sites + Sh::WARPS - 1) / Sh::WARPS;
    *nblk = grid;
    if (grid > 0) k_soap_force_mma<NS, PREC><<<grid, 32 * Sh::WARPS, smem, st>>>(P, S, I2, O);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

bool soap_force_mma_supported(const SoapParams &P) {
    return !P.raw && P.n_inst == 1 && P.amax == 8 && P.lmax == 8 && (P.ns == 1 || P.ns == 2);
}

static int launch_soap_force_mma(const SoapParams &P, const SiteArgs &S, const ForceIn &I,
                                 const ForceOut &O, int *nblk, cudaStream_t st) {
    TGB_CHECK(I.qoff && P.muf && P.g0f, TG_ERR_ARG, "the force pass needs qoff, muf and g0f");
    const bool fast = P.force_prec == 1;
    if (P.ns == 1)
        return fast ? force_mma_impl<1, 1>(P, S, I, O, nblk, st)
                    : force_mma_impl<1, 3>(P, S, I, O, nblk, st);
    return fast ? force_mma_impl<2, 1>(P, S, I, O, nblk, st)
                : force_mma_impl<2, 3>(P, S, I, O, nblk, st);
}

template <int NS, int AMAX, int LMAX, bool RAW>
static int force_tiles(const SoapParams &P, const SiteArgs &S, const ForceIn &I, const ForceOut &O,
                       int *nblk, cudaStream_t st, int tile) {
    switch (tile) {
        case 1: return force_impl<NS, AMAX, LMAX, 1, RAW>(P, S, I, O, nblk, st);
        case 2: return force_impl<NS, AMAX, LMAX, 2, RAW>(P, S, I, O, nblk, st);
        case 3: return force_impl<NS, AMAX, LMAX, 3, RAW>(P, S, I, O, nblk, st);
        default: return force_impl<NS, AMAX, LMAX, 0, RAW>(P, S, I, O, nblk, st);
    }
}

template <int NS, int AMAX, int LMAX>
static int force_tile(const SoapParams &P, const SiteArgs &S, const ForceIn &I, const ForceOut &O,
                      int *nblk, cudaStream_t st, int tile) {
    TGB_CHECK(P.raw || (I.qoff && P.muf && P.g0f), TG_ERR_ARG,
              "the force pass needs qoff, muf and g0f");
    if (P.n_inst > 1) {
        if constexpr (NS == 2)
            return P.raw ? force_impl<NS, AMAX, LMAX, 0, true, true>(P, S, I, O, nblk, st)
                         : force_impl<NS, AMAX, LMAX, 0, false, true>(P, S, I, O, nblk, st);
        set_error("species multiplicity needs two descriptor species");
        return TG_ERR_ARG;
    }
    if (P.raw) return force_tiles<NS, AMAX, LMAX, true>(P, S, I, O, nblk, st, tile);
    return force_tiles<NS, AMAX, LMAX, false>(P, S, I, O, nblk, st, tile);
}

int launch_soap_expand(const SoapParams &P, const SiteArgs &S, const DescOut &O, cudaStream_t st,
                       int tile) {
#define X(a, b, c) \
    if (P.ns == a && P.amax == b && P.lmax == c) return expand_tile<a, b, c>(P, S, O, st, tile);
    TGB_SOAP_SHAPES(X)
#undef X
    set_error("unsupported SOAP shape: n_species %d alpha_max %d l_max %d", P.ns, P.amax, P.lmax);
    return TG_ERR_ARG;
}

int launch_soap_force(const SoapParams &P, const SiteArgs &S, const ForceIn &I, const ForceOut &O,
                      int *nblk, cudaStream_t st, int tile) {
    if (tile == kForceTileMma) {
        TGB_CHECK(soap_force_mma_supported(P), TG_ERR_ARG,
                  "the tensor-core force tile needs alpha_max 8, l_max 8, 1 or 2 species and no "
                  "compression");
        return launch_soap_force_mma(P, S, I, O, nblk, st);
    }
#define X(a, b, c) \
    if (P.ns == a && P.amax == b && P.lmax == c)    \
        return force_tile<a, b, c>(P, S, I, O, nblk, st, tile);
    TGB_SOAP_SHAPES(X)
#undef X
    set_error("unsupported SOAP shape: n_species %d alpha_max %d l_max %d", P.ns, P.amax, P.lmax);
    return TG_ERR_ARG;
}

int launch_virial_reduce(const double *vpart, int nblk, double *virial_out, cudaStream_t st) {
    if (nblk <= 0) return TG_OK;
    // about 128 partials per block (four per lane), at most 1024 blocks
    const int grid = std::min(1024, (nblk + 127) / 128);
    k_virial_reduce<<<grid, dim3(32, 9), 0, st>>>(vpart, nblk, virial_out);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

}  // namespace tgb
