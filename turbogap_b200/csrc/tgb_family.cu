// tgb_family.cu -- distance_2b, core_pot and angle_3b energies, forces and virial
// on the device (src/gap.f90:400-1042), in FP64.
//
// One warp per central site. 2b and core_pot run a lane per neighbour pair;
// angle_3b runs a lane per (j < k) pair of neighbours, the triangle of the
// site's list flattened over the lanes so that every lane has work. The
// per-sparse-point sums of the 3b forces are folded: the three force vectors
// are linear in sum_s w_s dq_s (w_s = kernel or its derivative), so each
// triplet accumulates four scalars over the sparse set instead of nine
// vectors. Forces on the central site are reduced in the warp; 3b forces on
// neighbours and the energies are added atomically, the virial once per block.
#include "tgb_family.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace tgb {
namespace {

constexpr int FW = 4;                 // warps per block
constexpr double kBuffer = 0.5;       // gap_backend_cpu.f90:152,252 pass 0.5d0

struct FamArgs {
    int kind, n, pol;
    int sp0, sp1, sp2;
    double inv_s2[3];
    double rcut;
    double yp1, ypn;
    const double *p;
};

__device__ __forceinline__ int fold_atom(int j, int n) { return j < n ? j : j % n; }

__device__ __forceinline__ void cutoff_fn(double r, double rcut, double &fc, double &dfc) {
    // the cosine taper over the last 0.5 A before rcut (gap.f90:487-494)
    if (r < rcut - kBuffer) {
        fc = 1.0;
        dfc = 0.0;
    } else {
        const double t = 3.14159265358979323846 * (r - rcut + kBuffer) / kBuffer;
        fc = 0.5 * (cos(t) + 1.0);
        dfc = 0.5 * 3.14159265358979323846 / kBuffer * sin(t);
    }
}

// Cubic spline of the core_pot table (x, V, y2 interleaved in sp): value and
// slope; linear continuation with the end slopes outside the table.
__device__ __forceinline__ void spline_eval(const double *sp, int n, double yp1, double ypn, double r,
                                            double &v, double &dv) {
    const double x0 = sp[0], xn = sp[3 * (n - 1)];
    if (r < x0) {
        v = sp[1] + (r - x0) * yp1;
        dv = yp1;
        return;
    }
    if (r > xn) {
        v = sp[3 * (n - 1) + 1] + (r - xn) * ypn;
        dv = ypn;
        return;
    }
    // the interval [x_j, x_j+1) holding r: the first j with r < x_j+1 (last interval at x_n)
    int lo = 0, hi = n - 2;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (r < sp[3 * (mid + 1)]) hi = mid;
        else lo = mid + 1;
    }
    const int j = lo;
    const double xa = sp[3 * j], xb = sp[3 * (j + 1)];
    const double h = xb - xa;
    const double A = (xb - r) / h, B = 1.0 - A;
    const double ya = sp[3 * j + 1], yb = sp[3 * (j + 1) + 1];
    const double za = sp[3 * j + 2], zb = sp[3 * (j + 1) + 2];
    v = A * ya + B * yb + ((A * A * A - A) * za + (B * B * B - B) * zb) * (h * h / 6.0);
    dv = (yb - ya) / h + ((1.0 - 3.0 * A * A) * za + (3.0 * B * B - 1.0) * zb) * (h / 6.0);
}

// Sums a lane's packed virial (xx yy zz xy xz yz) over the block into vir (3 x 3).
__device__ __forceinline__ void block_virial(double (&v)[6], double *vir) {
    __shared__ double red[FW][6];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < 6; ++q) v[q] = warp_sum(v[q]);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 6; ++q) red[warp][q] = v[q];
    __syncthreads();
    if (threadIdx.x < 6) {
        double s = 0.0;
        for (int w = 0; w < FW; ++w) s += red[w][threadIdx.x];
        const int q = threadIdx.x;
        if (s != 0.0) {
            if (q < 3) {
                atomicAdd(vir + 4 * q, s);
            } else {
                const int a = q == 5 ? 1 : 0, b = q == 3 ? 1 : 2;
                atomicAdd(vir + a + 3 * b, s);
                atomicAdd(vir + b + 3 * a, s);
            }
        }
    }
}

// lane contribution w (f x^T + x f^T) to the packed virial
__device__ __forceinline__ void vir_add(double (&v)[6], double f0, double f1, double f2, double x0,
                                        double x1, double x2, double w) {
    v[0] += 2.0 * w * f0 * x0;
    v[1] += 2.0 * w * f1 * x1;
    v[2] += 2.0 * w * f2 * x2;
    v[3] += w * (f0 * x1 + f1 * x0);
    v[4] += w * (f0 * x2 + f2 * x0);
    v[5] += w * (f1 * x2 + f2 * x1);
}

// distance_2b (gap.f90:400-563) and core_pot (gap.f90:565-721): energy 1/2 V or
// sum_s w_s fc exp(-(r - Q_s)^2 / 2 sigma^2) per directed pair, force on the site.
template <int KIND>
__global__ void __launch_bounds__(32 * FW) k_family_pair(FamArgs F, SiteArgs S, const double *rjs,
                                                          int n_atoms, double *en, double *fo,
                                                          double *vir) {
    extern __shared__ double sp[];
    const int np_par = (KIND == TG_FAMILY_2B ? 2 : 3) * F.n;
    for (int t = threadIdx.x; t < np_par; t += blockDim.x) sp[t] = F.p[t];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int site = blockIdx.x * FW + warp;
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (site < S.n_sites) {
        const int row = S.site_row[site], atom = S.site_atom[site];
        const int zi = S.species[atom];
        if (zi == F.sp0 || zi == F.sp1) {
            const int64_t p0 = S.pstart[row];
            const int np = (int)(S.pstart[row + 1] - p0);
            double e = 0.0, f[3] = {0, 0, 0};
            for (int pp = 1 + lane; pp < np; pp += 32) {
                const int64_t p = p0 + pp;
                const int zj = S.species[fold_atom(S.nbr[p], n_atoms)];
                if (!((zi == F.sp0 && zj == F.sp1) || (zi == F.sp1 && zj == F.sp0))) continue;
                const double r = rjs[p];
                if (!(r < F.rcut)) continue;
                const double x0 = S.xyz[3 * p], x1 = S.xyz[3 * p + 1], x2 = S.xyz[3 * p + 2];
                double g;
                if constexpr (KIND == TG_FAMILY_2B) {
                    double fc, dfc;
                    cutoff_fn(r, F.rcut, fc, dfc);
                    double es = 0.0, gs = 0.0;
                    for (int s = 0; s < F.n; ++s) {
                        const double dr = r - sp[2 * s], w = sp[2 * s + 1];
                        const double we = w * exp(-0.5 * dr * dr * F.inv_s2[0]);
                        es += we;
                        gs += we * (dr * F.inv_s2[0] * fc + dfc);
                    }
                    e += fc * es;
                    g = -2.0 * gs;
                } else {
                    double vv, dv;
                    spline_eval(sp, F.n, F.yp1, F.ypn, r, vv, dv);
                    e += 0.5 * vv;
                    g = dv;
                }
                const double g_r = g / r;
                const double f0 = g_r * x0, f1 = g_r * x1, f2 = g_r * x2;
                f[0] += f0;
                f[1] += f1;
                f[2] += f2;
                vir_add(v, f0, f1, f2, x0, x1, x2, -0.25);
            }
            e = warp_sum(e);
#pragma unroll
            for (int q = 0; q < 3; ++q) f[q] = warp_sum(f[q]);
            if (lane == 0) {
                atomicAdd(en + atom, e);
#pragma unroll
                for (int q = 0; q < 3; ++q) atomicAdd(fo + 3 * (size_t)atom + q, f[q]);
            }
        }
    }
    block_virial(v, vir);
}

__device__ __forceinline__ double cov_pp(double r) {   // gap.f90:1049-1080, d = 3, q = 1
    if (r >= 1.0) return 0.0;
    if (r <= 0.0) return 1.0;
    const double om = 1.0 - r, om2 = om * om;
    return om2 * om2 * (4.0 * r + 1.0);
}
__device__ __forceinline__ double cov_pp_der(double r) {   // gap.f90:1081-1112
    if (r >= 1.0 || r <= 0.0) return 0.0;
    const double om = 1.0 - r, om3 = om * om * om;
    return (-4.0 * om3 * (4.0 * r + 1.0) + 4.0 * om3 * om) / r;
}

// angle_3b (gap.f90:724-1042): triplets (i; j < k) of the site's list with
// descriptor q = (r_ij + r_ik, (r_ij - r_ik)^2, r_jk).
__global__ void __launch_bounds__(32 * FW) k_family_3b(FamArgs F, SiteArgs S, const double *rjs,
                                                        int n_atoms, double *en, double *fo,
                                                        double *vir) {
    extern __shared__ double sp[];
    for (int t = threadIdx.x; t < 4 * F.n; t += blockDim.x) sp[t] = F.p[t];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int site = blockIdx.x * FW + warp;
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (site < S.n_sites) {
        const int row = S.site_row[site], atom = S.site_atom[site];
        if (S.species[atom] == F.sp0) {
            const int64_t p0 = S.pstart[row];
            const int m = (int)(S.pstart[row + 1] - p0) - 1;   // pairs after the self pair
            const int64_t T = (int64_t)m * (m - 1) / 2;
            double e = 0.0, fi[3] = {0, 0, 0};
            for (int64_t t = lane; t < T; t += 32) {
                // row a of the strict upper triangle holds m - 1 - a entries
                int a = (int)floor(((2.0 * m - 1.0) - sqrt((2.0 * m - 1.0) * (2.0 * m - 1.0) - 8.0 * (double)t)) * 0.5);
                a = max(0, min(a, m - 2));
                while (a > 0 && (int64_t)a * (2 * m - a - 1) / 2 > t) --a;
                while (a < m - 2 && (int64_t)(a + 1) * (2 * m - a - 2) / 2 <= t) ++a;
                const int b = (int)(t - (int64_t)a * (2 * m - a - 1) / 2) + a + 1;
                const int64_t kj = p0 + 1 + a, kk = p0 + 1 + b;
                const int ja = fold_atom(S.nbr[kj], n_atoms), ka = fold_atom(S.nbr[kk], n_atoms);
                const int zj = S.species[ja], zk = S.species[ka];
                const double r12 = rjs[kj], r13 = rjs[kk];
                if ((zj != F.sp1 && zj != F.sp2) || r12 > F.rcut) continue;
                if (!(((zj == F.sp1 && zk == F.sp2) || (zj == F.sp2 && zk == F.sp1)) && r13 < F.rcut))
                    continue;
                if (!(r12 < F.rcut)) continue;
                const double x12[3] = {S.xyz[3 * kj], S.xyz[3 * kj + 1], S.xyz[3 * kj + 2]};
                const double x13[3] = {S.xyz[3 * kk], S.xyz[3 * kk + 1], S.xyz[3 * kk + 2]};
                const double x23[3] = {x13[0] - x12[0], x13[1] - x12[1], x13[2] - x12[2]};
                const double r23 = sqrt(x23[0] * x23[0] + x23[1] * x23[1] + x23[2] * x23[2]);
                double u12[3], u13[3], u23[3];
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    u12[q] = x12[q] / r12;
                    u13[q] = x13[q] / r13;
                    u23[q] = x23[q] / r23;
                }
                double fc12, d12, fc13, d13;
                cutoff_fn(r12, F.rcut, fc12, d12);
                cutoff_fn(r13, F.rcut, fc13, d13);
                const double fc = fc12 * fc13;
                const double q1 = r12 + r13, q2 = (r12 - r13) * (r12 - r13), q3 = r23;
                // esum = sum_s k_s; (A, B, C) = sum_s w_s dq_s with w = k (exp) or k' (pol)
                double esum = 0.0, A = 0.0, B = 0.0, C = 0.0;
                for (int s = 0; s < F.n; ++s) {
                    const double e1 = (q1 - sp[4 * s]) * F.inv_s2[0];
                    const double e2 = (q2 - sp[4 * s + 1]) * F.inv_s2[1];
                    const double e3 = (q3 - sp[4 * s + 2]) * F.inv_s2[2];
                    const double rr2 = (q1 - sp[4 * s]) * e1 + (q2 - sp[4 * s + 1]) * e2 +
                                       (q3 - sp[4 * s + 2]) * e3;
                    const double pref = sp[4 * s + 3];
                    double k, w;
                    if (F.pol) {
                        const double rr = sqrt(rr2);
                        k = pref * cov_pp(rr);
                        w = pref * cov_pp_der(rr);
                    } else {
                        k = pref * exp(-0.5 * rr2);
                        w = k;
                    }
                    esum += k;
                    A += w * e1;
                    B += w * e2;
                    C += w * e3;
                }
                e += fc * esum;
                // exp: a = esum dfc + fc sum_s k d; pol: a = esum dfc - fc sum_s k' d
                const double sg = F.pol ? -fc : fc;
                const double dd = 2.0 * (r12 - r13);
                double f1[3], f2[3], f3[3];
#pragma unroll
                for (int l = 0; l < 3; ++l) {
                    const double D1 = A * (u12[l] + u13[l]) + B * dd * (u12[l] - u13[l]);
                    const double D2 = -A * u12[l] - B * dd * u12[l] + C * u23[l];
                    const double D3 = -A * u13[l] + B * dd * u13[l] - C * u23[l];
                    const double dfl = fc12 * d13 * u13[l] + fc13 * d12 * u12[l];
                    f1[l] = -(esum * dfl + sg * D1);
                    f2[l] = -(-esum * fc13 * d12 * u12[l] + sg * D2);
                    f3[l] = -(-esum * fc12 * d13 * u13[l] + sg * D3);
                }
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    fi[q] += f1[q];
                    atomicAdd(fo + 3 * (size_t)ja + q, f2[q]);
                    atomicAdd(fo + 3 * (size_t)ka + q, f3[q]);
                }
                vir_add(v, f2[0], f2[1], f2[2], x12[0], x12[1], x12[2], 0.5);
                vir_add(v, f3[0], f3[1], f3[2], x13[0], x13[1], x13[2], 0.5);
            }
            e = warp_sum(e);
#pragma unroll
            for (int q = 0; q < 3; ++q) fi[q] = warp_sum(fi[q]);
            if (lane == 0) {
                atomicAdd(en + atom, e);
#pragma unroll
                for (int q = 0; q < 3; ++q) atomicAdd(fo + 3 * (size_t)atom + q, fi[q]);
            }
        }
    }
    block_virial(v, vir);
}

// read_files.f90:5454-5505: second derivatives of the interpolating cubic spline
// (the tridiagonal system solved by forward elimination and back substitution),
// with a natural end wherever the given slope exceeds 0.99e30; such an end slope
// is then replaced by the spline's own slope there.
void core_pot_spline(int n, const double *x, const double *V, double &yp1, double &ypn,
                     std::vector<double> &y2) {
    y2.assign(n, 0.0);
    std::vector<double> u(n, 0.0);
    if (!(yp1 > 0.99e30)) {
        y2[0] = -0.5;
        u[0] = 3.0 / (x[1] - x[0]) * ((V[1] - V[0]) / (x[1] - x[0]) - yp1);
    }
    for (int i = 1; i + 1 < n; ++i) {
        const double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
        const double piv = sig * y2[i - 1] + 2.0;
        y2[i] = (sig - 1.0) / piv;
        const double slope_jump = (V[i + 1] - V[i]) / (x[i + 1] - x[i]) - (V[i] - V[i - 1]) / (x[i] - x[i - 1]);
        u[i] = (6.0 * slope_jump / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / piv;
    }
    double qn = 0.0, un = 0.0;
    if (!(ypn > 0.99e30)) {
        qn = 0.5;
        un = 3.0 / (x[n - 1] - x[n - 2]) * (ypn - (V[n - 1] - V[n - 2]) / (x[n - 1] - x[n - 2]));
    }
    y2[n - 1] = (un - qn * u[n - 2]) / (qn * y2[n - 2] + 1.0);
    for (int i = n - 2; i >= 0; --i) y2[i] = y2[i] * y2[i + 1] + u[i];
    auto slope_at = [&](int j, double r) {
        const double h = x[j + 1] - x[j];
        const double A = (x[j + 1] - r) / h, B = 1.0 - A;
        return (V[j + 1] - V[j]) / h + ((1.0 - 3.0 * A * A) * y2[j] + (3.0 * B * B - 1.0) * y2[j + 1]) * (h / 6.0);
    };
    if (yp1 > 0.99e30) yp1 = slope_at(0, x[0]);
    if (ypn > 0.99e30) ypn = slope_at(n - 2, x[n - 1]);
}

}  // namespace

int family_create(const tg_family &f, Family &F) {
    TGB_CHECK(f.kind == TG_FAMILY_2B || f.kind == TG_FAMILY_3B || f.kind == TG_FAMILY_CORE_POT,
              TG_ERR_ARG, "unknown family kind %d", f.kind);
    TGB_CHECK(f.n >= (f.kind == TG_FAMILY_CORE_POT ? 2 : 1) && f.n <= kFamilyMaxN, TG_ERR_ARG,
              "family size %d outside [1, %d]", f.n, kFamilyMaxN);
    F.kind = f.kind;
    F.n = f.n;
    for (int q = 0; q < 3; ++q) F.sp[q] = f.species[q];
    std::vector<double> h;
    if (f.kind == TG_FAMILY_CORE_POT) {
        TGB_CHECK(f.x && f.V, TG_ERR_ARG, "core_pot needs its table");
        for (int i = 1; i < f.n; ++i)
            TGB_CHECK(f.x[i] > f.x[i - 1], TG_ERR_ARG, "core_pot nodes must increase (node %d)", i);
        double yp1 = f.yp1, ypn = f.ypn;
        std::vector<double> y2;
        core_pot_spline(f.n, f.x, f.V, yp1, ypn, y2);
        F.yp1 = yp1;
        F.ypn = ypn;
        F.rcut = f.x[f.n - 1];   // gap.f90:605: rcut = maxval(x)
        h.resize(3 * (size_t)f.n);
        for (int i = 0; i < f.n; ++i) {
            h[3 * i] = f.x[i];
            h[3 * i + 1] = f.V[i];
            h[3 * i + 2] = y2[i];
        }
    } else {
        TGB_CHECK(f.Qs && f.alphas && f.cutoff, TG_ERR_ARG, "family needs Qs, alphas and cutoff");
        TGB_CHECK(f.rcut > kBuffer, TG_ERR_ARG, "family rcut %.3f must exceed the 0.5 A buffer", f.rcut);
        F.rcut = f.rcut;
        const int nsig = f.kind == TG_FAMILY_2B ? 1 : 3;
        for (int q = 0; q < nsig; ++q) {
            TGB_CHECK(f.sigma[q] > 0.0, TG_ERR_ARG, "family sigma must be positive");
            F.sigma[q] = f.sigma[q];
        }
        const double d2 = f.delta * f.delta;
        if (f.kind == TG_FAMILY_2B) {
            h.resize(2 * (size_t)f.n);
            for (int s = 0; s < f.n; ++s) {
                h[2 * s] = f.Qs[s];
                h[2 * s + 1] = d2 * f.alphas[s] * f.cutoff[s];
            }
        } else {
            TGB_CHECK(f.kernel_type == TG_KERNEL_EXP || f.kernel_type == TG_KERNEL_POL, TG_ERR_ARG,
                      "3b kernel_type must be exp or pol");
            F.pol = f.kernel_type == TG_KERNEL_POL;
            h.resize(4 * (size_t)f.n);
            for (int s = 0; s < f.n; ++s) {
                for (int q = 0; q < 3; ++q) h[4 * s + q] = f.Qs[s + (size_t)q * f.n];
                h[4 * s + 3] = 2.0 * d2 * f.alphas[s] * f.cutoff[s];
            }
        }
    }
    dev_free(F.p);
    TGB_TRY(dev_alloc(&F.p, h.size()));
    TGB_CUDA(cudaMemcpy(F.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
    return TG_OK;
}

void family_sites(const Family &F, const int *species_h, int beg, int end, std::vector<int> &out) {
    out.clear();
    for (int i = beg; i < end; ++i) {
        const int z = species_h[i];
        const bool c = F.kind == TG_FAMILY_3B ? z == F.sp[0] : (z == F.sp[0] || z == F.sp[1]);
        if (c) out.push_back(i);
    }
}

int evaluate_family(const Family &F, const SiteArgs &S, const double *rjs, int n_atoms, double *en,
                    double *fo, double *vir, cudaStream_t st) {
    if (S.n_sites <= 0) return TG_OK;
    FamArgs A{};
    A.kind = F.kind;
    A.n = F.n;
    A.pol = F.pol;
    A.sp0 = F.sp[0];
    A.sp1 = F.sp[1];
    A.sp2 = F.sp[2];
    for (int q = 0; q < 3; ++q) A.inv_s2[q] = 1.0 / (F.sigma[q] * F.sigma[q]);
    A.rcut = F.rcut;
    A.yp1 = F.yp1;
    A.ypn = F.ypn;
    A.p = F.p;
    const int grid = (S.n_sites + FW - 1) / FW;
    const int per = F.kind == TG_FAMILY_2B ? 2 : F.kind == TG_FAMILY_3B ? 4 : 3;
    const size_t smem = sizeof(double) * per * (size_t)F.n;
    static bool attr[4] = {};
    auto setattr = [&](const void *k, int idx) -> int {
        if (!attr[idx]) {
            TGB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)(sizeof(double) * 4 * kFamilyMaxN)));
            attr[idx] = true;
        }
        return TG_OK;
    };
    if (F.kind == TG_FAMILY_2B) {
        TGB_TRY(setattr((const void *)k_family_pair<TG_FAMILY_2B>, 1));
        k_family_pair<TG_FAMILY_2B><<<grid, 32 * FW, smem, st>>>(A, S, rjs, n_atoms, en, fo, vir);
    } else if (F.kind == TG_FAMILY_CORE_POT) {
        TGB_TRY(setattr((const void *)k_family_pair<TG_FAMILY_CORE_POT>, 3));
        k_family_pair<TG_FAMILY_CORE_POT><<<grid, 32 * FW, smem, st>>>(A, S, rjs, n_atoms, en, fo, vir);
    } else {
        TGB_TRY(setattr((const void *)k_family_3b, 2));
        k_family_3b<<<grid, 32 * FW, smem, st>>>(A, S, rjs, n_atoms, en, fo, vir);
    }
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

}  // namespace tgb
