// tg_oracle.cpp -- FP64 CPU restatement of the TurboGAP SOAP-GAP path.
//
// TEST INFRASTRUCTURE ONLY (the checker for the CUDA backend; never linked by
// the product). See tg_oracle.h for the parity status of each part.
//
// Build: make -C oracle   (g++ -O2 -fopenmp -ffp-contract=off)
// -ffp-contract=off keeps a*b+c as two roundings, as the reference's gfortran
// build does on x86-64 without -march flags; the neighbour-list geometry is
// compared bit for bit against the GPU and must not be contracted.

#include "tg_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;

// Fortran MODULO for reals as gfortran evaluates it (fmod, then shift into the
// sign of p; exact zero takes the sign of p).
inline double f_modulo(double a, double p) {
    double r = std::fmod(a, p);
    if (r != 0.0) {
        if ((a < 0.0) != (p < 0.0)) r += p;
    } else {
        r = std::copysign(0.0, p);
    }
    return r;
}

inline double dot3(const double *x, const double *y) {
    double s = 0.0;
    s = s + x[0] * y[0];
    s = s + x[1] * y[1];
    s = s + x[2] * y[2];
    return s;
}

inline void cross3(const double *a, const double *b, double *c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// Cache-blocked FP64 GEMMs standing in for BLAS dgemm (the reference links a
// system BLAS). AVX2/FMA clones are selected at run time; OpenMP over rows.
// C[n x m] = A[n x k] . B[m x k]^T (all row-major)
__attribute__((target_clones("avx2,fma", "default"), optimize("fp-contract=fast")))
void gemm_nt_blocked(int n, int m, int k, const double *A, const double *B, double *C) {
    const int BI = 16, BS = 96;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i0 = 0; i0 < n; i0 += BI) {
        const int i1 = std::min(n, i0 + BI);
        for (int s0 = 0; s0 < m; s0 += BS) {
            const int s1 = std::min(m, s0 + BS);
            for (int i = i0; i < i1; ++i) {
                const double *a = A + (size_t)i * k;
                for (int s = s0; s < s1; ++s) {
                    const double *b = B + (size_t)s * k;
                    double acc = 0.0;
#pragma omp simd reduction(+ : acc)
                    for (int d = 0; d < k; ++d) acc += a[d] * b[d];
                    C[(size_t)i * m + s] = acc;
                }
            }
        }
    }
}

// C[n x m] = A[n x k] . B[k x m] (all row-major), C zeroed by the caller.
__attribute__((target_clones("avx2,fma", "default"), optimize("fp-contract=fast")))
void gemm_nn_blocked(int n, int m, int k, const double *A, const double *B, double *C) {
    const int BI = 16, BS = 64;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i0 = 0; i0 < n; i0 += BI) {
        const int i1 = std::min(n, i0 + BI);
        for (int s0 = 0; s0 < k; s0 += BS) {
            const int s1 = std::min(k, s0 + BS);
            for (int i = i0; i < i1; ++i) {
                double *c = C + (size_t)i * m;
                for (int s = s0; s < s1; ++s) {
                    const double f = A[(size_t)i * k + s];
                    const double *b = B + (size_t)s * m;
#pragma omp simd
                    for (int d = 0; d < m; ++d) c[d] += f * b[d];
                }
            }
        }
    }
}

inline bool box_is_orthorhombic(const double *a, const double *b, const double *c) {
    const double tol = 1.e-6;
    return std::fabs(a[1]) < tol && std::fabs(a[2]) < tol && std::fabs(b[0]) < tol &&
           std::fabs(b[2]) < tol && std::fabs(c[0]) < tol && std::fabs(c[1]) < tol;
}

}  // namespace

extern "C" {

int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

// neighbors.f90:47-163 (get_distance), PBC on all three axes.
void orc_get_distance(const double *posi, const double *posj, const double *a,
                      const double *b, const double *c, double *dist, double *d,
                      int *i_shift) {
    if (box_is_orthorhombic(a, b, c)) {
        for (int i = 0; i < 3; ++i) dist[i] = posj[i] - posi[i];
        i_shift[0] = (int)std::floor(dist[0] / a[0]);
        i_shift[1] = (int)std::floor(dist[1] / b[1]);
        i_shift[2] = (int)std::floor(dist[2] / c[2]);
        const double L[3] = {a[0], b[1], c[2]};
        double d2 = 0.0;
        for (int i = 0; i < 3; ++i) {
            dist[i] = f_modulo(posj[i] - posi[i], L[i]);
            if (dist[i] > L[i] / 2.0) dist[i] = dist[i] - L[i];
            d2 = d2 + dist[i] * dist[i];
        }
        *d = std::sqrt(d2);
        return;
    }
    // Triclinic: Gram inverse, then the 27 integer images around the real solution.
    double mat[3][3], inv[3][3];
    mat[0][0] = dot3(a, a); mat[0][1] = dot3(a, b); mat[0][2] = dot3(a, c);
    mat[1][0] = mat[0][1];  mat[1][1] = dot3(b, b); mat[1][2] = dot3(b, c);
    mat[2][0] = mat[0][2];  mat[2][1] = mat[1][2];  mat[2][2] = dot3(c, c);
    double md = -mat[0][2] * mat[0][2] * mat[1][1] + 2.0 * mat[0][1] * mat[0][2] * mat[1][2] -
                mat[0][0] * mat[1][2] * mat[1][2] - mat[0][1] * mat[0][1] * mat[2][2] +
                mat[0][0] * mat[1][1] * mat[2][2];
    inv[0][0] = mat[1][1] * mat[2][2] - mat[1][2] * mat[1][2];
    inv[0][1] = mat[0][2] * mat[1][2] - mat[0][1] * mat[2][2];
    inv[0][2] = mat[0][1] * mat[1][2] - mat[0][2] * mat[1][1];
    inv[1][0] = inv[0][1];
    inv[1][1] = mat[0][0] * mat[2][2] - mat[0][2] * mat[0][2];
    inv[1][2] = mat[0][1] * mat[0][2] - mat[0][0] * mat[1][2];
    inv[2][0] = inv[0][2];
    inv[2][1] = inv[1][2];
    inv[2][2] = mat[0][0] * mat[1][1] - mat[0][1] * mat[0][1];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) inv[i][j] = inv[i][j] / md;
    double dd[3];
    for (int i = 0; i < 3; ++i) dd[i] = posj[i] - posi[i];
    double v[3] = {-1.0 * dot3(dd, a), -1.0 * dot3(dd, b), -1.0 * dot3(dd, c)};
    double ir[3];
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int j = 0; j < 3; ++j) s = s + inv[i][j] * v[j];
        ir[i] = s;
    }
    int idx[3];
    for (int i = 0; i < 3; ++i) {
        i_shift[i] = (int)std::floor(-ir[i]);
        idx[i] = (int)std::lround(ir[i]);
    }
    double res_opt = 1.e10, opt[3] = {0, 0, 0};
    for (int i = idx[0] - 1; i <= idx[0] + 1; ++i)
        for (int j = idx[1] - 1; j <= idx[1] + 1; ++j)
            for (int k = idx[2] - 1; k <= idx[2] + 1; ++k) {
                double t[3];
                for (int q = 0; q < 3; ++q)
                    t[q] = dd[q] + (double)i * a[q] + (double)j * b[q] + (double)k * c[q];
                double res = dot3(t, t);
                if (res < res_opt) {
                    res_opt = res;
                    opt[0] = t[0]; opt[1] = t[1]; opt[2] = t[2];
                }
            }
    for (int q = 0; q < 3; ++q) dist[q] = opt[q];
    *d = std::sqrt(dot3(dist, dist));
}

// neighbors.f90:175-236
void orc_number_of_unit_cells(const double *a, const double *b, const double *c,
                              double rcut, int *indices) {
    double axb[3], cxa[3], bxc[3];
    cross3(a, b, axb);
    cross3(c, a, cxa);
    cross3(b, c, bxc);
    double n1 = std::sqrt(dot3(axb, axb)), n2 = std::sqrt(dot3(cxa, cxa)),
           n3 = std::sqrt(dot3(bxc, bxc));
    for (int i = 0; i < 3; ++i) { axb[i] /= n1; cxa[i] /= n2; bxc[i] /= n3; }
    double m[3][3] = {{dot3(axb, a), dot3(axb, b), dot3(axb, c)},
                      {dot3(cxa, a), dot3(cxa, b), dot3(cxa, c)},
                      {dot3(bxc, a), dot3(bxc, b), dot3(bxc, c)}};
    double md = -m[0][2] * m[1][1] * m[2][0] + m[0][1] * m[1][2] * m[2][0] +
                m[0][2] * m[1][0] * m[2][1] - m[0][0] * m[1][2] * m[2][1] -
                m[0][1] * m[1][0] * m[2][2] + m[0][0] * m[1][1] * m[2][2];
    double inv[3][3];
    inv[0][0] = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    inv[0][1] = m[0][2] * m[2][1] - m[0][1] * m[2][2];
    inv[0][2] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
    inv[1][0] = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    inv[1][1] = m[0][0] * m[2][2] - m[0][2] * m[2][0];
    inv[1][2] = m[0][2] * m[1][0] - m[0][0] * m[1][2];
    inv[2][0] = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    inv[2][1] = m[0][1] * m[2][0] - m[0][0] * m[2][1];
    inv[2][2] = m[0][0] * m[1][1] - m[0][1] * m[1][0];
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int j = 0; j < 3; ++j) s = s + (inv[i][j] / md) * (2.0 * rcut);
        s = std::fabs(s);
        int k = (int)s;
        if (s > (double)k) k = k + 1;
        indices[i] = k;
    }
}

// read_files.f90:320-380: replicas ordered a-index, then b, then c, then atom.
void orc_make_supercell(int n_sites, const double *positions, const int *species,
                        const double *a, const double *b, const double *c,
                        const int *indices, double *positions_sc, int *species_sc) {
    int64_t counter = 0;
    for (int i2 = 1; i2 <= indices[0]; ++i2)
        for (int j2 = 1; j2 <= indices[1]; ++j2)
            for (int k2 = 1; k2 <= indices[2]; ++k2)
                for (int i = 0; i < n_sites; ++i) {
                    for (int q = 0; q < 3; ++q)
                        positions_sc[3 * counter + q] =
                            positions[3 * i + q] + (double)(i2 - 1) * a[q] +
                            (double)(j2 - 1) * b[q] + (double)(k2 - 1) * c[q];
                    species_sc[counter] = species[i];
                    ++counter;
                }
}

// neighbors.f90:243-605 (build_neighbors_list) with rebuild_neighbors_list = .true.
int64_t orc_build_neighbors_list(int n_sites_supercell, const double *positions,
                                 int n_sites, double *a_box, double *b_box, double *c_box,
                                 double rcut_max, const int *indices,
                                 const int *species_supercell, const int *do_list,
                                 int64_t cap, int *n_neigh, int *neighbors_list,
                                 double *rjs, double *thetas, double *phis, double *xyz,
                                 int *neighbor_species) {
    bool is_box_square = box_is_orthorhombic(a_box, b_box, c_box);
    if (is_box_square) {
        a_box[1] = 0.0; a_box[2] = 0.0; b_box[0] = 0.0;
        b_box[2] = 0.0; c_box[0] = 0.0; c_box[1] = 0.0;
    }
    bool is_box_small = indices[0] > 1 || indices[1] > 1 || indices[2] > 1;
    std::vector<int> list;
    list.reserve((size_t)n_sites * 64);
    for (int i = 0; i < n_sites; ++i) n_neigh[i] = 0;
    const double tol = 1.e-10;
    double dist[3], d;
    int ish[3];
    if (is_box_square && !is_box_small) {
        const int mx = (int)(a_box[0] / rcut_max);
        const int my = (int)(b_box[1] / rcut_max);
        const int mz = (int)(c_box[2] / rcut_max);
        std::vector<int> head((size_t)mx * my * mz, 0), this_list(n_sites + 1, 0);
        const double center[3] = {a_box[0] / 2.0, b_box[1] / 2.0, c_box[2] / 2.0};
        auto cell_of = [&](int i, int *ci, int *cj, int *ck) {
            orc_get_distance(center, positions + 3 * i, a_box, b_box, c_box, dist, &d, ish);
            for (int q = 0; q < 3; ++q) dist[q] = dist[q] + center[q];
            *ci = (int)(dist[0] / (a_box[0] + tol) * (double)mx);
            *cj = (int)(dist[1] / (b_box[1] + tol) * (double)my);
            *ck = (int)(dist[2] / (c_box[2] + tol) * (double)mz);
        };
        auto fmod_int = [](int x, int m) { int r = x % m; return r < 0 ? r + m : r; };
        for (int i = 1; i <= n_sites; ++i) {
            int ci, cj, ck;
            cell_of(i - 1, &ci, &cj, &ck);
            int j = 1 + fmod_int(ci, mx) + fmod_int(cj, my) * mx + fmod_int(ck, mz) * my * mx;
            this_list[i] = head[j - 1];
            head[j - 1] = i;
        }
        for (int i = 1; i <= n_sites; ++i) {
            if (!do_list[i - 1]) continue;
            n_neigh[i - 1] += 1;
            list.push_back(i);
            int ci, cj, ck;
            cell_of(i - 1, &ci, &cj, &ck);
            const int i2 = 1 + ci, j2 = 1 + cj, k2 = 1 + ck;
            for (int k3 = k2 - 1; k3 <= k2 + 1; ++k3) {
                if (mz == 1 && k3 != 1) continue;
                if (mz == 2 && k2 == 1 && k3 == 0) continue;
                if (mz == 2 && k2 == 2 && k3 == 3) continue;
                for (int j3 = j2 - 1; j3 <= j2 + 1; ++j3) {
                    if (my == 1 && j3 != 1) continue;
                    if (my == 2 && j2 == 1 && j3 == 0) continue;
                    if (my == 2 && j2 == 2 && j3 == 3) continue;
                    for (int i3 = i2 - 1; i3 <= i2 + 1; ++i3) {
                        if (mx == 1 && i3 != 1) continue;
                        if (mx == 2 && i2 == 1 && i3 == 0) continue;
                        if (mx == 2 && i2 == 2 && i3 == 3) continue;
                        int j = 1 + fmod_int(i3 - 1, mx) + fmod_int(j3 - 1, my) * mx +
                                fmod_int(k3 - 1, mz) * mx * my;
                        int k = head[j - 1];
                        while (k != 0) {
                            if (k != i) {
                                orc_get_distance(positions + 3 * (i - 1), positions + 3 * (k - 1),
                                                 a_box, b_box, c_box, dist, &d, ish);
                                if (d < rcut_max) {
                                    n_neigh[i - 1] += 1;
                                    list.push_back(k);
                                }
                            }
                            k = this_list[k];
                        }
                    }
                }
            }
        }
    } else {
        for (int i = 1; i <= n_sites; ++i) {
            if (!do_list[i - 1]) continue;
            n_neigh[i - 1] += 1;
            list.push_back(i);
            for (int j = 1; j <= n_sites_supercell; ++j) {
                if (j == i) continue;
                orc_get_distance(positions + 3 * (i - 1), positions + 3 * (j - 1), a_box, b_box,
                                 c_box, dist, &d, ish);
                if (d < rcut_max) {
                    n_neigh[i - 1] += 1;
                    list.push_back(j);
                }
            }
        }
    }
    const int64_t n_pairs = (int64_t)list.size();
    if (n_pairs > cap) return -n_pairs;
    int64_t k2 = 0;
    for (int i = 1; i <= n_sites; ++i) {
        if (!do_list[i - 1]) { k2 += n_neigh[i - 1]; continue; }
        for (int k = 1; k <= n_neigh[i - 1]; ++k, ++k2) {
            const int j = list[k2];
            neighbors_list[k2] = j;
            if (k == 1) {
                rjs[k2] = 0.0;
                xyz[3 * k2] = xyz[3 * k2 + 1] = xyz[3 * k2 + 2] = 0.0;
                thetas[k2] = 0.0;
                phis[k2] = 0.0;
                neighbor_species[k2] = species_supercell[i - 1];
            } else {
                orc_get_distance(positions + 3 * (i - 1), positions + 3 * (j - 1), a_box, b_box,
                                 c_box, dist, &d, ish);
                rjs[k2] = d;
                xyz[3 * k2] = dist[0]; xyz[3 * k2 + 1] = dist[1]; xyz[3 * k2 + 2] = dist[2];
                if (std::fabs(dist[2]) >= d) {
                    thetas[k2] = dist[2] > 0.0 ? 0.0 : std::acos(-1.0);
                } else {
                    thetas[k2] = std::acos(dist[2] / d);
                }
                phis[k2] = std::atan2(dist[1], dist[0]);
                neighbor_species[k2] = species_supercell[j - 1];
            }
        }
    }
    return n_pairs;
}

// ---------------------------------------------------------------------------
// Descriptor (published method; see tg_oracle.h).
// ---------------------------------------------------------------------------

int orc_soap_n_tot(const orc_soap_hypers *h) {
    int n = 0;
    for (int s = 0; s < h->n_species; ++s) n += h->alpha_max[s];
    return n;
}

// read_files.f90:5233-5235; a compressed block has the dim its compression
// gives (read_files.f90:5171, 5213-5216)
int orc_soap_dim(const orc_soap_hypers *h) {
    if (h->compress_nonzero > 0) return h->compress_dim;
    const int n = orc_soap_n_tot(h);
    return n * (n + 1) / 2 * (h->l_max + 1);
}

// Orthonormal poly3 basis on [0, rc]: phi_n(x) = rc^{-1/2} sqrt(2n+7) t^3 P_n^{(0,6)}(2t-1),
// t = (rc - x)/rc, n = 0..alpha_max-1. This is Gram-Schmidt of (rc - x)^{alpha+2},
// alpha = 1..alpha_max. W[n][j] holds sqrt(2n+7) times the (integer) coefficient of
// t^j in P_n^{(0,6)}(2t-1), so phi_n = rc^{-1/2} sum_j W[n][j] t^{j+3}.
void orc_poly3_W(int alpha_max, double *W) {
    auto binom = [](int n, int k) -> int64_t {
        if (k < 0 || k > n) return 0;
        int64_t r = 1;
        for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
        return r;
    };
    for (int n = 0; n < alpha_max; ++n) {
        std::vector<int64_t> coef(alpha_max, 0);
        // P_n^{(0,6)}(x) = sum_s C(n, n-s) C(n+6, s) ((x-1)/2)^s ((x+1)/2)^(n-s),
        // with x = 2t-1: (t-1)^s t^(n-s).
        for (int s = 0; s <= n; ++s) {
            const int64_t base = binom(n, n - s) * binom(n + 6, s);
            for (int i = 0; i <= s; ++i) {
                const int64_t term = base * binom(s, i) * (((s - i) % 2) ? -1 : 1);
                coef[n - s + i] += term;
            }
        }
        const double nrm = std::sqrt((double)(2 * n + 7));
        for (int j = 0; j < alpha_max; ++j) W[n * alpha_max + j] = nrm * (double)coef[j];
    }
}

namespace {

struct SpeciesRadial {
    int amax;
    std::vector<double> W;
};

// m_k = int_0^1 t^k exp(-(t - tr)^2 / (2 s^2)) dt, k = 0..kmax, by the upward
// recurrence m_{k+1} = tr m_k + s^2 (k m_{k-1} - G1 + [k==0] G0), where
// G1 = exp(-(1-tr)^2/2s^2) (x = 0 end), G0 = exp(-tr^2/2s^2) (x = rc end).
void scaled_moments(double tr, double s, int kmax, double *m) {
    const double g1 = std::exp(-(1.0 - tr) * (1.0 - tr) / (2.0 * s * s));
    const double g0 = std::exp(-tr * tr / (2.0 * s * s));
    m[0] = s * std::sqrt(kPi / 2.0) *
           (std::erf((1.0 - tr) / (std::sqrt(2.0) * s)) + std::erf(tr / (std::sqrt(2.0) * s)));
    for (int k = 0; k < kmax; ++k) {
        double mk1 = tr * m[k] + s * s * ((k > 0 ? k * m[k - 1] : 0.0) - g1 + (k == 0 ? g0 : 0.0));
        m[k + 1] = mk1;
    }
}

// Smooth cut-off filter over the buffer zone: f = exp(-nf t^2 / (1 - t^2)),
// t = (r - r_soft)/(r_hard - r_soft). Returns f and df/dr.
void buffer_filter(double r, double rh, double rs, double nf, double *f, double *df) {
    if (r >= rh) { *f = 0.0; *df = 0.0; return; }
    if (!(rs < rh) || r <= rs) { *f = 1.0; *df = 0.0; return; }
    const double w = rh - rs;
    const double t = (r - rs) / w;
    const double den = 1.0 - t * t;
    const double e = std::exp(-nf * t * t / den);
    *f = e;
    *df = e * (-nf) * (2.0 * t / (den * den)) / w;
}

// Polynomial amplitude scaling: (1 - 3x^2 + 2x^3)^A, x = r/r_hard.
void amplitude(double r, double rh, double A, double *f, double *df) {
    if (r >= rh) { *f = 0.0; *df = 0.0; return; }
    if (A == 0.0) { *f = 1.0; *df = 0.0; return; }
    const double x = r / rh;
    const double P = 1.0 - 3.0 * x * x + 2.0 * x * x * x;
    const double dP = (-6.0 * x + 6.0 * x * x) / rh;
    *f = std::pow(P, A);
    *df = A * std::pow(P, A - 1.0) * dP;
}

// e^{-k} i_l(k) for l = 0..lmax+1 by the power series of the modified spherical
// Bessel function (all terms positive, so no cancellation at any k).
void scaled_msbessel(double k, int lmax1, double *out) {
    const double ek = std::exp(-k);
    double pref = 1.0;  // k^l / (2l+1)!!
    for (int l = 0; l <= lmax1; ++l) {
        if (l > 0) pref *= k / (double)(2 * l + 1);
        double term = 1.0, sum = 1.0;
        const double x = 0.5 * k * k;
        for (int j = 1; j < 400; ++j) {
            term *= x / ((double)j * (double)(2 * l + 2 * j + 1));
            sum += term;
            if (term < 1e-18 * sum) break;
        }
        out[l] = ek * pref * sum;
    }
}

}  // namespace

void orc_radial(const orc_soap_hypers *h, int s, double r, int self_pair, double *R,
                double *dR) {
    const int amax = h->alpha_max[s];
    const double rh = h->rcut_hard[s];
    std::vector<double> W(amax * amax);
    orc_poly3_W(amax, W.data());
    double w, dw;
    if (self_pair) {
        w = h->global_scaling[s] * h->central_weight[s];
        dw = 0.0;
        r = 0.0;
    } else {
        double fa, dfa, fc, dfc;
        amplitude(r, rh, h->amplitude_scaling[s], &fa, &dfa);
        buffer_filter(r, rh, h->rcut_soft[s], h->nf[s], &fc, &dfc);
        w = h->global_scaling[s] * fa * fc;
        dw = h->global_scaling[s] * (dfa * fc + fa * dfc);
    }
    for (int n = 0; n < amax; ++n) { R[n] = 0.0; dR[n] = 0.0; }
    if (w == 0.0 && dw == 0.0) return;
    const int re = h->radial_enhancement;
    const double sig = h->atom_sigma_r[s] * (1.0 + h->atom_sigma_r_scaling[s] * r);
    const double dsig = h->atom_sigma_r[s] * h->atom_sigma_r_scaling[s];
    const double tr = (rh - r) / rh, sc = sig / rh;
    const int kmax = amax + 2 + re + 2;
    std::vector<double> m(kmax + 1);
    scaled_moments(tr, sc, kmax, m.data());
    // e_k = int t^k (1-t)^re G dt and its r-derivative
    auto e_of = [&](const double *mm, int k) {
        if (re == 0) return mm[k];
        if (re == 1) return mm[k] - mm[k + 1];
        return mm[k] - 2.0 * mm[k + 1] + mm[k + 2];
    };
    // d m_k/dr = (-1/rh)(1/sc^2)(m_{k+1} - tr m_k) + (dsig/rh)(1/sc^3)(m_{k+2} - 2tr m_{k+1} + tr^2 m_k)
    std::vector<double> dm(kmax - 1);
    for (int k = 0; k + 2 <= kmax; ++k) {
        const double j1 = m[k + 1] - tr * m[k];
        const double j2 = m[k + 2] - 2.0 * tr * m[k + 1] + tr * tr * m[k];
        dm[k] = (-1.0 / rh) * j1 / (sc * sc) + (dsig / rh) * j2 / (sc * sc * sc);
    }
    const double pre = std::pow(rh, 0.5 + re);
    for (int n = 0; n < amax; ++n) {
        double v = 0.0, dv = 0.0;
        for (int j = 0; j < amax; ++j) {
            const double c = W[n * amax + j];
            if (c == 0.0) continue;
            v += c * e_of(m.data(), j + 3);
            dv += c * e_of(dm.data(), j + 3);
        }
        v *= pre;
        dv *= pre;
        R[n] = w * v;
        dR[n] = dw * v + w * dv;
    }
}

void orc_angular(const orc_soap_hypers *h, int s, double r, double *a, double *da) {
    const int L = h->l_max;
    const double st = h->atom_sigma_t[s] * (1.0 + h->atom_sigma_t_scaling[s] * r);
    const double dst = h->atom_sigma_t[s] * h->atom_sigma_t_scaling[s];
    const double k = r * r / (st * st);
    const double dk = 2.0 * r / (st * st) - 2.0 * r * r * dst / (st * st * st);
    std::vector<double> ei(L + 2);
    scaled_msbessel(k, L + 1, ei.data());
    for (int l = 0; l <= L; ++l) {
        a[l] = 4.0 * kPi * ei[l];
        double dil;  // e^{-k} i_l'(k)
        if (l == 0) dil = ei[1];
        else dil = ((double)l * ei[l - 1] + (double)(l + 1) * ei[l + 1]) / (double)(2 * l + 1);
        da[l] = 4.0 * kPi * (dil - ei[l]) * dk;
    }
}

// Real orthonormal spherical harmonics from Cartesian u (|u| = 1):
//   Y_l0 = N_l0 Q_l^0(z), Y_lm = sqrt2 N_lm Q_l^m(z) Re((x+iy)^m), Y_l-m = ... Im(...)
// with Q_l^m = d^m P_l / dz^m and N_lm = sqrt((2l+1)/(4pi) (l-m)!/(l+m)!).
void orc_real_ylm(int L, const double *u, double *Y, double *dY) {
    const double x = u[0], y = u[1], z = u[2];
    std::vector<double> C(L + 2), S(L + 2);
    C[0] = 1.0; S[0] = 0.0;
    for (int m = 0; m <= L; ++m) {
        C[m + 1] = x * C[m] - y * S[m];
        S[m + 1] = x * S[m] + y * C[m];
    }
    // Q[l][m] for m <= l <= L, plus Q[l][l+1] = 0
    std::vector<double> Q((L + 1) * (L + 2), 0.0);
    auto q = [&](int l, int m) -> double & { return Q[l * (L + 2) + m]; };
    for (int m = 0; m <= L; ++m) {
        double dfact = 1.0;
        for (int k = 1; k <= 2 * m - 1; k += 2) dfact *= (double)k;
        q(m, m) = dfact;
        if (m + 1 <= L) q(m + 1, m) = (double)(2 * m + 1) * z * q(m, m);
        for (int l = m + 2; l <= L; ++l)
            q(l, m) = ((double)(2 * l - 1) * z * q(l - 1, m) - (double)(l + m - 1) * q(l - 2, m)) /
                      (double)(l - m);
    }
    for (int l = 0; l <= L; ++l) {
        for (int m = 0; m <= l; ++m) {
            double ratio = 1.0;  // (l-m)!/(l+m)!
            for (int k = l - m + 1; k <= l + m; ++k) ratio /= (double)k;
            const double N = std::sqrt((2.0 * l + 1.0) / (4.0 * kPi) * ratio);
            const double Qlm = q(l, m);
            const double Qlm1 = (m + 1 <= l) ? q(l, m + 1) : 0.0;
            if (m == 0) {
                const int i = l * l + l;
                Y[i] = N * Qlm;
                if (dY) { dY[3 * i] = 0.0; dY[3 * i + 1] = 0.0; dY[3 * i + 2] = N * Qlm1; }
            } else {
                const double f = std::sqrt(2.0) * N;
                const int ip = l * l + l + m, im = l * l + l - m;
                Y[ip] = f * Qlm * C[m];
                Y[im] = f * Qlm * S[m];
                if (dY) {
                    dY[3 * ip] = f * Qlm * (double)m * C[m - 1];
                    dY[3 * ip + 1] = -f * Qlm * (double)m * S[m - 1];
                    dY[3 * ip + 2] = f * Qlm1 * C[m];
                    dY[3 * im] = f * Qlm * (double)m * S[m - 1];
                    dY[3 * im + 1] = f * Qlm * (double)m * C[m - 1];
                    dY[3 * im + 2] = f * Qlm1 * S[m];
                }
            }
        }
    }
}

void orc_get_soap(const orc_soap_hypers *h, int n_sites, const int *n_neigh, int n_pairs,
                  const int *mask, const double *rjs, const double *xyz, double *soap,
                  double *soap_cart_der, double *sqrt_dot_p) {
    const int ns = h->n_species, L = h->l_max, L2 = (L + 1) * (L + 1);
    const int n_tot = orc_soap_n_tot(h), dimf = n_tot * (n_tot + 1) / 2 * (L + 1);
    // compression: the power spectrum p (dimf entries) is mapped to v = P p
    // (dim entries) and v is normalised; uncompressed, v = p
    const bool comp = h->compress_nonzero > 0;
    const int dim = comp ? h->compress_dim : dimf;
    std::vector<int> ch0(ns + 1, 0);
    for (int s = 0; s < ns; ++s) ch0[s + 1] = ch0[s] + h->alpha_max[s];
    std::vector<int64_t> start(n_sites + 1, 0);
    for (int i = 0; i < n_sites; ++i) start[i + 1] = start[i] + n_neigh[i];
    // power-spectrum index table: d -> (n, n', l)
    std::vector<int> pn(dimf), pn2(dimf), pl(dimf);
    {
        int d = 0;
        for (int n = 0; n < n_tot; ++n)
            for (int n2 = n; n2 < n_tot; ++n2)
                for (int l = 0; l <= L; ++l) { pn[d] = n; pn2[d] = n2; pl[d] = l; ++d; }
    }
    const double sqrt2 = std::sqrt(2.0);
#pragma omp parallel
    {
        std::vector<double> c((size_t)n_tot * L2), Y(L2), dY(3 * L2), R(16 * 4), dR(16 * 4),
            a(L + 1), da(L + 1), p(dimf), dc, dp(3 * (size_t)dimf), v(dim), dv(3 * (size_t)dim);
        // v = P p over the nonzero entries (1-based i, j), in file order
        auto compress = [&](const double *x, double *y, int stride) {
            std::fill(y, y + (size_t)stride * dim, 0.0);
            for (int k = 0; k < h->compress_nonzero; ++k) {
                const int i = h->compress_i[k] - 1, j = h->compress_j[k] - 1;
                for (int q = 0; q < stride; ++q)
                    y[(size_t)stride * i + q] += h->compress_el[k] * x[(size_t)stride * j + q];
            }
        };
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < n_sites; ++i) {
            const int64_t k0 = start[i], nn = n_neigh[i];
            std::fill(c.begin(), c.end(), 0.0);
            if (soap_cart_der) dc.assign((size_t)nn * n_tot * L2 * 3, 0.0);
            for (int64_t kk = 0; kk < nn; ++kk) {
                const int64_t k = k0 + kk;
                const bool self = (kk == 0);
                const double r = rjs[k];
                double u[3] = {0, 0, 0};
                if (!self) {
                    for (int q = 0; q < 3; ++q) u[q] = xyz[3 * k + q] / r;
                    orc_real_ylm(L, u, Y.data(), dY.data());
                }
                for (int s = 0; s < ns; ++s) {
                    if (!mask[k + (int64_t)n_pairs * s]) continue;
                    const int amax = h->alpha_max[s];
                    if (self) {
                        orc_radial(h, s, 0.0, 1, R.data(), dR.data());
                        // a_0(0) = 4 pi, a_l(0) = 0 for l > 0; Y_00 = 1/sqrt(4 pi)
                        for (int n = 0; n < amax; ++n)
                            c[(size_t)(ch0[s] + n) * L2] += R[n] * 4.0 * kPi / std::sqrt(4.0 * kPi);
                        continue;
                    }
                    if (!(r < h->rcut_hard[s])) continue;
                    orc_radial(h, s, r, 0, R.data(), dR.data());
                    orc_angular(h, s, r, a.data(), da.data());
                    for (int n = 0; n < amax; ++n) {
                        for (int l = 0; l <= L; ++l) {
                            const double rho = R[n] * a[l], drho = dR[n] * a[l] + R[n] * da[l];
                            for (int m = -l; m <= l; ++m) {
                                const int lm = l * l + l + m;
                                c[(size_t)(ch0[s] + n) * L2 + lm] += rho * Y[lm];
                                if (soap_cart_der) {
                                    const double *g = &dY[3 * lm];
                                    const double ug = u[0] * g[0] + u[1] * g[1] + u[2] * g[2];
                                    double *t = &dc[(((size_t)kk * n_tot + ch0[s] + n) * L2 + lm) * 3];
                                    for (int q = 0; q < 3; ++q)
                                        t[q] += drho * u[q] * Y[lm] + rho * (g[q] - ug * u[q]) / r;
                                }
                            }
                        }
                    }
                }
            }
            // power spectrum, compression and normalisation
            for (int d = 0; d < dimf; ++d) {
                const int n = pn[d], n2 = pn2[d], l = pl[d];
                double pv = 0.0;
                for (int m = -l; m <= l; ++m) {
                    const int lm = l * l + l + m;
                    pv += c[(size_t)n * L2 + lm] * c[(size_t)n2 * L2 + lm];
                }
                if (n != n2) pv *= sqrt2;
                p[d] = pv;
            }
            if (comp) compress(p.data(), v.data(), 1);
            else std::copy(p.begin(), p.end(), v.begin());
            double nrm2 = 0.0;
            for (int d = 0; d < dim; ++d) nrm2 += v[d] * v[d];
            const double nrm = std::sqrt(nrm2);
            if (sqrt_dot_p) sqrt_dot_p[i] = nrm;
            for (int d = 0; d < dim; ++d) soap[(size_t)i * dim + d] = nrm > 0.0 ? v[d] / nrm : 0.0;
            if (!soap_cart_der) continue;
            double *self_der = soap_cart_der + (size_t)k0 * 3 * dim;
            std::fill(self_der, self_der + 3 * (size_t)dim, 0.0);
            for (int64_t kk = 1; kk < nn; ++kk) {
                double *out = soap_cart_der + (size_t)(k0 + kk) * 3 * dim;
                if (nrm == 0.0) { std::fill(out, out + 3 * (size_t)dim, 0.0); continue; }
                const double *dck = &dc[(size_t)kk * n_tot * L2 * 3];
                for (int d = 0; d < dimf; ++d) {
                    const int n = pn[d], n2 = pn2[d], l = pl[d];
                    double g[3] = {0, 0, 0};
                    for (int m = -l; m <= l; ++m) {
                        const int lm = l * l + l + m;
                        const double *g1 = &dck[((size_t)n * L2 + lm) * 3];
                        const double *g2 = &dck[((size_t)n2 * L2 + lm) * 3];
                        const double c1 = c[(size_t)n * L2 + lm], c2 = c[(size_t)n2 * L2 + lm];
                        for (int q = 0; q < 3; ++q) g[q] += g1[q] * c2 + c1 * g2[q];
                    }
                    const double mu = (n != n2) ? sqrt2 : 1.0;
                    for (int q = 0; q < 3; ++q) dp[3 * (size_t)d + q] = mu * g[q];
                }
                if (comp) compress(dp.data(), dv.data(), 3);
                else std::copy(dp.begin(), dp.end(), dv.begin());
                double qdp[3] = {0, 0, 0};
                for (int d = 0; d < dim; ++d)
                    for (int q = 0; q < 3; ++q) qdp[q] += (v[d] / nrm) * dv[3 * (size_t)d + q];
                for (int d = 0; d < dim; ++d) {
                    const double qd = v[d] / nrm;
                    for (int q = 0; q < 3; ++q) {
                        const double val = (dv[3 * (size_t)d + q] - qd * qdp[q]) / nrm;
                        out[3 * (size_t)d + q] = val;
                        self_der[3 * (size_t)d + q] -= val;
                    }
                }
            }
        }
    }
}

// gap.f90:66-259 (get_soap_energy_and_forces). soap(n_soap, n_sites),
// soap_der(3, n_soap, P), Qs(n_soap, n_sparse): all column-major.
void orc_soap_energy_and_forces(int n_soap, int n_sites, const double *soap,
                                const double *soap_der, int n_sparse, const double *Qs,
                                const double *alphas, double delta, double zeta0, double e0,
                                const int *n_neigh, const int *neighbors_list,
                                const double *xyz, int n_sites0, int do_forces,
                                double *energies, double *forces, double *virial) {
    bool is_zeta_int = false;
    int zeta_int = 0;
    double zeta = zeta0;
    if (std::fabs(zeta0 - (double)(int)zeta0) < 1.e-5) {
        is_zeta_int = true;
        zeta_int = (int)zeta0;
        zeta = (double)zeta_int;
    }
    auto ipow = [](double x, int e) {
        double r = 1.0;
        for (int k = 0; k < e; ++k) r *= x;
        return r;
    };
    // kernels(n_sites, n_sparse) = soap^T Qs  (dgemm 't','n'), kept row-major per site here
    std::vector<double> K((size_t)n_sites * n_sparse);
    gemm_nt_blocked(n_sites, n_sparse, n_soap, soap, Qs, K.data());
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n_sites; ++i) {
        double e = 0.0;
        for (int s = 0; s < n_sparse; ++s) {
            const double k = K[(size_t)i * n_sparse + s];
            const double kz = is_zeta_int ? ipow(k, zeta_int) : std::pow(k, zeta);
            e += kz * alphas[s];
        }
        energies[i] = delta * delta * e + e0;
    }
    if (!do_forces) return;
    // kernels_der = K^(zeta-1) (alphas folded in); Qss = -zeta delta^2 kernels_der Qs^T
    std::vector<double> Qss((size_t)n_sites * n_soap, 0.0);
    const double pref = -zeta * delta * delta;
    // kernels_der (alphas folded in, times -zeta delta^2), then Qss = kd Qs (dgemm 'n','t')
    std::vector<double> KD((size_t)n_sites * n_sparse);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n_sites; ++i)
        for (int s = 0; s < n_sparse; ++s) {
            const double k = K[(size_t)i * n_sparse + s];
            KD[(size_t)i * n_sparse + s] =
                pref * (is_zeta_int ? ipow(k, zeta_int - 1) : std::pow(k, zeta - 1.0)) * alphas[s];
        }
    gemm_nn_blocked(n_sites, n_soap, n_sparse, KD.data(), Qs, Qss.data());
    // pair loop (gap.f90:206-224); each pair's force computed in parallel, then
    // accumulated in the reference's serial order.
    std::vector<int64_t> start(n_sites + 1, 0);
    for (int i = 0; i < n_sites; ++i) start[i + 1] = start[i] + n_neigh[i];
    const int64_t P = start[n_sites];
    std::vector<double> pf((size_t)P * 3);
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < n_sites; ++i) {
        const double *qss = &Qss[(size_t)i * n_soap];
        for (int64_t l = start[i]; l < start[i + 1]; ++l) {
            const double *sd = soap_der + (size_t)l * 3 * n_soap;
            for (int k = 0; k < 3; ++k) {
                double acc = 0.0;
                for (int d = 0; d < n_soap; ++d) acc += qss[d] * sd[3 * (size_t)d + k];
                pf[3 * l + k] = acc;
            }
        }
    }
    for (int q = 0; q < 9; ++q) virial[q] = 0.0;
    for (int64_t q = 0; q < 3 * (int64_t)n_sites0; ++q) forces[q] = 0.0;
    for (int64_t l = 0; l < P; ++l) {
        const int j2 = (neighbors_list[l] - 1) % n_sites0;
        const double *f = &pf[3 * l];
        for (int k = 0; k < 3; ++k) forces[3 * (size_t)j2 + k] += f[k];
        const double *x = xyz + 3 * l;
        for (int k1 = 0; k1 < 3; ++k1)
            for (int k2 = 0; k2 < 3; ++k2)
                virial[k1 + 3 * k2] += 0.5 * (f[k1] * x[k2] + f[k2] * x[k1]);
    }
}

// gap_interface.f90:41-480 (get_gap_soap) for a prediction with forces.
int orc_get_gap_soap(const orc_soap_hypers *h, int n_total_sites, int n_sites0,
                     const int *n_neigh0, const int *neighbors_list0, const double *rjs0,
                     const double *xyz0, const int *species_batch, const int *species_all,
                     int n_sparse, const double *Qs, const double *alphas, double delta,
                     double zeta, int do_forces, double *energies0, double *forces0,
                     double *virial) {
    const int ns = h->n_species;
    auto first_species = [&](int z) {
        for (int s = 0; s < ns; ++s)
            if (h->species_z[s] == z) return s + 1;
        return 0;
    };
    auto multiplicity = [&](int z) {
        int m = 0;
        for (int s = 0; s < ns; ++s) m += (h->species_z[s] == z);
        return m;
    };
    double rcut_max = 0.0;
    for (int s = 0; s < ns; ++s) rcut_max = std::max(rcut_max, h->rcut_hard[s]);
    const int cs = h->central_species;
    auto is_central = [&](int i) { return cs == 0 || first_species(species_batch[i]) == cs; };
    auto fold = [&](int j) { return (j - 1) % n_total_sites + 1; };
    int n_sites = 0;
    int64_t n_atom_pairs = 0, k = 0;
    std::vector<char> seen(n_total_sites + 1, 0);
    for (int i = 0; i < n_sites0; ++i) {
        if (is_central(i)) {
            ++n_sites;
            for (int j = 0; j < n_neigh0[i]; ++j, ++k) {
                const int j2 = fold(neighbors_list0[k]);
                if (rjs0[k] < rcut_max && multiplicity(species_all[j2 - 1]) > 0) {
                    ++n_atom_pairs;
                    seen[j2] = 1;
                }
            }
        } else {
            k += n_neigh0[i];
        }
    }
    int n_all_sites = 0;
    for (int i = 1; i <= n_total_sites; ++i) n_all_sites += seen[i];
    std::vector<int> n_neigh(n_sites), nl(n_atom_pairs), in_to_out_site(n_all_sites + 1, 0),
        out_to_in_site(n_total_sites + 1, 0), mask((size_t)n_atom_pairs * ns);
    std::vector<double> rjs(n_atom_pairs), xyz(3 * (size_t)n_atom_pairs);
    k = 0;
    int i2 = 0;
    for (int i = 0; i < n_sites0; ++i) {
        const int j = fold(neighbors_list0[k]);
        if (is_central(i)) {
            ++i2;
            in_to_out_site[i2] = j;
            out_to_in_site[j] = i2;
        }
        k += n_neigh0[i];
    }
    k = 0;
    i2 = 0;
    int i4 = 0;
    int64_t k2 = 0;
    for (int i = 0; i < n_sites0; ++i) {
        if (!is_central(i)) { k += n_neigh0[i]; continue; }
        ++i2;
        int j2 = 0;
        for (int j = 1; j <= n_neigh0[i]; ++j, ++k) {
            const int j3 = fold(neighbors_list0[k]);
            if (!(rjs0[k] < rcut_max && multiplicity(species_all[j3 - 1]) > 0)) continue;
            ++j2;
            rjs[k2] = rjs0[k];
            for (int q = 0; q < 3; ++q) xyz[3 * k2 + q] = xyz0[3 * k + q];
            for (int s = 0; s < ns; ++s)
                mask[k2 + (size_t)n_atom_pairs * s] = (h->species_z[s] == species_all[j3 - 1]);
            if (j > 1 && out_to_in_site[j3] == 0) {
                ++i4;
                in_to_out_site[n_sites + i4] = j3;
                out_to_in_site[j3] = n_sites + i4;
                nl[k2] = out_to_in_site[j3];
            } else if (j > 1) {
                nl[k2] = out_to_in_site[j3];
            } else {
                nl[k2] = i2;
            }
            ++k2;
        }
        n_neigh[i2 - 1] = j2;
    }
    const int dim = orc_soap_dim(h);
    std::vector<double> soap((size_t)dim * n_sites);
    std::vector<double> der;
    if (do_forces) der.resize((size_t)3 * dim * n_atom_pairs);
    if (n_sites > 0)
        orc_get_soap(h, n_sites, n_neigh.data(), (int)n_atom_pairs, mask.data(), rjs.data(),
                     xyz.data(), soap.data(), do_forces ? der.data() : nullptr, nullptr);
    std::vector<double> energies(n_sites, 0.0), forces(3 * (size_t)n_all_sites, 0.0);
    for (int q = 0; q < 9; ++q) virial[q] = 0.0;
    if (n_sites > 0)
        orc_soap_energy_and_forces(dim, n_sites, soap.data(), do_forces ? der.data() : nullptr,
                                   n_sparse, Qs, alphas, delta, zeta, 0.0, n_neigh.data(),
                                   nl.data(), xyz.data(), n_all_sites, do_forces,
                                   energies.data(), forces.data(), virial);
    for (int i = 1; i <= n_sites; ++i) energies0[in_to_out_site[i] - 1] = energies[i - 1];
    if (do_forces)
        for (int i = 1; i <= n_all_sites; ++i)
            for (int q = 0; q < 3; ++q)
                forces0[3 * (size_t)(in_to_out_site[i] - 1) + q] = forces[3 * (size_t)(i - 1) + q];
    return n_sites;
}

// neighbors.f90:609-778 (soap_batch_memory_model + get_number_of_atom_pairs)
int orc_atom_pair_batches(int n_sites, const int *n_neigh, const double *rjs, double rcut,
                          int l_max, int n_max, int n_soap, int n_species, double max_gbytes,
                          int *i_beg, int *i_end, int *j_beg, int *j_end) {
    int64_t k = 0, n_in = 0;
    for (int i = 0; i < n_sites; ++i)
        for (int j = 0; j < n_neigh[i]; ++j, ++k)
            if (rjs[k] < rcut) ++n_in;
    const int64_t n_atom_pairs = k;
    const int k_max = 1 + l_max * (l_max + 1) / 2 + l_max;
    const double bpp = 48.0 * k_max * n_max + 64.0 * k_max + 48.0 * n_soap + 16.0 * n_max +
                       4.0 * n_species + 56.0;
    const double bps = 16.0 * k_max * n_max + 8.0 * n_soap + 16.0;
    const double est = 1.10 * ((double)n_in * bpp + (double)n_sites * bps) / (1024.0 * 1024.0 * 1024.0);
    const double ratio = est / max_gbytes;
    int n_chunks = (int)std::ceil(ratio);
    if (n_chunks > n_sites) n_chunks = n_sites;
    if (n_chunks == 0) return 0;
    const double ppc = (double)n_in / (double)n_chunks;
    i_beg[0] = 1; j_beg[0] = 1;
    i_end[n_chunks - 1] = n_sites;
    j_end[n_chunks - 1] = (int)n_atom_pairs;
    if (n_chunks == 1) return 1;
    k = 0;
    int64_t k2 = 0;
    int ic = 1;
    for (int i = 1; i <= n_sites; ++i) {
        for (int j = 0; j < n_neigh[i - 1]; ++j) {
            ++k;
            if (rjs[k - 1] < rcut) ++k2;
        }
        // Fortran: int(float(i_chunk)*pairs_per_chunk); float() of a small
        // integer is exact, the product is taken in double.
        if (k2 >= (int64_t)((double)(float)ic * ppc)) {
            i_end[ic - 1] = i;
            j_end[ic - 1] = (int)k;
            ++ic;
            i_beg[ic - 1] = i + 1;
            j_beg[ic - 1] = (int)k + 1;
            if (ic == n_chunks) break;
        }
    }
    return n_chunks;
}

// md.f90:226-283 (velocity_verlet) with no fixed atoms.
void orc_velocity_verlet(int n, double *positions, double *positions_prev,
                         double *velocities, const double *forces, double *forces_prev,
                         const double *masses, double dt, double *dt_prev, int first_step) {
    if (!first_step) {
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < 3; ++j)
                velocities[3 * i + j] = velocities[3 * i + j] +
                                        0.5 * (forces[3 * i + j] + forces_prev[3 * i + j]) /
                                            masses[i] * (*dt_prev);
    }
    std::memcpy(positions_prev, positions, sizeof(double) * 3 * n);
    std::memcpy(forces_prev, forces, sizeof(double) * 3 * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < 3; ++j)
            positions[3 * i + j] = positions[3 * i + j] + velocities[3 * i + j] * dt +
                                   0.5 * forces[3 * i + j] / masses[i] * (dt * dt);
    *dt_prev = dt;
}

// md.f90:316-344
void orc_remove_cm_vel(int n, double *vel, const double *m) {
    double cm[3] = {0, 0, 0}, tm = 0.0;
    for (int i = 0; i < n; ++i) {
        for (int q = 0; q < 3; ++q) cm[q] = cm[q] + m[i] * vel[3 * i + q];
        tm = tm + m[i];
    }
    for (int q = 0; q < 3; ++q) cm[q] = cm[q] / tm;
    for (int i = 0; i < n; ++i)
        for (int q = 0; q < 3; ++q) vel[3 * i + q] = vel[3 * i + q] - cm[q];
}

// md.f90:348-380
void orc_wrap_pbc(int n, double *positions, const double *a, const double *b, const double *c) {
    const double zero[3] = {0, 0, 0};
    double dist[3], d;
    int ish[3];
    for (int i = 0; i < n; ++i) {
        orc_get_distance(zero, positions + 3 * i, a, b, c, dist, &d, ish);
        for (int q = 0; q < 3; ++q)
            positions[3 * i + q] = positions[3 * i + q] - (double)ish[0] * a[q] -
                                   (double)ish[1] * b[q] - (double)ish[2] * c[q];
    }
}

// turbogap.f90:896-997 + 1253-1378 + 1941/2009: one structure, every block,
// memory-budget batches, summed into totals; e0 by species.
int orc_evaluate_range(int n_sites, const double *positions, const int *species,
                       const double *a, const double *b, const double *c, int n_blocks,
                       const orc_gap_block *blocks, const double *e0_by_species,
                       int n_species_total, double neighbors_buffer, double max_gbytes,
                       int site_beg, int site_end, double *energies, double *forces,
                       double *virial, int64_t *n_pairs_out);

int orc_evaluate(int n_sites, const double *positions, const int *species, const double *a,
                 const double *b, const double *c, int n_blocks, const orc_gap_block *blocks,
                 const double *e0_by_species, int n_species_total, double neighbors_buffer,
                 double max_gbytes, double *energies, double *forces, double *virial,
                 int64_t *n_pairs_out) {
    return orc_evaluate_range(n_sites, positions, species, a, b, c, n_blocks, blocks,
                              e0_by_species, n_species_total, neighbors_buffer, max_gbytes, 0,
                              n_sites, energies, forces, virial, n_pairs_out);
}

// The share of one MPI rank (turbogap.f90:930-942): neighbour lists and SOAP work
// for sites site_beg..site_end-1 only (do_list), forces from those sites' energies.
int orc_evaluate_range(int n_sites, const double *positions, const int *species,
                       const double *a, const double *b, const double *c, int n_blocks,
                       const orc_gap_block *blocks, const double *e0_by_species,
                       int n_species_total, double neighbors_buffer, double max_gbytes,
                       int site_beg, int site_end, double *energies, double *forces,
                       double *virial, int64_t *n_pairs_out) {
    return orc_evaluate_full(n_sites, positions, species, a, b, c, n_blocks, blocks, 0, nullptr,
                             e0_by_species, n_species_total, neighbors_buffer, max_gbytes,
                             site_beg, site_end, energies, forces, virial, n_pairs_out);
}

// read_files.f90:5454-5505
void orc_core_pot_spline(int n, const double *x, const double *V, double *yp1, double *ypn,
                         double *y2) {
    std::vector<double> u(n, 0.0);
    if (*yp1 > 0.99e30) {
        y2[0] = 0.0;
        u[0] = 0.0;
    } else {
        y2[0] = -0.5;
        u[0] = (3.0 / (x[1] - x[0])) * ((V[1] - V[0]) / (x[1] - x[0]) - *yp1);
    }
    for (int i = 1; i < n - 1; ++i) {
        const double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
        const double p = sig * y2[i - 1] + 2.0;
        y2[i] = (sig - 1.0) / p;
        u[i] = (V[i + 1] - V[i]) / (x[i + 1] - x[i]) - (V[i] - V[i - 1]) / (x[i] - x[i - 1]);
        u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p;
    }
    double qn, un;
    if (*ypn > 0.99e30) {
        qn = 0.0;
        un = 0.0;
    } else {
        qn = 0.5;
        un = (3.0 / (x[n - 1] - x[n - 2])) * (*ypn - (V[n - 1] - V[n - 2]) / (x[n - 1] - x[n - 2]));
    }
    y2[n - 1] = (un - qn * u[n - 2]) / (qn * y2[n - 2] + 1.0);
    for (int i = n - 2; i >= 0; --i) y2[i] = y2[i] * y2[i + 1] + u[i];
    // natural ends: the slope of the spline at the end node (splines.f90:123-183;
    // at x(n) the last interval is used)
    auto slope = [&](int j, double r) {
        const double h = x[j + 1] - x[j], h6 = h / 6.0;
        const double A = (x[j + 1] - r) / h, B = 1.0 - A;
        return -1.0 / h * V[j] + 1.0 / h * V[j + 1] + (1.0 - 3.0 * A * A) * h6 * y2[j] +
               (3.0 * B * B - 1.0) * h6 * y2[j + 1];
    };
    if (*yp1 > 0.99e30) *yp1 = slope(0, x[0]);
    if (*ypn > 0.99e30) *ypn = slope(n - 2, x[n - 1]);
}

namespace {

// splines.f90:35-121 (value) and 123-183 (derivative), for r < rcut
int spline_interval(const orc_family *f, double r) {
    int j = 0;
    while (j < f->n - 2 && !(r < f->x[j + 1])) ++j;
    return j;
}
double spline_value(const orc_family *f, double r) {
    const int n = f->n;
    if (r < f->x[0]) return f->V[0] + (r - f->x[0]) * f->yp1;
    if (r > f->x[n - 1]) return f->V[n - 1] + (r - f->x[n - 1]) * f->ypn;
    const int j = spline_interval(f, r);
    const double h = f->x[j + 1] - f->x[j], h26 = h * h / 6.0;
    const double A = (f->x[j + 1] - r) / h, B = 1.0 - A;
    const double C = (A * A * A - A) * h26, D = (B * B * B - B) * h26;
    return A * f->V[j] + B * f->V[j + 1] + C * f->y2[j] + D * f->y2[j + 1];
}
double spline_slope(const orc_family *f, double r) {
    const int n = f->n;
    if (r < f->x[0]) return f->yp1;
    if (r > f->x[n - 1]) return f->ypn;
    const int j = spline_interval(f, r);
    const double h = f->x[j + 1] - f->x[j], h6 = h / 6.0;
    const double A = (f->x[j + 1] - r) / h, B = 1.0 - A;
    return -1.0 / h * f->V[j] + 1.0 / h * f->V[j + 1] + (1.0 - 3.0 * A * A) * h6 * f->y2[j] +
           (3.0 * B * B - 1.0) * h6 * f->y2[j + 1];
}

// gap.f90:1049-1112, d = 3, q = 1 (j = 3)
double cov_pp(double r) {
    if (r >= 1.0) return 0.0;
    if (r <= 0.0) return 1.0;
    const double om = 1.0 - r;
    return om * om * om * om * (4.0 * r + 1.0);
}
double cov_pp_der(double r) {
    if (r >= 1.0 || r <= 0.0) return 0.0;
    const double om = 1.0 - r;
    return (-4.0 * om * om * om * (4.0 * r + 1.0) + om * om * om * om * 4.0) / r;
}

}  // namespace

// gap.f90:400-563 (2b), 565-721 (core_pot), 724-1042 (3b)
void orc_family_energy_forces(const orc_family *f, int n_sites, const int *n_neigh,
                              const int *neighbors_list, const double *rjs, const double *xyz,
                              const int *species, const int *neighbor_species, int n_sites0,
                              double *energies, double *forces, double *virial) {
    const double pi = std::acos(-1.0);
    const double buffer = 0.5;   // gap_backend_cpu.f90:152,252 pass 0.5d0
    for (int i = 0; i < n_sites; ++i) energies[i] = 0.0;
    for (int i = 0; i < 3 * n_sites0; ++i) forces[i] = 0.0;
    for (int q = 0; q < 9; ++q) virial[q] = 0.0;
    auto vir_add = [&](const double *fv, const double *x, double w) {
        for (int k1 = 0; k1 < 3; ++k1)
            for (int k2 = 0; k2 < 3; ++k2)
                virial[k1 + 3 * k2] += w * (fv[k1] * x[k2] + fv[k2] * x[k1]);
    };
    if (f->kind == 1 || f->kind == 3) {
        const int sp1 = f->sp[0], sp2 = f->sp[1];
        const double rcut = f->kind == 1 ? f->rcut : f->x[f->n - 1];
        int64_t k = 0;
        for (int i = 0; i < n_sites; ++i) {
            if (species[i] != sp1 && species[i] != sp2) {
                k += n_neigh[i];
                continue;
            }
            ++k;
            for (int j = 1; j < n_neigh[i]; ++j, ++k) {
                const int ns = neighbor_species[k];
                if (!((species[i] == sp1 && ns == sp2) || (species[i] == sp2 && ns == sp1))) continue;
                const double r = rjs[k];
                if (!(r < rcut)) continue;
                const double *x = xyz + 3 * k;
                double fv[3];
                if (f->kind == 1) {
                    double fc = 1.0, dfc = 0.0;
                    if (!(r < rcut - buffer)) {
                        fc = (std::cos(pi * (r - rcut + buffer) / buffer) + 1.0) / 2.0;
                        dfc = pi / 2.0 / buffer * std::sin(pi * (r - rcut + buffer) / buffer);
                    }
                    const double d2 = f->delta * f->delta, s2 = f->sigma[0] * f->sigma[0];
                    for (int s = 0; s < f->n; ++s) {
                        const double ex = std::exp(-0.5 * (r - f->Qs[s]) * (r - f->Qs[s]) / s2);
                        energies[i] += d2 * f->alphas[s] * f->cutoff[s] * fc * ex;
                        const double g = -2.0 * d2 * f->alphas[s] * f->cutoff[s] * ex *
                                         ((r - f->Qs[s]) / s2 * fc + dfc);
                        for (int q = 0; q < 3; ++q) fv[q] = g * x[q] / r;
                        for (int q = 0; q < 3; ++q) forces[3 * i + q] += fv[q];
                        vir_add(fv, x, -0.25);
                    }
                } else {
                    energies[i] += 0.5 * spline_value(f, r);
                    const double dv = spline_slope(f, r);
                    for (int q = 0; q < 3; ++q) fv[q] = dv * x[q] / r;
                    for (int q = 0; q < 3; ++q) forces[3 * i + q] += fv[q];
                    vir_add(fv, x, -0.25);
                }
            }
        }
        return;
    }
    // angle_3b
    const int sp0 = f->sp[0], sp1 = f->sp[1], sp2 = f->sp[2];
    const double rcut = f->rcut;
    const int ns = f->n;
    const double *Q1 = f->Qs, *Q2 = f->Qs + ns, *Q3 = f->Qs + 2 * ns;
    const double s1 = f->sigma[0] * f->sigma[0], s2 = f->sigma[1] * f->sigma[1],
                 s3 = f->sigma[2] * f->sigma[2];
    std::vector<double> pref(ns), rr(ns), kern(ns), kder(ns), dq1(ns), dq2(ns), dq3(ns);
    for (int s = 0; s < ns; ++s) pref[s] = 2.0 * f->delta * f->delta * f->alphas[s] * f->cutoff[s];
    int64_t k = 0;
    for (int i = 0; i < n_sites; ++i) {
        if (species[i] != sp0) {
            k += n_neigh[i];
            continue;
        }
        const int64_t kself = k;
        ++k;
        const int i3 = (neighbors_list[kself] - 1) % n_sites0;
        for (int j = 1; j < n_neigh[i]; ++j) {
            const int64_t kj = kself + j;
            const double r12 = rjs[kj];
            const int nsj = neighbor_species[kj];
            if ((nsj != sp1 && nsj != sp2) || r12 > rcut) continue;
            const int j3 = (neighbors_list[kj] - 1) % n_sites0;
            const double *x12 = xyz + 3 * kj;
            double u12[3] = {x12[0] / r12, x12[1] / r12, x12[2] / r12};
            for (int j2 = j + 1; j2 < n_neigh[i]; ++j2) {
                const int64_t k2 = kself + j2;
                const double r13 = rjs[k2];
                const int nsk = neighbor_species[k2];
                if (!(((nsj == sp1 && nsk == sp2) || (nsj == sp2 && nsk == sp1)) && r13 < rcut)) continue;
                const int k3 = (neighbors_list[k2] - 1) % n_sites0;
                const double *x13 = xyz + 3 * k2;
                double u13[3] = {x13[0] / r13, x13[1] / r13, x13[2] / r13};
                double x23[3] = {x13[0] - x12[0], x13[1] - x12[1], x13[2] - x12[2]};
                const double r23 = std::sqrt(x23[0] * x23[0] + x23[1] * x23[1] + x23[2] * x23[2]);
                double u23[3] = {x23[0] / r23, x23[1] / r23, x23[2] / r23};
                if (!(r12 < rcut && r13 < rcut)) continue;
                double fc12 = 1.0, fc13 = 1.0, df12[3] = {0, 0, 0}, df13[3] = {0, 0, 0};
                if (!(r12 < rcut - buffer)) {
                    fc12 = (std::cos(pi * (r12 - rcut + buffer) / buffer) + 1.0) / 2.0;
                    const double t = std::sin(pi * (r12 - rcut + buffer) / buffer) / 2.0 * pi / buffer;
                    for (int q = 0; q < 3; ++q) df12[q] = t * u12[q];
                }
                if (!(r13 < rcut - buffer)) {
                    fc13 = (std::cos(pi * (r13 - rcut + buffer) / buffer) + 1.0) / 2.0;
                    const double t = std::sin(pi * (r13 - rcut + buffer) / buffer) / 2.0 * pi / buffer;
                    for (int q = 0; q < 3; ++q) df13[q] = t * u13[q];
                }
                const double fc = fc12 * fc13;
                double dfc[3];
                for (int q = 0; q < 3; ++q) dfc[q] = fc12 * df13[q] + fc13 * df12[q];
                const double qv1 = r12 + r13, qv2 = (r12 - r13) * (r12 - r13), qv3 = r23;
                for (int s = 0; s < ns; ++s) {
                    double t = (qv1 - Q1[s]) * (qv1 - Q1[s]) / s1;
                    t += (qv2 - Q2[s]) * (qv2 - Q2[s]) / s2;
                    t += (qv3 - Q3[s]) * (qv3 - Q3[s]) / s3;
                    rr[s] = std::sqrt(t);
                    dq1[s] = (qv1 - Q1[s]) / s1;
                    dq2[s] = (qv2 - Q2[s]) / s2;
                    dq3[s] = (qv3 - Q3[s]) / s3;
                }
                double esum = 0.0;
                if (!f->kernel_pol) {
                    for (int s = 0; s < ns; ++s) kern[s] = pref[s] * std::exp(-0.5 * rr[s] * rr[s]);
                } else {
                    for (int s = 0; s < ns; ++s) {
                        kern[s] = pref[s] * cov_pp(rr[s]);
                        kder[s] = pref[s] * cov_pp_der(rr[s]);
                    }
                }
                for (int s = 0; s < ns; ++s) esum += kern[s];
                energies[i] += fc * esum;
                double f1[3], f2[3], f3[3];
                for (int l = 0; l < 3; ++l) {
                    double a1 = 0.0, a2 = 0.0, a3 = 0.0;
                    for (int s = 0; s < ns; ++s) {
                        const double d1 = dq1[s] * (u12[l] + u13[l]) +
                                          dq2[s] * 2.0 * (r12 - r13) * (u12[l] - u13[l]);
                        const double d2 = -dq1[s] * u12[l] - dq2[s] * 2.0 * (r12 - r13) * u12[l] +
                                          dq3[s] * u23[l];
                        const double d3 = -dq1[s] * u13[l] - dq2[s] * 2.0 * (r13 - r12) * u13[l] -
                                          dq3[s] * u23[l];
                        if (!f->kernel_pol) {
                            a1 += kern[s] * (dfc[l] + fc * d1);
                            a2 += kern[s] * (-fc13 * df12[l] + fc * d2);
                            a3 += kern[s] * (-fc12 * df13[l] + fc * d3);
                        } else {
                            a1 += kern[s] * dfc[l] - kder[s] * fc * d1;
                            a2 += -kern[s] * fc13 * df12[l] - kder[s] * fc * d2;
                            a3 += -kern[s] * fc12 * df13[l] - kder[s] * fc * d3;
                        }
                    }
                    f1[l] = -a1;
                    f2[l] = -a2;
                    f3[l] = -a3;
                }
                for (int q = 0; q < 3; ++q) {
                    forces[3 * i3 + q] += f1[q];
                    forces[3 * j3 + q] += f2[q];
                    forces[3 * k3 + q] += f3[q];
                }
                vir_add(f2, x12, 0.5);
                vir_add(f3, x13, 0.5);
            }
        }
        k = kself + n_neigh[i];
    }
}

int orc_evaluate_full(int n_sites, const double *positions, const int *species, const double *a,
                      const double *b, const double *c, int n_blocks, const orc_gap_block *blocks,
                      int n_families, const orc_family *families, const double *e0_by_species,
                      int n_species_total, double neighbors_buffer, double max_gbytes,
                      int site_beg, int site_end, double *energies, double *forces,
                      double *virial, int64_t *n_pairs_out) {
    if (site_beg < 0) site_beg = 0;
    if (site_end > n_sites || site_end < 0) site_end = n_sites;
    double rcut_max = 0.0;
    for (int b = 0; b < n_blocks; ++b)
        for (int s = 0; s < blocks[b].hypers.n_species; ++s)
            rcut_max = std::max(rcut_max, blocks[b].hypers.rcut_hard[s]);
    for (int q = 0; q < n_families; ++q)
        rcut_max = std::max(rcut_max, families[q].kind == 3 ? families[q].x[families[q].n - 1]
                                                             : families[q].rcut);
    rcut_max += neighbors_buffer;
    int indices[3];
    orc_number_of_unit_cells(a, b, c, rcut_max, indices);
    const int nrep = indices[0] * indices[1] * indices[2];
    const int nsc = n_sites * nrep;
    std::vector<double> pos_sc(3 * (size_t)nsc);
    std::vector<int> spec_sc(nsc);
    orc_make_supercell(n_sites, positions, species, a, b, c, indices, pos_sc.data(), spec_sc.data());
    double A[3], B[3], C[3];
    for (int q = 0; q < 3; ++q) {
        A[q] = a[q] * indices[0];
        B[q] = b[q] * indices[1];
        C[q] = c[q] * indices[2];
    }
    std::vector<int> do_list(n_sites, 0), n_neigh(n_sites);
    for (int i = site_beg; i < site_end; ++i) do_list[i] = 1;
    int64_t cap = (int64_t)n_sites * 64;
    std::vector<int> nl, nspec;
    std::vector<double> rjs, th, ph, xyz;
    int64_t np;
    for (;;) {
        nl.resize(cap); nspec.resize(cap); rjs.resize(cap); th.resize(cap); ph.resize(cap);
        xyz.resize(3 * cap);
        double a2[3] = {A[0], A[1], A[2]}, b2[3] = {B[0], B[1], B[2]}, c2[3] = {C[0], C[1], C[2]};
        np = orc_build_neighbors_list(nsc, pos_sc.data(), n_sites, a2, b2, c2, rcut_max, indices,
                                      spec_sc.data(), do_list.data(), cap, n_neigh.data(),
                                      nl.data(), rjs.data(), th.data(), ph.data(), xyz.data(),
                                      nspec.data());
        if (np >= 0) break;
        cap = -np;
    }
    if (n_pairs_out) *n_pairs_out = np;
    // turbogap.f90:1253-1261: each rank assigns e0 to its own sites i_beg..i_end
    for (int i = 0; i < n_sites; ++i) {
        const int z = species[i];
        const bool mine = i >= site_beg && i < site_end;
        energies[i] = (mine && z >= 1 && z <= n_species_total && e0_by_species) ? e0_by_species[z - 1]
                                                                                 : 0.0;
    }
    std::vector<double> e_soap(n_sites, 0.0), f_soap(3 * (size_t)n_sites, 0.0);
    double v_soap[9] = {0};
    std::vector<int64_t> pstart(n_sites + 1, 0);
    for (int i = 0; i < n_sites; ++i) pstart[i + 1] = pstart[i] + n_neigh[i];
    std::vector<int> ib(n_sites + 1), ie(n_sites + 1), jb(n_sites + 1), je(n_sites + 1);
    std::vector<double> te(n_sites), tf(3 * (size_t)n_sites);
    for (int bi = 0; bi < n_blocks; ++bi) {
        const orc_gap_block &blk = blocks[bi];
        const orc_soap_hypers *h = &blk.hypers;
        double brc = 0.0;
        for (int s = 0; s < h->n_species; ++s) brc = std::max(brc, h->rcut_hard[s]);
        const int nmax = orc_soap_n_tot(h), dim = orc_soap_dim(h);
        const int nr = site_end - site_beg;
        const int64_t p_off = pstart[site_beg];
        const int nch = orc_atom_pair_batches(nr, n_neigh.data() + site_beg, rjs.data() + p_off, brc,
                                              h->l_max, nmax, dim, h->n_species, max_gbytes,
                                              ib.data(), ie.data(), jb.data(), je.data());
        for (int ch = 0; ch < nch; ++ch) {
            const int i0 = site_beg + ib[ch] - 1, i1 = site_beg + ie[ch];
            const int64_t j0 = p_off + jb[ch] - 1;
            std::fill(te.begin(), te.end(), 0.0);
            std::fill(tf.begin(), tf.end(), 0.0);
            double tv[9];
            orc_get_gap_soap(h, n_sites, i1 - i0, n_neigh.data() + i0, nl.data() + j0,
                             rjs.data() + j0, xyz.data() + 3 * j0, species + i0, species,
                             blk.n_sparse, blk.Qs, blk.alphas, blk.delta, blk.zeta, 1, te.data(),
                             tf.data(), tv);
            for (int i = 0; i < n_sites; ++i) e_soap[i] += te[i];
            for (size_t q = 0; q < tf.size(); ++q) f_soap[q] += tf[q];
            for (int q = 0; q < 9; ++q) v_soap[q] += tv[q];
        }
    }
    for (int i = 0; i < n_sites; ++i) energies[i] += e_soap[i];
    for (size_t q = 0; q < f_soap.size(); ++q) forces[q] = f_soap[q];
    for (int q = 0; q < 9; ++q) virial[q] = v_soap[q];
    // gap_backend_cpu.f90:79-267: every family over this rank's sites and pairs,
    // added to the totals (neighbor_species from the supercell species)
    if (n_families > 0) {
        const int nr = site_end - site_beg;
        const int64_t p0 = pstart[site_beg];
        std::vector<double> fe(n_sites), ff(3 * (size_t)n_sites);
        double fv[9];
        for (int q = 0; q < n_families; ++q) {
            orc_family_energy_forces(&families[q], nr, n_neigh.data() + site_beg, nl.data() + p0,
                                     rjs.data() + p0, xyz.data() + 3 * p0, species + site_beg,
                                     nspec.data() + p0, n_sites, fe.data(), ff.data(), fv);
            for (int i = 0; i < nr; ++i) energies[site_beg + i] += fe[i];
            if (families[q].kind == 2) {
                for (size_t t = 0; t < ff.size(); ++t) forces[t] += ff[t];
            } else {
                for (int i = 0; i < nr; ++i)
                    for (int t = 0; t < 3; ++t) forces[3 * (site_beg + i) + t] += ff[3 * i + t];
            }
            for (int t = 0; t < 9; ++t) virial[t] += fv[t];
        }
    }
    return 0;
}

}  // extern "C"
