// tgb_vdw.cu -- Tkatchenko-Scheffler dispersion from Hirshfeld volumes on the
// device: get_ts_energy_and_forces (src/vdw.f90:163-493) behind tg_get_ts_energy_and_forces.
//
// The volumes and their per-pair derivatives come from the local-property
// predictor (tg_get_local_property, hirshfeld_predict's contract). One warp per
// site: lanes take the pairs of the site's list, the site's energy and the two
// volume prefactors are warp sums, forces and the local virial go out through
// FP64 atomics and the virial is reduced per block. FP64 throughout, with the
// reference's formulas and pair filters, including its quirks: the self pair
// (r = 0) is outside every (rcut_inner, rcut) test, so the central atom's own
// volume gradient adds no force, and the pair force lands on the central atom
// only (the full list holds each pair twice).
#include "tgb_common.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace tgb {
namespace {

struct TsArgs {
    int n_sites, n_sites0, n_species;
    const double *v, *v_der, *v_neigh, *rjs, *xyz, *scaling;
    const int64_t *start;
    const int *nbr, *nspec;
    double rcut, buffer, rcut_inner, buffer_inner, sR, d, x_min, x_max;
    const double *c6_ref, *r0_ref, *alpha0_ref;
    int do_forces;
    double *energies, *forces, *local_virial, *vpart;
};

__device__ __forceinline__ int fmod1(int j, int n) {   // modulo(j - 1, n) for 1-based j >= 1
    return (j - 1) % n;
}

// misc.f90:479-494
__device__ __forceinline__ double poly_cut(double x, double x_min, double x_max) {
    if (x < x_min) return 0.0;
    if (x >= x_max) return 1.0;
    const double c = x - (x_max + x_min) / 2.0, w = x_max - x_min;
    return 0.5 + 1.5 * c / w - 2.0 * c * c * c / (w * w * w);
}

// vdw.f90:287-322: r6 = 1/r^6 times the buffer smoothing, and its r-derivative
// (taken from the unsmoothed r6, as the reference does before it scales r6)
__device__ __forceinline__ void ts_r6(const TsArgs &A, double r, double &r6, double &r6d) {
    const double raw = 1.0 / (r * r * r * r * r * r);
    r6 = raw;
    r6d = -6.0 / r * raw;
    const bool buf = (A.buffer > 0.0 || A.buffer_inner > 0.0) &&
                     ((r > A.rcut - A.buffer && r < A.rcut) ||
                      (r < A.rcut_inner + A.buffer_inner && r > A.rcut_inner));
    if (!buf) return;
    double rb;
    if (r <= A.rcut_inner + A.buffer_inner) {
        const double rbf = -(r - A.rcut_inner - A.buffer_inner) / A.buffer_inner;
        r6d += 6.0 * raw / (-A.buffer_inner) * (-rbf + rbf * rbf);
        rb = (r - A.rcut_inner - A.buffer_inner) / (-A.buffer_inner);
    } else {
        const double rbf = (r - A.rcut + A.buffer) / A.buffer;
        r6d += 6.0 * raw / A.buffer * (-rbf + rbf * rbf);
        rb = (r - A.rcut + A.buffer) / A.buffer;
    }
    r6 = raw * (1.0 - 3.0 * rb * rb + 2.0 * rb * rb * rb);
}

// One warp per site i: energies(i), then (do_forces) the volume-gradient forces
// on the site's neighbours and the pair forces on i, the virial and the local
// virial diagonal.
__global__ void k_ts(TsArgs A) {
    __shared__ double vred[8][9];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * (blockDim.x >> 5) + warp;
    double vir[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (i < A.n_sites) {
        const int64_t k0 = A.start[i], k1 = A.start[i + 1];
        const int i2 = fmod1(A.nbr[k0], A.n_sites0);
        // the central atom's quantities from its self pair (vdw.f90:343-351)
        const int si = A.nspec[k0] - 1;
        const double vi = A.v_neigh[k0];
        const double c6_ii = A.c6_ref[si] * vi * vi * A.scaling[i2];
        const double r0_i = A.r0_ref[si] * pow(vi, 1.0 / 3.0);
        const double a0_i = A.alpha0_ref[si] * vi;
        double e = 0.0, pf1 = 0.0, pf2 = 0.0;
        for (int64_t k = k0 + 1 + lane; k < k1; k += 32) {
            const double r = A.rjs[k];
            if (!(r > A.rcut_inner && r < A.rcut)) continue;
            const int sj = A.nspec[k] - 1, j2 = fmod1(A.nbr[k], A.n_sites0);
            const double vj = A.v_neigh[k];
            const double c6_jj = A.c6_ref[sj] * vj * vj * A.scaling[j2];
            const double a0_j = A.alpha0_ref[sj] * vj;
            const double c6_ij = (c6_ii == 0.0 || c6_jj == 0.0)
                                     ? 0.0
                                     : (2.0 * c6_ii * c6_jj) / (a0_j / a0_i * c6_ii + a0_i / a0_j * c6_jj);
            const double r0_ij = r0_i + A.r0_ref[sj] * pow(vj, 1.0 / 3.0);
            double r6, r6d;
            ts_r6(A, r, r6, r6d);
            const double ed = exp(-A.d * (r / (A.sR * r0_ij) - 1.0));
            const double fd = 1.0 / (1.0 + ed);
            e += c6_ij * r6 * fd;
            if (!A.do_forces) continue;
            pf1 += c6_ij * fd * r6;
            pf2 -= c6_ij * fd * fd * r * r6 * ed * A.d / A.sR / (r0_ij * r0_ij);
        }
        e = warp_sum(e);
        if (lane == 0) A.energies[i] = -0.5 * e;
        if (A.do_forces) {
            pf1 = warp_sum(pf1);
            pf2 = warp_sum(pf2);
            // vdw.f90:413-420 (i2 there is the central atom's species)
            const double vh = A.v[i];
            if (vh == 0.0) {
                pf1 = 0.0;
                pf2 = 0.0;
            } else {
                pf1 = pf1 / vh;
                pf2 = pf2 * A.r0_ref[si] / 3.0 / pow(vh, 2.0 / 3.0);
            }
            const double pref = pf1 + pf2;
            for (int64_t k = k0 + lane; k < k1; k += 32) {
                const double r = A.rjs[k];
                if (!(r > A.rcut_inner && r < A.rcut)) continue;
                const int j2 = fmod1(A.nbr[k], A.n_sites0);
                const double x[3] = {A.xyz[3 * k], A.xyz[3 * k + 1], A.xyz[3 * k + 2]};
                const double pc = poly_cut(r, A.x_min, A.x_max);
                const double *g = A.v_der + 3 * k;
                if (!(g[0] == 0.0 && g[1] == 0.0 && g[2] == 0.0)) {
                    const double f[3] = {g[0] * pref, g[1] * pref, g[2] * pref};
                    for (int q = 0; q < 3; ++q) {
                        atomicAdd(A.forces + 3 * (size_t)j2 + q, f[q]);
                        atomicAdd(A.local_virial + 3 * (size_t)j2 + q, f[q] * x[q] * pc);
                        for (int q2 = 0; q2 < 3; ++q2)
                            vir[3 * q + q2] += 0.5 * (f[q] * x[q2] + f[q2] * x[q]);
                    }
                }
                // the pair term (vdw.f90:455-485), with the pair quantities again
                const int sj = A.nspec[k] - 1;
                const double vj = A.v_neigh[k];
                const double c6_jj = A.c6_ref[sj] * vj * vj * A.scaling[j2];
                const double a0_j = A.alpha0_ref[sj] * vj;
                const double c6_ij = (c6_ii == 0.0 || c6_jj == 0.0)
                                         ? 0.0
                                         : (2.0 * c6_ii * c6_jj) /
                                               (a0_j / a0_i * c6_ii + a0_i / a0_j * c6_jj);
                const double r0_ij = r0_i + A.r0_ref[sj] * pow(vj, 1.0 / 3.0);
                double f[3] = {0.0, 0.0, 0.0};
                if (r0_ij != 0.0) {
                    double r6, r6d;
                    ts_r6(A, r, r6, r6d);
                    const double ed = exp(-A.d * (r / (A.sR * r0_ij) - 1.0));
                    const double fd = 1.0 / (1.0 + ed);
                    const double s = c6_ij / r * fd * (-r6d - r6 * fd * ed * A.d / A.sR / r0_ij);
                    for (int q = 0; q < 3; ++q) f[q] = s * x[q];
                }
                if (j2 != i2)
                    for (int q = 0; q < 3; ++q) atomicAdd(A.forces + 3 * (size_t)i2 + q, f[q]);
                for (int q = 0; q < 3; ++q) {
                    atomicAdd(A.local_virial + 3 * (size_t)j2 + q, -0.5 * f[q] * x[q] * pc);
                    for (int q2 = 0; q2 < 3; ++q2)
                        vir[3 * q + q2] -= 0.25 * (f[q] * x[q2] + f[q2] * x[q]);
                }
            }
        }
    }
    for (int q = 0; q < 9; ++q) vir[q] = warp_sum(vir[q]);
    if (lane == 0)
        for (int q = 0; q < 9; ++q) vred[warp][q] = vir[q];
    __syncthreads();
    if (threadIdx.x < 9) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += vred[w][threadIdx.x];
        A.vpart[(size_t)blockIdx.x * 9 + threadIdx.x] = s;
    }
}

template <typename T>
struct DevBuf {
    T *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    int alloc(size_t n) {
        TGB_CUDA(cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)));
        return TG_OK;
    }
    int put(const T *h, size_t n, cudaStream_t st) {
        TGB_TRY(alloc(n));
        if (n) TGB_CUDA(cudaMemcpyAsync(p, h, sizeof(T) * n, cudaMemcpyHostToDevice, st));
        return TG_OK;
    }
};

}  // namespace
}  // namespace tgb

using namespace tgb;

extern "C" int tg_get_ts_energy_and_forces(
    int32_t n_sites, int32_t n_sites0, const double *hirshfeld_v, const double *hirshfeld_v_cart_der,
    const int32_t *n_neigh, const int32_t *neighbors_list, const int32_t *neighbor_species,
    double rcut, double buffer, double rcut_inner, double buffer_inner, const double *rjs,
    const double *xyz, const double *hirshfeld_v_neigh, double sR, double d, int32_t n_species,
    const double *c6_ref, const double *r0_ref, const double *alpha0_ref, int32_t do_forces,
    double x_min, double x_max, const double *mbd_ts_scaling, double *energies, double *forces0,
    double *virial, double *local_virial_diag0) {
    TGB_CHECK(n_sites >= 0 && n_sites0 >= 1 && n_species >= 1 && n_neigh && neighbors_list &&
                  neighbor_species && rjs && xyz && hirshfeld_v && hirshfeld_v_neigh && c6_ref &&
                  r0_ref && alpha0_ref && mbd_ts_scaling && energies,
              TG_ERR_ARG, "null or empty TS argument");
    TGB_CHECK(!do_forces || (hirshfeld_v_cart_der && forces0 && virial && local_virial_diag0),
              TG_ERR_ARG, "forces need the volume derivatives and the force, virial outputs");
    std::vector<int64_t> start(n_sites + 1, 0);
    for (int i = 0; i < n_sites; ++i) start[i + 1] = start[i] + n_neigh[i];
    const int64_t P = start[n_sites];
    for (int64_t k = 0; k < P; ++k) {
        TGB_CHECK(neighbor_species[k] >= 1 && neighbor_species[k] <= n_species && neighbors_list[k] >= 1,
                  TG_ERR_ARG, "pair %lld: species %d or neighbour %d out of range", (long long)k,
                  neighbor_species[k], neighbors_list[k]);
    }
    for (int i = 0; i < n_sites; ++i)
        TGB_CHECK(n_neigh[i] >= 1, TG_ERR_ARG, "site %d has no self pair", i);
    cudaStream_t st = nullptr;
    TGB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
    DevBuf<int64_t> dstart;
    DevBuf<int> dnbr, dspec;
    DevBuf<double> dv, dvd, dvn, drjs, dxyz, dsc, dc6, dr0, da0, den, dfo, dlv, dvp;
    TGB_TRY(dstart.put(start.data(), start.size(), st));
    TGB_TRY(dnbr.put(neighbors_list, P, st));
    TGB_TRY(dspec.put(neighbor_species, P, st));
    TGB_TRY(dv.put(hirshfeld_v, n_sites, st));
    TGB_TRY(dvn.put(hirshfeld_v_neigh, P, st));
    TGB_TRY(drjs.put(rjs, P, st));
    TGB_TRY(dxyz.put(xyz, 3 * (size_t)P, st));
    TGB_TRY(dsc.put(mbd_ts_scaling, n_sites0, st));
    TGB_TRY(dc6.put(c6_ref, n_species, st));
    TGB_TRY(dr0.put(r0_ref, n_species, st));
    TGB_TRY(da0.put(alpha0_ref, n_species, st));
    if (do_forces) TGB_TRY(dvd.put(hirshfeld_v_cart_der, 3 * (size_t)P, st));
    TGB_TRY(den.alloc(n_sites));
    TGB_TRY(dfo.alloc(3 * (size_t)n_sites0));
    TGB_TRY(dlv.alloc(3 * (size_t)n_sites0));
    TGB_CUDA(cudaMemsetAsync(dfo.p, 0, sizeof(double) * 3 * n_sites0, st));
    TGB_CUDA(cudaMemsetAsync(dlv.p, 0, sizeof(double) * 3 * n_sites0, st));
    const int warps = 8, grid = (n_sites + warps - 1) / warps;
    TGB_TRY(dvp.alloc(9 * (size_t)std::max(grid, 1)));
    TsArgs A{n_sites, n_sites0, n_species, dv.p, dvd.p, dvn.p, drjs.p, dxyz.p, dsc.p, dstart.p,
             dnbr.p, dspec.p, rcut, buffer, rcut_inner, buffer_inner, sR, d, x_min, x_max,
             dc6.p, dr0.p, da0.p, do_forces ? 1 : 0, den.p, dfo.p, dlv.p, dvp.p};
    if (grid > 0) {
        k_ts<<<grid, 32 * warps, 0, st>>>(A);
        TGB_CUDA(cudaGetLastError());
    }
    std::vector<double> vp(9 * (size_t)std::max(grid, 1), 0.0);
    if (n_sites > 0)
        TGB_CUDA(cudaMemcpyAsync(energies, den.p, sizeof(double) * n_sites, cudaMemcpyDeviceToHost, st));
    if (do_forces) {
        TGB_CUDA(cudaMemcpyAsync(forces0, dfo.p, sizeof(double) * 3 * n_sites0, cudaMemcpyDeviceToHost, st));
        TGB_CUDA(cudaMemcpyAsync(local_virial_diag0, dlv.p, sizeof(double) * 3 * n_sites0,
                                 cudaMemcpyDeviceToHost, st));
        if (grid > 0)
            TGB_CUDA(cudaMemcpyAsync(vp.data(), dvp.p, sizeof(double) * 9 * grid, cudaMemcpyDeviceToHost, st));
    }
    TGB_CUDA(cudaStreamSynchronize(st));
    if (do_forces) {
        // virial(k1, k2), column-major as the Fortran array
        for (int q = 0; q < 9; ++q) virial[q] = 0.0;
        for (int b = 0; b < grid; ++b)
            for (int q = 0; q < 3; ++q)
                for (int q2 = 0; q2 < 3; ++q2) virial[q + 3 * q2] += vp[9 * (size_t)b + 3 * q + q2];
    }
    return TG_OK;
}
