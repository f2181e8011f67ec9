// tgb_neighbors.cu -- neighbour lists and FP64 MD kernels.
//
// Compiled with --fmad=false: every expression here must round exactly as the
// reference's FP64 Fortran does (two roundings for a*b+c), so that neighbour
// indices, rjs and xyz are bit-identical to build_neighbors_list
// (src/neighbors.f90:243-605) and velocity_verlet (src/md.f90:226-283) matches
// given identical inputs.

#include "tgb_neighbors.cuh"

#include <algorithm>

#include <cub/device/device_scan.cuh>

namespace tgb {

// Fortran MODULO for reals as gfortran evaluates it: fmod, then shift into the
// sign of p; an exact zero takes the sign of p. fmod(a, p) == a whenever |a| < |p|,
// which skips the slow path for positions already inside the box.
__device__ __forceinline__ double f_modulo(double a, double p) {
    double r = (fabs(a) < fabs(p)) ? a : fmod(a, p);
    if (r != 0.0) {
        if ((a < 0.0) != (p < 0.0)) r = r + p;
    } else {
        r = copysign(0.0, p);
    }
    return r;
}

__device__ __forceinline__ double dot3(const double *x, const double *y) {
    double s = x[0] * y[0];
    s = s + x[1] * y[1];
    s = s + x[2] * y[2];
    return s;
}

// get_distance (src/neighbors.f90:47-163), all-periodic.
__device__ void get_distance(const double *posi, const double *posj, const Box &bx, double *dist,
                             double *d) {
    if (bx.ortho) {
        double d2 = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double L = bx.L[i];
            double v = f_modulo(posj[i] - posi[i], L);
            if (v > L / 2.0) v = v - L;
            dist[i] = v;
            d2 = d2 + v * v;
        }
        *d = sqrt(d2);
        return;
    }
    double dd[3] = {posj[0] - posi[0], posj[1] - posi[1], posj[2] - posi[2]};
    double v[3] = {-1.0 * dot3(dd, bx.a), -1.0 * dot3(dd, bx.b), -1.0 * dot3(dd, bx.c)};
    double ir[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int j = 0; j < 3; ++j) s = s + bx.inv[i][j] * v[j];
        ir[i] = s;
    }
    int idx[3];
    for (int i = 0; i < 3; ++i) idx[i] = (int)llround(ir[i]);
    double res_opt = 1.e10, opt[3] = {0, 0, 0};
    for (int i = idx[0] - 1; i <= idx[0] + 1; ++i)
        for (int j = idx[1] - 1; j <= idx[1] + 1; ++j)
            for (int k = idx[2] - 1; k <= idx[2] + 1; ++k) {
                double t[3];
                for (int q = 0; q < 3; ++q)
                    t[q] = dd[q] + (double)i * bx.a[q] + (double)j * bx.b[q] + (double)k * bx.c[q];
                const double res = dot3(t, t);
                if (res < res_opt) {
                    res_opt = res;
                    opt[0] = t[0]; opt[1] = t[1]; opt[2] = t[2];
                }
            }
    dist[0] = opt[0]; dist[1] = opt[1]; dist[2] = opt[2];
    *d = sqrt(dot3(dist, dist));
}

namespace {

__device__ __forceinline__ int imod(int x, int m) {
    int r = x % m;
    return r < 0 ? r + m : r;
}

// Cell of atom i (neighbors.f90:398-408): MIC vector from the box centre,
// shifted back by the centre, scaled by cells per length.
__device__ __forceinline__ void cell_coords(const double *p, const Box &bx, const CellGrid &g,
                                            int *ci) {
    const double tol = 1.e-10;
    const double ctr[3] = {bx.L[0] / 2.0, bx.L[1] / 2.0, bx.L[2] / 2.0};
    double dist[3], d;
    get_distance(ctr, p, bx, dist, &d);
    const int m[3] = {g.mx, g.my, g.mz};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double v = dist[q] + ctr[q];
        ci[q] = (int)(v / (bx.L[q] + tol) * (double)m[q]);
    }
}

__global__ void k_cell_assign(int n, const double *__restrict__ pos, Box bx, CellGrid g,
                              int *__restrict__ cell_xyz, int *__restrict__ cell_count,
                              const int *__restrict__ when) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (when && !*when)) return;
    int c[3];
    cell_coords(pos + 3 * (size_t)i, bx, g, c);
    cell_xyz[3 * i] = c[0];
    cell_xyz[3 * i + 1] = c[1];
    cell_xyz[3 * i + 2] = c[2];
    const int id = imod(c[0], g.mx) + imod(c[1], g.my) * g.mx + imod(c[2], g.mz) * g.my * g.mx;
    atomicAdd(&cell_count[id], 1);
}

__global__ void k_cell_fill(int n, const int *__restrict__ cell_xyz, CellGrid g,
                            const int *__restrict__ cell_start, int *__restrict__ cell_fill,
                            int *__restrict__ cell_atoms, const int *__restrict__ when) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (when && !*when)) return;
    const int id = imod(cell_xyz[3 * i], g.mx) + imod(cell_xyz[3 * i + 1], g.my) * g.mx +
                   imod(cell_xyz[3 * i + 2], g.mz) * g.my * g.mx;
    const int slot = atomicAdd(&cell_fill[id], 1);
    cell_atoms[cell_start[id] + slot] = i;
}

// The reference links each cell's atoms by head insertion, so a cell is walked
// in descending atom index (neighbors.f90:398-408, 460-463).
__global__ void k_cell_sort(int ncells, const int *__restrict__ cell_start,
                            const int *__restrict__ cell_count, int *__restrict__ cell_atoms,
                            const int *__restrict__ when) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells || (when && !*when)) return;
    int *a = cell_atoms + cell_start[c];
    const int n = cell_count[c];
    for (int i = 1; i < n; ++i) {
        const int v = a[i];
        int j = i - 1;
        while (j >= 0 && a[j] < v) {
            a[j + 1] = a[j];
            --j;
        }
        a[j + 1] = v;
    }
}

struct PairSink {
    // count mode when nbr == nullptr
    int64_t base;
    int64_t cap;
    int *nbr;
    double *rjs;
    double *xyz;
    unsigned *err;
    int count;
    __device__ __forceinline__ void emit(int j, double d, const double *dist) {
        if (nbr) {
            const int64_t p = base + count;
            if (p < cap) {
                nbr[p] = j;
                rjs[p] = d;
                xyz[3 * p] = dist[0];
                xyz[3 * p + 1] = dist[1];
                xyz[3 * p + 2] = dist[2];
            } else {
                atomicOr(err, (unsigned)DEV_ERR_NEIGH_CAPACITY);
            }
        }
        ++count;
    }
};

// Cell-list search (neighbors.f90:409-472): per atom, self first, then the cells
// k3 (z) outer, j3, i3 inner with the reference's skips for 1- and 2-cell axes,
// each cell in descending atom index. The candidates of the (up to) 27 cells form
// one flattened sequence in that order; lanes test 32 consecutive candidates at a
// time and emit the accepted ones in sequence order (ballot + prefix popcount),
// so the pairs come out exactly in the reference's order.
// One CTA per cell: its warps stage the candidates of the cell's neighbourhood in
// shared memory together (CAP at a time), and warp w lists the cell's atoms w,
// w + WARPS, ... from there, so candidate positions and indices are read from
// global memory once per cell instead of once per atom.
// Three uses, as in the batched search: count (pstart and slots unset), count
// into slot rows (slots > 0: pair e of site i at row i * slots + e while e <
// slots, *ovf set past it), and fill at pstart (only when *gate is set, if given).
constexpr int kNlCellWarps = 4, kNlCellCap = 256;   // 7 KB of staging per CTA

// The 27 neighbour cells' candidate ranges (lane c < 27) and their inclusive
// prefix sum over the warp; the flattened candidate f of a warp lies in the cell
// found by binary lifting over the prefix sums.
struct CellWalk {
    int cstart, ccount, incl, total;
    __device__ __forceinline__ void scan(int lane) {
        incl = ccount;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        total = __shfl_sync(0xffffffffu, incl, 31);
    }
    // slot in cell_atoms of candidate fc (every lane of the warp calls it)
    __device__ __forceinline__ int slot_of(int fc) const {
        int c = 0;
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
            const int probe = c + step - 1;
            const int v = __shfl_sync(0xffffffffu, incl, probe < 31 ? probe : 31);
            if (probe < 27 && v <= fc) c += step;
        }
        const int cs = __shfl_sync(0xffffffffu, cstart, c);
        const int before = __shfl_sync(0xffffffffu, incl, c) - __shfl_sync(0xffffffffu, ccount, c);
        return cs + (fc - before);
    }
};

// Candidates [f_beg, f_end) of the walk into shared memory, warp w taking every
// WARPS-th group of 32 (positions from the cell-ordered copy when there is one).
template <int WARPS>
__device__ __forceinline__ void stage_candidates(const CellWalk &cw, int f_beg, int f_end, int w,
                                                 int lane, const int *__restrict__ cell_atoms,
                                                 const double *__restrict__ cell_pos,
                                                 const double *__restrict__ pos, int *sk,
                                                 double *sx, double *sy, double *sz) {
    for (int f0 = f_beg + 32 * w; f0 < f_end; f0 += 32 * WARPS) {   // warp-uniform trip count
        const int f = f0 + lane;
        const int slot = cw.slot_of(f < f_end ? f : f_end - 1);
        if (f < f_end) {
            const int k = cell_atoms[slot];
            const double *pk = cell_pos ? cell_pos + 3 * (size_t)slot : pos + 3 * (size_t)k;
            sk[f - f_beg] = k;
            sx[f - f_beg] = pk[0];
            sy[f - f_beg] = pk[1];
            sz[f - f_beg] = pk[2];
        }
    }
}

template <int WARPS, int CAP>
__global__ void __launch_bounds__(32 * WARPS)
    k_nl_cells_cell(int ncells, const double *__restrict__ pos, Box bx, CellGrid g, double rcut,
                    const int *__restrict__ do_list, const int *__restrict__ cell_xyz,
                    const int *__restrict__ cell_start, const int *__restrict__ cell_count,
                    const int *__restrict__ cell_atoms, const double *__restrict__ cell_pos,
                    int *__restrict__ n_neigh, const int64_t *__restrict__ pstart, int64_t cap,
                    int *__restrict__ nbr, double *__restrict__ rjs, double *__restrict__ xyz,
                    unsigned *err, const int *__restrict__ when, int slots, int *__restrict__ ovf,
                    const int *__restrict__ gate) {
    __shared__ double sx[CAP], sy[CAP], sz[CAP];
    __shared__ int sk[CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int cell = blockIdx.x;   // every exit before the loop is CTA-uniform
    if (cell >= ncells || (when && !*when) || (gate && !*gate)) return;
    const int na = cell_count[cell];
    if (na == 0) return;
    const int c0 = cell_start[cell];
    const bool slotted = !pstart && slots > 0;
    const bool writes = pstart || slotted;
    const int a0 = cell_atoms[c0];
    const int i2 = 1 + cell_xyz[3 * a0], j2 = 1 + cell_xyz[3 * a0 + 1], k2 = 1 + cell_xyz[3 * a0 + 2];
    const int mx = g.mx, my = g.my, mz = g.mz;
    CellWalk cw{0, 0, 0, 0};
    if (lane < 27) {
        const int k3 = k2 - 1 + lane / 9, j3 = j2 - 1 + (lane / 3) % 3, i3 = i2 - 1 + lane % 3;
        bool skip = false;
        skip |= (mz == 1 && k3 != 1) || (mz == 2 && k2 == 1 && k3 == 0) || (mz == 2 && k2 == 2 && k3 == 3);
        skip |= (my == 1 && j3 != 1) || (my == 2 && j2 == 1 && j3 == 0) || (my == 2 && j2 == 2 && j3 == 3);
        skip |= (mx == 1 && i3 != 1) || (mx == 2 && i2 == 1 && i3 == 0) || (mx == 2 && i2 == 2 && i3 == 3);
        if (!skip) {
            const int c = imod(i3 - 1, mx) + imod(j3 - 1, my) * mx + imod(k3 - 1, mz) * mx * my;
            cw.cstart = cell_start[c];
            cw.ccount = cell_count[c];
        }
    }
    cw.scan(lane);
    const int total = cw.total;
    const int nround = (total + CAP - 1) / CAP;
    const double rc2 = rcut * rcut, rc2_lo = rc2 * (1.0 - 1e-12), rc2_hi = rc2 * (1.0 + 1e-12);
    if (nround == 1) {
        stage_candidates<WARPS>(cw, 0, total, w, lane, cell_atoms, cell_pos, pos, sk, sx, sy, sz);
        __syncthreads();
    }
    for (int ag = 0; ag < na; ag += WARPS) {   // CTA-uniform trip count
        const int a = ag + w;
        const int i = a < na ? cell_atoms[c0 + a] : -1;
        const bool listed = i >= 0 && !(do_list && !do_list[i]);   // warp-uniform
        if (i >= 0 && !listed && !pstart && lane == 0) n_neigh[i] = 0;
        double pi[3] = {0.0, 0.0, 0.0};
        int64_t base = 0, lim = 0;
        if (listed) {
            pi[0] = pos[3 * (size_t)i];
            pi[1] = pos[3 * (size_t)i + 1];
            pi[2] = pos[3 * (size_t)i + 2];
            base = pstart ? pstart[i] : (slotted ? (int64_t)i * slots : 0);
            lim = pstart ? cap : base + slots;
            if (writes && lane == 0) {   // self pair first
                if (base < lim) {
                    nbr[base] = i;
                    rjs[base] = 0.0;
                    xyz[3 * base] = 0.0;
                    xyz[3 * base + 1] = 0.0;
                    xyz[3 * base + 2] = 0.0;
                } else {
                    atomicOr(err, (unsigned)DEV_ERR_NEIGH_CAPACITY);
                }
            }
        }
        int count = 1;
        for (int r = 0; r < nround; ++r) {   // CTA-uniform trip count
            const int f_beg = r * CAP, f_end = min(total, f_beg + CAP);
            if (nround > 1) {   // a large neighbourhood: staged again, round by round
                __syncthreads();   // every warp is done with the previous round
                stage_candidates<WARPS>(cw, f_beg, f_end, w, lane, cell_atoms, cell_pos, pos, sk, sx,
                                        sy, sz);
                __syncthreads();
            }
            if (!listed) continue;
            for (int f0 = f_beg; f0 < f_end; f0 += 32) {   // warp-uniform trip count
                const int f = f0 + lane;
                bool take = false;
                int k = -1;
                double dist[3] = {0.0, 0.0, 0.0}, d = 0.0;
                if (f < f_end) {
                    k = sk[f - f_beg];
                    if (k != i) {
                        const double pk[3] = {sx[f - f_beg], sy[f - f_beg], sz[f - f_beg]};
                        double d2 = 0.0;
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            const double L = bx.L[q];
                            double v = f_modulo(pk[q] - pi[q], L);
                            if (v > L / 2.0) v = v - L;
                            dist[q] = v;
                            d2 = d2 + v * v;
                        }
                        if (d2 < rc2_lo) {
                            take = true;
                            if (writes) d = sqrt(d2);
                        } else if (d2 <= rc2_hi) {
                            d = sqrt(d2);
                            take = d < rcut;
                        }
                    }
                }
                const unsigned m = __ballot_sync(0xffffffffu, take);
                if (writes && take) {
                    const int64_t p = base + count + __popc(m & ((1u << lane) - 1u));
                    if (p < lim) {
                        nbr[p] = k;
                        rjs[p] = d;
                        xyz[3 * p] = dist[0];
                        xyz[3 * p + 1] = dist[1];
                        xyz[3 * p + 2] = dist[2];
                    } else if (slotted) {
                        *ovf = 1;   // the filling search makes this build
                    } else {
                        atomicOr(err, (unsigned)DEV_ERR_NEIGH_CAPACITY);
                    }
                }
                count += __popc(m);
            }
        }
        if (listed && !pstart && lane == 0) n_neigh[i] = count;
    }
}

// Slot rows to the compact arrays (a warp per site), unless a row overflowed.
__global__ void k_nl_compact(int n_sites, int slots, const int *__restrict__ n_neigh,
                             const int64_t *__restrict__ pstart, const int *__restrict__ snbr,
                             const double *__restrict__ srjs, const double *__restrict__ sxyz,
                             const int *__restrict__ ovf, const int *__restrict__ when, int64_t cap,
                             int *__restrict__ nbr, double *__restrict__ rjs,
                             double *__restrict__ xyz, unsigned *err) {
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n_sites || *ovf || (when && !*when)) return;
    const int cnt = n_neigh[i];
    const int64_t dst = pstart[i], src = (int64_t)i * slots;
    if (dst + cnt > cap) {
        if (lane == 0) atomicOr(err, (unsigned)DEV_ERR_NEIGH_CAPACITY);
        return;
    }
    for (int e = lane; e < cnt; e += 32) {
        nbr[dst + e] = snbr[src + e];
        rjs[dst + e] = srjs[src + e];
    }
    for (int e = lane; e < 3 * cnt; e += 32) xyz[3 * dst + e] = sxyz[3 * src + e];
}

// O(N * N_supercell) search (neighbors.f90:474-514): ascending supercell index.
__global__ void k_nl_brute(int n_sites, int n_sc, const double *__restrict__ pos, Box bx,
                           double rcut, const int *__restrict__ do_list, int *__restrict__ n_neigh,
                           const int64_t *__restrict__ pstart, int64_t cap, int *__restrict__ nbr,
                           double *__restrict__ rjs, double *__restrict__ xyz, unsigned *err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_sites) return;
    if (do_list && !do_list[i]) {
        if (!pstart) n_neigh[i] = 0;
        return;
    }
    PairSink sink{pstart ? pstart[i] : 0, cap, pstart ? nbr : nullptr, rjs, xyz, err, 0};
    const double zero3[3] = {0.0, 0.0, 0.0};
    sink.emit(i, 0.0, zero3);
    const double *pi = pos + 3 * (size_t)i;
    for (int j = 0; j < n_sc; ++j) {
        if (j == i) continue;
        double dist[3], d;
        get_distance(pi, pos + 3 * (size_t)j, bx, dist, &d);
        if (d < rcut) sink.emit(j, d, dist);
    }
    if (!pstart) n_neigh[i] = sink.count;
}

__global__ void k_pstart_zero(int64_t *pstart) { pstart[0] = 0; }

// positions in cell order, so that a cell's candidates are read contiguously
__global__ void k_cell_gather_pos(int n, const int *__restrict__ cell_atoms,
                                  const double *__restrict__ pos, double *__restrict__ cell_pos,
                                  const int *__restrict__ when) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || (when && !*when)) return;
    const int k = cell_atoms[s];
    cell_pos[3 * (size_t)s] = pos[3 * (size_t)k];
    cell_pos[3 * (size_t)s + 1] = pos[3 * (size_t)k + 1];
    cell_pos[3 * (size_t)s + 2] = pos[3 * (size_t)k + 2];
}

__global__ void k_angles(int64_t P, const double *__restrict__ rjs, const double *__restrict__ xyz,
                         const int *__restrict__ is_self, double *__restrict__ th,
                         double *__restrict__ ph) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= P) return;
    if (is_self[p]) {
        th[p] = 0.0;
        ph[p] = 0.0;
        return;
    }
    const double d = rjs[p];
    const double x = xyz[3 * p], y = xyz[3 * p + 1], z = xyz[3 * p + 2];
    if (fabs(z) >= d) th[p] = z > 0.0 ? 0.0 : acos(-1.0);
    else th[p] = acos(z / d);
    ph[p] = atan2(y, x);
}

// read_files.f90:347-363 supercell replicas: a-index, b, c, then atom.
__global__ void k_supercell(int n, const double *__restrict__ pos, const double *a,
                            const double *b, const double *c, int ia, int ib, int ic,
                            double *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nrep = ia * ib * ic;
    if (t >= n * nrep) return;
    const int r = t / n, i = t % n;
    const int i2 = r / (ib * ic), j2 = (r / ic) % ib, k2 = r % ic;
#pragma unroll
    for (int q = 0; q < 3; ++q)
        out[3 * (size_t)t + q] = pos[3 * (size_t)i + q] + (double)i2 * a[q] + (double)j2 * b[q] +
                                 (double)k2 * c[q];
}

// velocity_verlet (md.f90:226-283) on (3, n) arrays, no fixed atoms.
__global__ void k_velocity_verlet(int n, double *__restrict__ pos, double *__restrict__ pos_prev,
                                  double *__restrict__ vel, const double *__restrict__ f,
                                  double *__restrict__ f_prev, const double *__restrict__ m,
                                  double dt, double dt_prev, int first_step) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * n) return;
    const int i = t / 3;
    const double mi = m[i];
    double v = vel[t];
    if (!first_step) v = v + 0.5 * (f[t] + f_prev[t]) / mi * dt_prev;
    vel[t] = v;
    const double p = pos[t];
    pos_prev[t] = p;
    f_prev[t] = f[t];
    pos[t] = p + v * dt + 0.5 * f[t] / mi * (dt * dt);
}

// wrap_pbc (md.f90:348-380), orthorhombic: i_shift = floor(x / L).
__global__ void k_wrap_ortho(int n, double *__restrict__ pos, Box bx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double *p = pos + 3 * (size_t)i;
    const double s0 = floor(p[0] / bx.a[0]), s1 = floor(p[1] / bx.b[1]), s2 = floor(p[2] / bx.c[2]);
#pragma unroll
    for (int q = 0; q < 3; ++q)
        p[q] = p[q] - (double)(int)s0 * bx.a[q] - (double)(int)s1 * bx.b[q] -
               (double)(int)s2 * bx.c[q];
}

// wrap_pbc (md.f90:348-380), triclinic: i_shift from get_distance of the origin
// and the atom (neighbors.f90:107-140): floor of minus the Gram-inverse solution,
// in the reference's operation order.
__global__ void k_wrap_tri(int n, double *__restrict__ pos, Box bx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double *p = pos + 3 * (size_t)i;
    const double dd[3] = {p[0], p[1], p[2]};   // posj - posi with posi = 0
    const double v[3] = {-1.0 * dot3(dd, bx.a), -1.0 * dot3(dd, bx.b), -1.0 * dot3(dd, bx.c)};
    int sh[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double s = 0.0;
        for (int j = 0; j < 3; ++j) s = s + bx.inv[r][j] * v[j];
        sh[r] = (int)floor(-s);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q)
        p[q] = p[q] - (double)sh[0] * bx.a[q] - (double)sh[1] * bx.b[q] - (double)sh[2] * bx.c[q];
}

// sum_i m_i v_i (3) and sum_i m_i (1) into acc[4] (FP64 atomics, then apply)
__global__ void k_cm_accumulate(int n, const double *__restrict__ vel, const double *__restrict__ m,
                                double *acc) {
    double s[4] = {0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double mi = m[i];
        s[0] += mi * vel[3 * (size_t)i];
        s[1] += mi * vel[3 * (size_t)i + 1];
        s[2] += mi * vel[3 * (size_t)i + 2];
        s[3] += mi;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) s[q] = warp_sum(s[q]);
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 4; ++q) atomicAdd(&acc[q], s[q]);
}

__global__ void k_cm_apply(int n, double *__restrict__ vel, const double *__restrict__ acc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * n) return;
    vel[t] = vel[t] - acc[t % 3] / acc[3];
}

__global__ void k_kinetic(int n, const double *__restrict__ vel, const double *__restrict__ m,
                          double *acc) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double *v = vel + 3 * (size_t)i;
        s += 0.5 * m[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc, s);
}

}  // namespace

Box make_box(const double *a, const double *b, const double *c) {
    Box bx{};
    for (int q = 0; q < 3; ++q) { bx.a[q] = a[q]; bx.b[q] = b[q]; bx.c[q] = c[q]; }
    const double tol = 1.e-6;
    bx.ortho = fabs(a[1]) < tol && fabs(a[2]) < tol && fabs(b[0]) < tol && fabs(b[2]) < tol &&
               fabs(c[0]) < tol && fabs(c[1]) < tol;
    bx.L[0] = a[0]; bx.L[1] = b[1]; bx.L[2] = c[2];
    // Gram matrix inverse for the triclinic branch (neighbors.f90:107-134).
    auto d3 = [](const double *x, const double *y) {
        double s = x[0] * y[0];
        s = s + x[1] * y[1];
        s = s + x[2] * y[2];
        return s;
    };
    double m[3][3];
    m[0][0] = d3(a, a); m[0][1] = d3(a, b); m[0][2] = d3(a, c);
    m[1][0] = m[0][1];  m[1][1] = d3(b, b); m[1][2] = d3(b, c);
    m[2][0] = m[0][2];  m[2][1] = m[1][2];  m[2][2] = d3(c, c);
    const double md = -m[0][2] * m[0][2] * m[1][1] + 2.0 * m[0][1] * m[0][2] * m[1][2] -
                      m[0][0] * m[1][2] * m[1][2] - m[0][1] * m[0][1] * m[2][2] +
                      m[0][0] * m[1][1] * m[2][2];
    double inv[3][3];
    inv[0][0] = m[1][1] * m[2][2] - m[1][2] * m[1][2];
    inv[0][1] = m[0][2] * m[1][2] - m[0][1] * m[2][2];
    inv[0][2] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
    inv[1][0] = inv[0][1];
    inv[1][1] = m[0][0] * m[2][2] - m[0][2] * m[0][2];
    inv[1][2] = m[0][1] * m[0][2] - m[0][0] * m[1][2];
    inv[2][0] = inv[0][2];
    inv[2][1] = inv[1][2];
    inv[2][2] = m[0][0] * m[1][1] - m[0][1] * m[0][1];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) bx.inv[i][j] = inv[i][j] / md;
    return bx;
}

void host_unit_cells(const double *a, const double *b, const double *c, double rcut, int *indices) {
    auto cross = [](const double *x, const double *y, double *z) {
        z[0] = x[1] * y[2] - x[2] * y[1];
        z[1] = x[2] * y[0] - x[0] * y[2];
        z[2] = x[0] * y[1] - x[1] * y[0];
    };
    auto d3 = [](const double *x, const double *y) {
        double s = x[0] * y[0];
        s = s + x[1] * y[1];
        s = s + x[2] * y[2];
        return s;
    };
    double axb[3], cxa[3], bxc[3];
    cross(a, b, axb);
    cross(c, a, cxa);
    cross(b, c, bxc);
    const double n1 = sqrt(d3(axb, axb)), n2 = sqrt(d3(cxa, cxa)), n3 = sqrt(d3(bxc, bxc));
    for (int i = 0; i < 3; ++i) { axb[i] /= n1; cxa[i] /= n2; bxc[i] /= n3; }
    const double m[3][3] = {{d3(axb, a), d3(axb, b), d3(axb, c)},
                            {d3(cxa, a), d3(cxa, b), d3(cxa, c)},
                            {d3(bxc, a), d3(bxc, b), d3(bxc, c)}};
    const double md = -m[0][2] * m[1][1] * m[2][0] + m[0][1] * m[1][2] * m[2][0] +
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
        s = fabs(s);
        int k = (int)s;
        if (s > (double)k) k = k + 1;
        indices[i] = k;
    }
}

int NeighborList::reserve(int ns, int nsc, int64_t pair_cap, const CellGrid &g) {
    if (ns > n_alloc_sites) {
        dev_free(n_neigh); dev_free(pstart); dev_free(cell_xyz);
        TGB_TRY(dev_alloc(&n_neigh, ns));
        TGB_TRY(dev_alloc(&pstart, (size_t)ns + 1));
        TGB_TRY(dev_alloc(&cell_xyz, 3 * (size_t)ns));
        n_alloc_sites = ns;
        size_t need = 0;
        cub::DeviceScan::InclusiveSum(nullptr, need, n_neigh, pstart + 1, ns);
        if (need > scan_bytes) {
            dev_free(scan_tmp);
            TGB_TRY(dev_alloc(reinterpret_cast<char **>(&scan_tmp), need));
            scan_bytes = need;
        }
    }
    if (nsc > n_alloc_sc) {
        dev_free(cell_atoms);
        dev_free(cell_pos);
        TGB_TRY(dev_alloc(&cell_atoms, nsc));
        TGB_TRY(dev_alloc(&cell_pos, 3 * (size_t)nsc));
        n_alloc_sc = nsc;
    }
    const int64_t ncells = (int64_t)g.mx * g.my * g.mz;
    if (ncells > n_alloc_cells) {
        dev_free(cell_count); dev_free(cell_start); dev_free(cell_fill);
        TGB_TRY(dev_alloc(&cell_count, ncells));
        TGB_TRY(dev_alloc(&cell_start, ncells + 1));
        TGB_TRY(dev_alloc(&cell_fill, ncells));
        n_alloc_cells = ncells;
        size_t need = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, need, cell_count, cell_start, (int)ncells);
        if (need > scan_bytes) {
            dev_free(scan_tmp);
            TGB_TRY(dev_alloc(reinterpret_cast<char **>(&scan_tmp), need));
            scan_bytes = need;
        }
    }
    if (pair_cap > cap) {
        dev_free(nbr); dev_free(rjs); dev_free(xyz);
        dev_free(nsp);
        TGB_TRY(dev_alloc(&nbr, pair_cap));
        TGB_TRY(dev_alloc(&rjs, pair_cap));
        TGB_TRY(dev_alloc(&xyz, 3 * pair_cap));
        TGB_TRY(dev_alloc(&nsp, pair_cap));
        cap = pair_cap;
    }
    if (!err) TGB_TRY(dev_alloc(&err, 1));
    return TG_OK;
}

int NeighborList::reserve_slots(int ns, int s) {
    dev_free(snbr); dev_free(srjs); dev_free(sxyz);
    slots = 0;
    TGB_TRY(dev_alloc(&snbr, (size_t)ns * s));
    TGB_TRY(dev_alloc(&srjs, (size_t)ns * s));
    TGB_TRY(dev_alloc(&sxyz, (size_t)3 * ns * s));
    if (!ovf) TGB_TRY(dev_alloc(&ovf, 1));
    slots = s;
    return TG_OK;
}

void NeighborList::release() {
    dev_free(snbr); dev_free(srjs); dev_free(sxyz); dev_free(ovf);
    dev_free(n_neigh); dev_free(pstart); dev_free(cell_xyz); dev_free(cell_atoms);
    dev_free(cell_count); dev_free(cell_start); dev_free(cell_fill); dev_free(nbr);
    dev_free(rjs); dev_free(xyz); dev_free(scan_tmp); dev_free(err); dev_free(cell_pos);
    dev_free(nsp);
    *this = NeighborList{};
}

CellGrid plan_cells(const Box &bx, double rcut, const int *indices, bool *use_cells) {
    CellGrid g{1, 1, 1};
    const bool small = indices[0] > 1 || indices[1] > 1 || indices[2] > 1;
    *use_cells = bx.ortho && !small;
    if (*use_cells) {
        g.mx = (int)(bx.L[0] / rcut);
        g.my = (int)(bx.L[1] / rcut);
        g.mz = (int)(bx.L[2] / rcut);
        if (g.mx < 1 || g.my < 1 || g.mz < 1) *use_cells = false;
    }
    if (!*use_cells) g = CellGrid{1, 1, 1};
    return g;
}

namespace {

// build_neighbors_list with rebuild_neighbors_list = .false. (neighbors.f90:544-590):
// the pair list stays, every pair's MIC vector and distance are recomputed with
// get_distance from the current positions. Runs only while *when is zero.
__global__ void k_nl_refresh(int n_sites, const double *__restrict__ pos, Box bx,
                             const int64_t *__restrict__ pstart, int64_t cap,
                             const int *__restrict__ nbr, double *__restrict__ rjs,
                             double *__restrict__ xyz, const int *__restrict__ when) {
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n_sites || *when) return;
    const double *pi = pos + 3 * (size_t)i;
    // a list that overflowed its capacity holds pairs only below cap (the build
    // raised the capacity error, which the host reports after the step)
    const int64_t p0 = pstart[i], p1 = min(pstart[i + 1], cap);
    for (int64_t p = p0 + 1 + lane; p < p1; p += 32) {   // the self pair keeps its zeros
        double dist[3], d;
        get_distance(pi, pos + 3 * (size_t)nbr[p], bx, dist, &d);
        rjs[p] = d;
        xyz[3 * p] = dist[0];
        xyz[3 * p + 1] = dist[1];
        xyz[3 * p + 2] = dist[2];
    }
}

// After the list phase of an evaluation: a rebuilt list restarts the displacement
// accumulation (turbogap_md.f90:464-470 zeroes positions_diff when it decides to
// rebuild); counters[0] counts rebuilds, counters[1] evaluations.
__global__ void k_skin_reset(int n, const int *__restrict__ when, double *__restrict__ disp,
                             long long *__restrict__ counters) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool rebuilt = *when != 0;
    if (i == 0) {
        counters[1] += 1;
        if (rebuilt) counters[0] += 1;
    }
    if (i >= n || !rebuilt) return;
    disp[3 * (size_t)i] = 0.0;
    disp[3 * (size_t)i + 1] = 0.0;
    disp[3 * (size_t)i + 2] = 0.0;
}

// turbogap_md.f90:451-470: positions_diff += positions - positions_prev; the list
// is rebuilt before the next evaluation once some atom's squared displacement
// exceeds neighbors_buffer / 2 (the reference compares the square with half
// the buffer length).
__global__ void k_skin_check(int n, const double *__restrict__ pos,
                             const double *__restrict__ pos_prev, double *__restrict__ disp,
                             double thresh, int *__restrict__ when) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double v = (disp[3 * (size_t)i + q] + pos[3 * (size_t)i + q]) - pos_prev[3 * (size_t)i + q];
        disp[3 * (size_t)i + q] = v;
        s = s + v * v;
    }
    if (s > thresh) atomicOr(when, 1);
}

}  // namespace

namespace {
__global__ void k_pair_species(const int64_t *__restrict__ pend, int64_t cap,
                               const int *__restrict__ nbr, const int *__restrict__ species,
                               int n_atoms, signed char *__restrict__ nsp) {
    const int64_t P = min(*pend, cap);
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int j = nbr[p];
        nsp[p] = (signed char)species[j < n_atoms ? j : j % n_atoms];
    }
}
}  // namespace

int launch_pair_species(const int64_t *pend, int64_t cap, const int *nbr, const int *species,
                        int n_atoms, signed char *nsp, cudaStream_t st) {
    if (!nsp || cap <= 0 || n_atoms <= 0) return TG_OK;
    int dev = 0, n_sm = 0;
    TGB_CUDA(cudaGetDevice(&dev));
    TGB_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    const int64_t want = (cap + 255) / 256;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)n_sm * 16));
    k_pair_species<<<grid, 256, 0, st>>>(pend, cap, nbr, species, n_atoms, nsp);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

int launch_pair_species(int n_sites, const NeighborList &nl, const int *species, int n_atoms,
                        cudaStream_t st) {
    if (n_sites <= 0) return TG_OK;
    return launch_pair_species(nl.pstart + n_sites, nl.cap, nl.nbr, species, n_atoms, nl.nsp, st);
}

int launch_nl_refresh(int n_sites, const double *pos, const Box &bx, const NeighborList &nl,
                      const int *when, cudaStream_t st) {
    const int TB = 128;
    const int gw = (int)(((int64_t)n_sites * 32 + TB - 1) / TB);
    k_nl_refresh<<<gw, TB, 0, st>>>(n_sites, pos, bx, nl.pstart, nl.cap, nl.nbr, nl.rjs, nl.xyz,
                                    when);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

int launch_skin_reset(int n, const int *when, double *disp, long long *counters, cudaStream_t st) {
    k_skin_reset<<<(n + 255) / 256, 256, 0, st>>>(n, when, disp, counters);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

int launch_skin_check(int n, const double *pos, const double *pos_prev, double *disp, double thresh,
                      int *when, cudaStream_t st) {
    k_skin_check<<<(n + 255) / 256, 256, 0, st>>>(n, pos, pos_prev, disp, thresh, when);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

int nl_build(NeighborList &nl, int n_sites, int n_sc, const double *pos, const Box &bx,
             const CellGrid &g, bool use_cells, double rcut, const int *do_list,
             cudaStream_t st, const int *when) {
    TGB_CHECK(!when || use_cells, TG_ERR_ARG, "a gated list build needs the cell path");
    const int TB = 128;
    const int gb = (n_sites + TB - 1) / TB;
    const int gw = (int)(((int64_t)n_sites * 32 + TB - 1) / TB);   // one warp per site
    const bool one_pass = use_cells && nl.slots > 0 && nl.cap > 0;
    if (one_pass) TGB_CUDA(cudaMemsetAsync(nl.ovf, 0, sizeof(int), st));
    const int ncells = use_cells ? g.mx * g.my * g.mz : 0;
    const int gcell = ncells;   // one CTA per cell
    if (use_cells) {
        TGB_CUDA(cudaMemsetAsync(nl.cell_count, 0, sizeof(int) * ncells, st));
        TGB_CUDA(cudaMemsetAsync(nl.cell_fill, 0, sizeof(int) * ncells, st));
        k_cell_assign<<<gb, TB, 0, st>>>(n_sites, pos, bx, g, nl.cell_xyz, nl.cell_count, when);
        size_t bytes = nl.scan_bytes;
        TGB_CUDA(cub::DeviceScan::ExclusiveSum(nl.scan_tmp, bytes, nl.cell_count, nl.cell_start,
                                               ncells, st));
        k_cell_fill<<<gb, TB, 0, st>>>(n_sites, nl.cell_xyz, g, nl.cell_start, nl.cell_fill,
                                       nl.cell_atoms, when);
        k_cell_sort<<<(ncells + TB - 1) / TB, TB, 0, st>>>(ncells, nl.cell_start, nl.cell_count,
                                                           nl.cell_atoms, when);
        if (nl.cell_pos)
            k_cell_gather_pos<<<gb, TB, 0, st>>>(n_sites, nl.cell_atoms, pos, nl.cell_pos, when);
        k_nl_cells_cell<kNlCellWarps, kNlCellCap><<<gcell, 32 * kNlCellWarps, 0, st>>>(
            ncells, pos, bx, g, rcut, do_list, nl.cell_xyz, nl.cell_start, nl.cell_count,
            nl.cell_atoms, nl.cell_pos, nl.n_neigh, nullptr, nl.cap, one_pass ? nl.snbr : nullptr,
            one_pass ? nl.srjs : nullptr, one_pass ? nl.sxyz : nullptr, nl.err, when,
            one_pass ? nl.slots : 0, nl.ovf, nullptr);
    } else {
        k_nl_brute<<<gb, TB, 0, st>>>(n_sites, n_sc, pos, bx, rcut, do_list, nl.n_neigh, nullptr,
                                      nl.cap, nullptr, nullptr, nullptr, nl.err);
    }
    k_pstart_zero<<<1, 1, 0, st>>>(nl.pstart);
    size_t bytes = nl.scan_bytes;
    TGB_CUDA(cub::DeviceScan::InclusiveSum(nl.scan_tmp, bytes, nl.n_neigh, nl.pstart + 1, n_sites,
                                           st));
    if (use_cells) {
        if (one_pass)
            k_nl_compact<<<gw, TB, 0, st>>>(n_sites, nl.slots, nl.n_neigh, nl.pstart, nl.snbr,
                                            nl.srjs, nl.sxyz, nl.ovf, when, nl.cap, nl.nbr, nl.rjs,
                                            nl.xyz, nl.err);
        // the filling search: always in the two-pass build, after an overflow in the other
        k_nl_cells_cell<kNlCellWarps, kNlCellCap><<<gcell, 32 * kNlCellWarps, 0, st>>>(
            ncells, pos, bx, g, rcut, do_list, nl.cell_xyz, nl.cell_start, nl.cell_count,
            nl.cell_atoms, nl.cell_pos, nl.n_neigh, nl.pstart, nl.cap, nl.nbr, nl.rjs, nl.xyz,
            nl.err, when, 0, nullptr, one_pass ? nl.ovf : nullptr);
    } else {
        k_nl_brute<<<gb, TB, 0, st>>>(n_sites, n_sc, pos, bx, rcut, do_list, nl.n_neigh, nl.pstart,
                                      nl.cap, nl.nbr, nl.rjs, nl.xyz, nl.err);
    }
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

// ---------------------------------------------------------------- batches
int batch_plan_struct(BatchStruct &b, double rcut) {
    bool cells = true;
    for (int k = 0; k < 3; ++k) {
        b.m[k] = (int)(b.L[k] / rcut);
        if (b.m[k] < 3) cells = false;
        // images reaching within rcut of a minimum-image vector (|v| <= L / 2)
        b.img[k] = (int)((rcut + 0.5 * b.L[k]) / b.L[k]);
    }
    b.mode = cells ? 0 : 1;
    if (!cells) b.m[0] = b.m[1] = b.m[2] = 0;
    return cells ? b.m[0] * b.m[1] * b.m[2] : 0;
}

namespace {

__device__ __forceinline__ void batch_cell(const BatchStruct &b, const double *p, int *c) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double x = p[k] - b.L[k] * floor(p[k] / b.L[k]);   // into [0, L)
        int ck = (int)(x / b.L[k] * b.m[k]);
        c[k] = ck < 0 ? 0 : (ck >= b.m[k] ? b.m[k] - 1 : ck);
    }
}

__global__ void k_bcell_assign(int n, const double *__restrict__ pos,
                               const BatchStruct *__restrict__ st, const int *__restrict__ atom_struct,
                               int *__restrict__ cell_id, int *__restrict__ cell_count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const BatchStruct b = st[atom_struct[i]];
    if (b.mode != 0) {
        cell_id[i] = -1;
        return;
    }
    int c[3];
    batch_cell(b, pos + 3 * (size_t)i, c);
    const int id = b.coff + (c[0] * b.m[1] + c[1]) * b.m[2] + c[2];
    cell_id[i] = id;
    atomicAdd(&cell_count[id], 1);
}

__global__ void k_bcell_fill(int n, const int *__restrict__ cell_id,
                             const int *__restrict__ cell_start, int *__restrict__ cell_fill,
                             int *__restrict__ cell_atoms) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int id = cell_id[i];
    if (id < 0) return;
    cell_atoms[cell_start[id] + atomicAdd(&cell_fill[id], 1)] = i;
}

// ascending atom order inside each cell (a deterministic pair order)
__global__ void k_bcell_sort(int ncells, const int *__restrict__ cell_start,
                             const int *__restrict__ cell_count, int *__restrict__ cell_atoms) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int *a = cell_atoms + cell_start[c];
    const int n = cell_count[c];
    for (int i = 1; i < n; ++i) {
        const int v = a[i];
        int j = i - 1;
        while (j >= 0 && a[j] > v) {
            a[j + 1] = a[j];
            --j;
        }
        a[j + 1] = v;
    }
}

// One warp per atom. Candidates form one flattened sequence (the 27 cells around
// the atom's cell, or (image, atom) pairs of the structure); lanes test 32 at a
// time and emit accepted pairs in sequence order (ballot + prefix popcount).
// Count mode when pstart is null.
// Three uses: count (pstart and slots unset), count into slot rows (slots > 0:
// pair e of atom i at row i * slots + e while e < slots, *ovf set past it), and
// fill the compact arrays at pstart (run only when *gate is set, if gate given).
// With skip_cells set it lists only the atoms of image structures; k_bnl_cell
// lists those of the cell structures.
__global__ void k_bnl_warp(int n, const double *__restrict__ pos, const BatchStruct *__restrict__ st,
                           const int *__restrict__ atom_struct, const int *__restrict__ cell_id,
                           const int *__restrict__ cell_start, const int *__restrict__ cell_count,
                           const int *__restrict__ cell_atoms, const double *__restrict__ cell_pos,
                           double rcut, int *__restrict__ n_neigh,
                           const int64_t *__restrict__ pstart, int64_t cap, int *__restrict__ nbr,
                           double *__restrict__ xyz, unsigned *err, int slots,
                           int *__restrict__ ovf, const int *__restrict__ gate, int skip_cells) {
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n || (gate && !*gate)) return;
    // where pair e goes, and whether it fits
    const bool slotted = !pstart && slots > 0;
    const bool writes = pstart || slotted;
    const BatchStruct b = st[atom_struct[i]];
    if (skip_cells && b.mode == 0) return;   // k_bnl_cell lists the atoms of cell structures
    const double pi[3] = {pos[3 * (size_t)i], pos[3 * (size_t)i + 1], pos[3 * (size_t)i + 2]};
    const double invL[3] = {1.0 / b.L[0], 1.0 / b.L[1], 1.0 / b.L[2]};
    // candidate segments: lane c < 27 describes cell c (mode 0); mode 1 has one
    // segment per image
    const int nimg = (2 * b.img[0] + 1) * (2 * b.img[1] + 1) * (2 * b.img[2] + 1);
    int cstart = 0, ccount = 0;
    if (b.mode == 0) {
        if (lane < 27) {
            const int ci = cell_id[i] - b.coff;
            const int cx = ci / (b.m[1] * b.m[2]), cy = (ci / b.m[2]) % b.m[1], cz = ci % b.m[2];
            const int x = (cx + lane / 9 - 1 + b.m[0]) % b.m[0];
            const int y = (cy + (lane / 3) % 3 - 1 + b.m[1]) % b.m[1];
            const int z = (cz + lane % 3 - 1 + b.m[2]) % b.m[2];
            const int c = b.coff + (x * b.m[1] + y) * b.m[2] + z;
            cstart = cell_start[c];
            ccount = cell_count[c];
        }
    }
    int incl = ccount;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = b.mode == 0 ? __shfl_sync(0xffffffffu, incl, 31) : b.n * nimg;
    const int64_t base = pstart ? pstart[i] : (slotted ? (int64_t)i * slots : 0);
    const int64_t lim = pstart ? cap : base + slots;
    if (writes && lane == 0) {   // self pair first
        if (base < lim) {
            nbr[base] = i;
            xyz[3 * base] = 0.0;
            xyz[3 * base + 1] = 0.0;
            xyz[3 * base + 2] = 0.0;
        } else {
            atomicOr(err, (unsigned)DEV_ERR_NEIGH_CAPACITY);
        }
    }
    int count = 1;
    for (int f0 = 0; f0 < total; f0 += 32) {   // warp-uniform trip count
        const int f = f0 + lane;
        const int fc = f < total ? f : total - 1;
        int k = -1, slot = -1;
        int t[3] = {0, 0, 0};
        if (b.mode == 0) {
            int c = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const int probe = c + step - 1;
                const int v = __shfl_sync(0xffffffffu, incl, probe < 31 ? probe : 31);
                if (probe < 27 && v <= fc) c += step;
            }
            const int cs = __shfl_sync(0xffffffffu, cstart, c);
            const int before = __shfl_sync(0xffffffffu, incl, c) - __shfl_sync(0xffffffffu, ccount, c);
            if (f < total) {
                slot = cs + (fc - before);
                k = cell_atoms[slot];
            }
        } else if (f < total) {
            const int im = fc / b.n;
            k = b.off + (fc - im * b.n);
            const int ny = 2 * b.img[1] + 1, nz = 2 * b.img[2] + 1;
            t[0] = im / (ny * nz) - b.img[0];
            t[1] = (im / nz) % ny - b.img[1];
            t[2] = im % nz - b.img[2];
        }
        bool take = false;
        double dist[3] = {0.0, 0.0, 0.0};
        if (k >= 0) {
            const double *pk = slot >= 0 ? cell_pos + 3 * (size_t)slot : pos + 3 * (size_t)k;
            double d2 = 0.0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                double v = pk[q] - pi[q];
                // minimum image, by the reciprocal: rint differs from that of the
                // quotient only within an ulp of |v| = L / 2, a tie between two
                // images at the same distance
                v -= b.L[q] * rint(v * invL[q]);
                v += t[q] * b.L[q];
                dist[q] = v;
                d2 += v * v;
            }
            const bool self = k == i && t[0] == 0 && t[1] == 0 && t[2] == 0;
            take = !self && d2 < rcut * rcut;
        }
        const unsigned msk = __ballot_sync(0xffffffffu, take);
        if (writes && take) {
            const int64_t p = base + count + __popc(msk & ((1u << lane) - 1u));
            if (p < lim) {
                nbr[p] = k;
                xyz[3 * p] = dist[0];
                xyz[3 * p + 1] = dist[1];
                xyz[3 * p + 2] = dist[2];
            } else if (slotted) {
                *ovf = 1;   // the fallback search fills this build
            } else {
                atomicOr(err, (unsigned)DEV_ERR_NEIGH_CAPACITY);
            }
        }
        count += __popc(msk);
    }
    if (!pstart && lane == 0) n_neigh[i] = count;
}

// The cell structures' atoms by cell: one CTA per cell stages the candidates of
// the cell's 27-cell neighbourhood (the walk order of k_bnl_warp) in shared memory,
// CAP at a time, and warp w lists the cell's atoms w, w + WARPS, ... from there,
// with the tests and the three uses of k_bnl_warp.
template <int WARPS, int CAP>
__global__ void __launch_bounds__(32 * WARPS)
    k_bnl_cell(int n_cells, const double *__restrict__ pos, const BatchStruct *__restrict__ st,
               const int *__restrict__ atom_struct, const int *__restrict__ cell_start,
               const int *__restrict__ cell_count, const int *__restrict__ cell_atoms,
               const double *__restrict__ cell_pos, double rcut, int *__restrict__ n_neigh,
               const int64_t *__restrict__ pstart, int64_t cap, int *__restrict__ nbr,
               double *__restrict__ xyz, unsigned *err, int slots, int *__restrict__ ovf,
               const int *__restrict__ gate) {
    __shared__ double sx[CAP], sy[CAP], sz[CAP];
    __shared__ int sk[CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int cell = blockIdx.x;   // every exit before the loop is CTA-uniform
    if (cell >= n_cells || (gate && !*gate)) return;
    const int na = cell_count[cell];
    if (na == 0) return;
    const int c0 = cell_start[cell];
    const bool slotted = !pstart && slots > 0;
    const bool writes = pstart || slotted;
    const BatchStruct b = st[atom_struct[cell_atoms[c0]]];
    const double invL[3] = {1.0 / b.L[0], 1.0 / b.L[1], 1.0 / b.L[2]};
    CellWalk cw{0, 0, 0, 0};
    if (lane < 27) {
        const int ci = cell - b.coff;
        const int cx = ci / (b.m[1] * b.m[2]), cy = (ci / b.m[2]) % b.m[1], cz = ci % b.m[2];
        const int x = (cx + lane / 9 - 1 + b.m[0]) % b.m[0];
        const int y = (cy + (lane / 3) % 3 - 1 + b.m[1]) % b.m[1];
        const int z = (cz + lane % 3 - 1 + b.m[2]) % b.m[2];
        const int c = b.coff + (x * b.m[1] + y) * b.m[2] + z;
        cw.cstart = cell_start[c];
        cw.ccount = cell_count[c];
    }
    cw.scan(lane);
    const int total = cw.total;
    const int nround = (total + CAP - 1) / CAP;
    const double rc2 = rcut * rcut;
    if (nround == 1) {
        stage_candidates<WARPS>(cw, 0, total, w, lane, cell_atoms, cell_pos, pos, sk, sx, sy, sz);
        __syncthreads();
    }
    for (int ag = 0; ag < na; ag += WARPS) {   // CTA-uniform trip count
        const int a = ag + w;
        const int i = a < na ? cell_atoms[c0 + a] : -1;   // warp-uniform
        double pi[3] = {0.0, 0.0, 0.0};
        int64_t base = 0, lim = 0;
        if (i >= 0) {
            pi[0] = pos[3 * (size_t)i];
            pi[1] = pos[3 * (size_t)i + 1];
            pi[2] = pos[3 * (size_t)i + 2];
            base = pstart ? pstart[i] : (slotted ? (int64_t)i * slots : 0);
            lim = pstart ? cap : base + slots;
            if (writes && lane == 0) {   // self pair first
                if (base < lim) {
                    nbr[base] = i;
                    xyz[3 * base] = 0.0;
                    xyz[3 * base + 1] = 0.0;
                    xyz[3 * base + 2] = 0.0;
                } else {
                    atomicOr(err, (unsigned)DEV_ERR_NEIGH_CAPACITY);
                }
            }
        }
        int count = 1;
        for (int r = 0; r < nround; ++r) {   // CTA-uniform trip count
            const int f_beg = r * CAP, f_end = min(total, f_beg + CAP);
            if (nround > 1) {   // a large neighbourhood: staged again, round by round
                __syncthreads();   // every warp is done with the previous round
                stage_candidates<WARPS>(cw, f_beg, f_end, w, lane, cell_atoms, cell_pos, pos, sk, sx,
                                        sy, sz);
                __syncthreads();
            }
            if (i < 0) continue;
            for (int f0 = f_beg; f0 < f_end; f0 += 32) {   // warp-uniform trip count
                const int f = f0 + lane;
                bool take = false;
                int k = -1;
                double dist[3] = {0.0, 0.0, 0.0};
                if (f < f_end) {
                    k = sk[f - f_beg];
                    const double pk[3] = {sx[f - f_beg], sy[f - f_beg], sz[f - f_beg]};
                    double d2 = 0.0;
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        double v = pk[q] - pi[q];
                        v -= b.L[q] * rint(v * invL[q]);   // minimum image, as in k_bnl_warp
                        dist[q] = v;
                        d2 += v * v;
                    }
                    take = k != i && d2 < rc2;
                }
                const unsigned msk = __ballot_sync(0xffffffffu, take);
                if (writes && take) {
                    const int64_t p = base + count + __popc(msk & ((1u << lane) - 1u));
                    if (p < lim) {
                        nbr[p] = k;
                        xyz[3 * p] = dist[0];
                        xyz[3 * p + 1] = dist[1];
                        xyz[3 * p + 2] = dist[2];
                    } else if (slotted) {
                        *ovf = 1;   // the fallback search fills this build
                    } else {
                        atomicOr(err, (unsigned)DEV_ERR_NEIGH_CAPACITY);
                    }
                }
                count += __popc(msk);
            }
        }
        if (i >= 0 && !pstart && lane == 0) n_neigh[i] = count;
    }
}

// Slot rows to the compact arrays (a warp per atom), unless a row overflowed.
__global__ void k_bnl_compact(int n, int slots, const int *__restrict__ n_neigh,
                              const int64_t *__restrict__ pstart, const int *__restrict__ snbr,
                              const double *__restrict__ sxyz, const int *__restrict__ ovf,
                              int64_t cap, int *__restrict__ nbr, double *__restrict__ xyz,
                              unsigned *err) {
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n || *ovf) return;
    const int cnt = n_neigh[i];
    const int64_t dst = pstart[i], src = (int64_t)i * slots;
    if (dst + cnt > cap) {
        if (lane == 0) atomicOr(err, (unsigned)DEV_ERR_NEIGH_CAPACITY);
        return;
    }
    for (int e = lane; e < cnt; e += 32) nbr[dst + e] = snbr[src + e];
    for (int e = lane; e < 3 * cnt; e += 32) xyz[3 * dst + e] = sxyz[3 * src + e];
}

}  // namespace

int batch_nl_build(BatchNL &nl, const double *pos, double rcut, cudaStream_t st) {
    const int TB = 128, n = nl.n_atoms;
    const int gb = (n + TB - 1) / TB;
    const int gw = (int)(((int64_t)n * 32 + TB - 1) / TB);
    if (nl.n_cells > 0) {
        TGB_CUDA(cudaMemsetAsync(nl.cell_count, 0, sizeof(int) * nl.n_cells, st));
        TGB_CUDA(cudaMemsetAsync(nl.cell_fill, 0, sizeof(int) * nl.n_cells, st));
    }
    k_bcell_assign<<<gb, TB, 0, st>>>(n, pos, nl.st, nl.atom_struct, nl.cell_id, nl.cell_count);
    if (nl.n_cells > 0) {
        size_t bytes = nl.scan_bytes;
        TGB_CUDA(cub::DeviceScan::ExclusiveSum(nl.scan_tmp, bytes, nl.cell_count, nl.cell_start,
                                               nl.n_cells, st));
        k_bcell_fill<<<gb, TB, 0, st>>>(n, nl.cell_id, nl.cell_start, nl.cell_fill, nl.cell_atoms);
        k_bcell_sort<<<(nl.n_cells + TB - 1) / TB, TB, 0, st>>>(nl.n_cells, nl.cell_start,
                                                                 nl.cell_count, nl.cell_atoms);
        k_cell_gather_pos<<<gb, TB, 0, st>>>(nl.n_cell_atoms, nl.cell_atoms, pos, nl.cell_pos, nullptr);
    }
    const bool one_pass = nl.slots > 0 && nl.cap > 0;
    if (one_pass) TGB_CUDA(cudaMemsetAsync(nl.ovf, 0, sizeof(int), st));
    // atoms of cell structures by cell, the others (images) by atom
    const int gcell = nl.n_cells;   // one CTA per cell
    if (nl.n_cells > 0)
        k_bnl_cell<kNlCellWarps, kNlCellCap><<<gcell, 32 * kNlCellWarps, 0, st>>>(
            nl.n_cells, pos, nl.st, nl.atom_struct, nl.cell_start, nl.cell_count, nl.cell_atoms,
            nl.cell_pos, rcut, nl.n_neigh, nullptr, nl.cap, one_pass ? nl.snbr : nullptr,
            one_pass ? nl.sxyz : nullptr, nl.err, one_pass ? nl.slots : 0, nl.ovf, nullptr);
    k_bnl_warp<<<gw, TB, 0, st>>>(n, pos, nl.st, nl.atom_struct, nl.cell_id, nl.cell_start,
                                  nl.cell_count, nl.cell_atoms, nl.cell_pos, rcut, nl.n_neigh,
                                  nullptr, nl.cap, one_pass ? nl.snbr : nullptr,
                                  one_pass ? nl.sxyz : nullptr, nl.err, one_pass ? nl.slots : 0,
                                  nl.ovf, nullptr, nl.n_cells > 0);
    k_pstart_zero<<<1, 1, 0, st>>>(nl.pstart);
    size_t bytes = nl.scan_bytes;
    TGB_CUDA(cub::DeviceScan::InclusiveSum(nl.scan_tmp, bytes, nl.n_neigh, nl.pstart + 1, n, st));
    if (one_pass)
        k_bnl_compact<<<gw, TB, 0, st>>>(n, nl.slots, nl.n_neigh, nl.pstart, nl.snbr, nl.sxyz,
                                         nl.ovf, nl.cap, nl.nbr, nl.xyz, nl.err);
    // the filling search: always in the two-pass build, after an overflow in the other
    if (nl.n_cells > 0)
        k_bnl_cell<kNlCellWarps, kNlCellCap><<<gcell, 32 * kNlCellWarps, 0, st>>>(
            nl.n_cells, pos, nl.st, nl.atom_struct, nl.cell_start, nl.cell_count, nl.cell_atoms,
            nl.cell_pos, rcut, nl.n_neigh, nl.pstart, nl.cap, nl.nbr, nl.xyz, nl.err, 0, nullptr,
            one_pass ? nl.ovf : nullptr);
    k_bnl_warp<<<gw, TB, 0, st>>>(n, pos, nl.st, nl.atom_struct, nl.cell_id, nl.cell_start,
                                  nl.cell_count, nl.cell_atoms, nl.cell_pos, rcut, nl.n_neigh,
                                  nl.pstart, nl.cap, nl.nbr, nl.xyz, nl.err, 0, nullptr,
                                  one_pass ? nl.ovf : nullptr, nl.n_cells > 0);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

int launch_angles(int64_t P, const double *rjs, const double *xyz, const int *is_self, double *th,
                  double *ph, cudaStream_t st) {
    if (P == 0) return TG_OK;
    k_angles<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(P, rjs, xyz, is_self, th, ph);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

int launch_supercell(int n, const double *pos, const double *abc_dev, const int *indices,
                     double *out, cudaStream_t st) {
    const int tot = n * indices[0] * indices[1] * indices[2];
    k_supercell<<<(tot + 255) / 256, 256, 0, st>>>(n, pos, abc_dev, abc_dev + 3, abc_dev + 6,
                                                   indices[0], indices[1], indices[2], out);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

int launch_velocity_verlet(int n, double *pos, double *pos_prev, double *vel, const double *f,
                           double *f_prev, const double *m, double dt, double dt_prev, int first,
                           cudaStream_t st) {
    k_velocity_verlet<<<(3 * n + 255) / 256, 256, 0, st>>>(n, pos, pos_prev, vel, f, f_prev, m, dt,
                                                           dt_prev, first);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

int launch_wrap(int n, double *pos, const Box &bx, cudaStream_t st) {
    if (bx.ortho) k_wrap_ortho<<<(n + 255) / 256, 256, 0, st>>>(n, pos, bx);
    else k_wrap_tri<<<(n + 255) / 256, 256, 0, st>>>(n, pos, bx);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

int launch_remove_cm(int n, double *vel, const double *m, double *acc4, cudaStream_t st) {
    TGB_CUDA(cudaMemsetAsync(acc4, 0, 4 * sizeof(double), st));
    k_cm_accumulate<<<148, 256, 0, st>>>(n, vel, m, acc4);
    k_cm_apply<<<(3 * n + 255) / 256, 256, 0, st>>>(n, vel, acc4);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

int launch_kinetic(int n, const double *vel, const double *m, double *acc, cudaStream_t st) {
    TGB_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), st));
    k_kinetic<<<148, 256, 0, st>>>(n, vel, m, acc);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

}  // namespace tgb
