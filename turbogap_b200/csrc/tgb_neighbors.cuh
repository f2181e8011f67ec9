// tgb_neighbors.cuh -- neighbour-list and FP64 MD kernel interfaces.
#pragma once

#include "tgb_common.cuh"

namespace tgb {

template <class T>
int dev_alloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), n * sizeof(T));
    if (e != cudaSuccess) {
        set_error("cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
        *p = nullptr;
        return TG_ERR_NOMEM;
    }
    return TG_OK;
}

template <class T>
void dev_free(T *&p) {
    if (p) cudaFree(reinterpret_cast<void *>(p));
    p = nullptr;
}

// Simulation box (rows a, b, c). ortho: the reference's orthorhombic test
// (neighbors.f90:85-88, tolerance 1e-6 on the off-diagonal components).
struct Box {
    double a[3], b[3], c[3];
    double L[3];
    double inv[3][3];
    int ortho;
};

struct CellGrid {
    int mx, my, mz;
};

// Pairs in CSR order: site i owns [pstart[i], pstart[i+1]); the first pair of
// every site is the site itself (rjs = 0, xyz = 0). nbr holds 0-based
// supercell indices.
struct NeighborList {
    int n_alloc_sites = 0, n_alloc_sc = 0;
    int64_t n_alloc_cells = 0;
    int64_t cap = 0;
    int *n_neigh = nullptr;
    int64_t *pstart = nullptr;
    int *cell_xyz = nullptr;
    int *cell_atoms = nullptr;
    int *cell_count = nullptr;
    int *cell_start = nullptr;
    int *cell_fill = nullptr;
    int *nbr = nullptr;
    double *rjs = nullptr;
    double *xyz = nullptr;
    double *cell_pos = nullptr;   // optional: positions in cell order (coalesced candidate reads)
    // global species id of each pair's neighbour (launch_pair_species), so the
    // SOAP passes stream it instead of gathering species[neighbour]
    signed char *nsp = nullptr;
    void *scan_tmp = nullptr;
    size_t scan_bytes = 0;
    unsigned *err = nullptr;
    // One search pass on the cell path (as in the batched build): with slots > 0
    // and cap > 0 the search writes each site's pairs into fixed rows while it
    // counts them, a copy compacts the rows after the scan, and a site with more
    // than slots pairs sets *ovf, which sends the build to the filling search.
    int slots = 0;
    int *snbr = nullptr;
    double *srjs = nullptr, *sxyz = nullptr;
    int *ovf = nullptr;

    int reserve(int n_sites, int n_sc, int64_t pair_cap, const CellGrid &g);
    int reserve_slots(int n_sites, int slots);
    void release();
};

Box make_box(const double *a, const double *b, const double *c);

// number_of_unit_cells_for_given_cutoff (neighbors.f90:175-236), on the host.
void host_unit_cells(const double *a, const double *b, const double *c, double rcut, int *indices);
CellGrid plan_cells(const Box &bx, double rcut, const int *indices, bool *use_cells);

// Count, scan and fill. Pairs beyond nl.cap are dropped and flag
// DEV_ERR_NEIGH_CAPACITY; pstart[n_sites] is the required capacity.
// when (device int, optional, cell path only): the list kernels run only while
// it is nonzero, so a captured step can skip the rebuild on the device.
int nl_build(NeighborList &nl, int n_sites, int n_sc, const double *pos, const Box &bx,
             const CellGrid &g, bool use_cells, double rcut, const int *do_list,
             cudaStream_t st, const int *when = nullptr);

// Verlet-skin lists (neighbors_buffer > 0, turbogap_md.f90:451-470,
// neighbors.f90:544-590): refresh distances of the kept pairs while *when is 0;
// after the list phase restart the displacement sums if the list was rebuilt;
// after the integrator raise *when once |displacement|^2 > thresh.
// nsp[p] = species[neighbour of pair p mod n_atoms] for every pair of the list
// (the pair count read on the device from pstart[n_sites], capped at nl.cap).
int launch_pair_species(int n_sites, const NeighborList &nl, const int *species, int n_atoms,
                        cudaStream_t st);
// The same over raw arrays: pend = &pstart[n_sites] (the pair count), cap pairs at most.
int launch_pair_species(const int64_t *pend, int64_t cap, const int *nbr, const int *species,
                        int n_atoms, signed char *nsp, cudaStream_t st);

int launch_nl_refresh(int n_sites, const double *pos, const Box &bx, const NeighborList &nl,
                      const int *when, cudaStream_t st);
int launch_skin_reset(int n, const int *when, double *disp, long long *counters, cudaStream_t st);
int launch_skin_check(int n, const double *pos, const double *pos_prev, double *disp, double thresh,
                      int *when, cudaStream_t st);

// ---- many independent orthorhombic structures at once (batched evaluation).
// Structure s owns atoms [off, off + n) of the concatenated arrays. Boxes of at
// least 3 rcut on every axis use a cell grid of >= 3 cells per axis (minimum
// image); smaller boxes enumerate all atoms of the structure over the periodic
// images within reach (img[k] per axis). Pairs: self first, then the accepted
// candidates; nbr holds global atom indices (no supercell).
struct BatchStruct {
    int off, n;
    double L[3];
    int mode;        // 0: cells, 1: images
    int m[3];        // cells per axis (mode 0)
    int coff;        // first global cell (mode 0)
    int img[3];      // image range per axis (mode 1)
};

// Host-side plan of one structure (cells or images, counts); returns the cells used.
int batch_plan_struct(BatchStruct &b, double rcut);

struct BatchNL {
    int n_atoms = 0, n_structs = 0, n_cells = 0;
    int n_cell_atoms = 0;          // atoms of the structures that use cells
    int64_t cap = 0;
    BatchStruct *st = nullptr;     // device [n_structs]
    int *atom_struct = nullptr;    // device [n_atoms]
    int *cell_id = nullptr, *cell_count = nullptr, *cell_start = nullptr, *cell_fill = nullptr;
    int *cell_atoms = nullptr;
    double *cell_pos = nullptr;    // [n_atoms * 3] positions in cell order
    int *n_neigh = nullptr;
    int64_t *pstart = nullptr;
    int *nbr = nullptr;
    double *xyz = nullptr;
    void *scan_tmp = nullptr;
    size_t scan_bytes = 0;
    unsigned *err = nullptr;
    // One-pass build: with slots > 0 (and pair arrays, cap > 0) the search writes
    // each atom's pairs into slots fixed-size rows of snbr / sxyz while it counts
    // them, and a copy compacts the rows after the scan. An atom with more than
    // slots pairs sets *ovf, and the build then falls back to a second search
    // that fills the compact arrays directly; no host round trip either way.
    int slots = 0;
    int *snbr = nullptr;           // [n_atoms * slots]
    double *sxyz = nullptr;        // [n_atoms * slots * 3]
    int *ovf = nullptr;
};

// Count, scan and fill (pairs beyond nl.cap are dropped and flag DEV_ERR_NEIGH_CAPACITY;
// pstart[n_atoms] is the required capacity).
int batch_nl_build(BatchNL &nl, const double *pos, double rcut, cudaStream_t st);

int launch_angles(int64_t P, const double *rjs, const double *xyz, const int *is_self, double *th,
                  double *ph, cudaStream_t st);
int launch_supercell(int n, const double *pos, const double *abc_dev, const int *indices,
                     double *out, cudaStream_t st);
int launch_velocity_verlet(int n, double *pos, double *pos_prev, double *vel, const double *f,
                           double *f_prev, const double *m, double dt, double dt_prev, int first,
                           cudaStream_t st);
int launch_wrap(int n, double *pos, const Box &bx, cudaStream_t st);
int launch_remove_cm(int n, double *vel, const double *m, double *acc4, cudaStream_t st);
int launch_kinetic(int n, const double *vel, const double *m, double *acc, cudaStream_t st);

}  // namespace tgb
