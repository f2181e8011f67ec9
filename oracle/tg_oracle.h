/*
 * tg_oracle.h -- FP64 CPU restatement of the TurboGAP SOAP-GAP energy/force path.
 *
 * TEST INFRASTRUCTURE ONLY. The oracle is the checker for the CUDA backend in
 * turbogap_b200/; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load it. Nothing in the product path links or calls it.
 *
 * Parity status
 *   - neighbour lists, MIC geometry, supercell build, get_gap_soap remap, the GAP
 *     kernel/forces/virial and velocity-Verlet are restated line for line from the
 *     reference Fortran (citations at each function below);
 *   - the SOAP descriptor itself lives in the soap_turbo submodule, which is not
 *     shipped with the reference (src/soap_turbo/ is empty; pinned upstream is
 *     TiganyZ/soap_turbo @ df92bda21f48ec0e0031c096eb3d48bf1d7b89d8, branch
 *     "cleanup"). It is restated here from the published method (Caro, PRB 100,
 *     024112 (2019); Bartok et al., PRB 87, 184115 (2013)) under the conventions
 *     the reference pins at its call site (gap_interface.f90:312-325). No golden
 *     vectors for the descriptor exist in the reference tree, so descriptor
 *     values are PARITY UNPINNED; the descriptor's building blocks are pinned
 *     against independent implementations (scipy special functions and
 *     quadrature) and the whole path against finite differences (the
 *     tests/fd_gap methodology of the reference).
 *
 * Conventions: Fortran layout. Arrays named (3, n) are column-major with the 3
 * fastest; neighbour indices are 1-based supercell indices exactly as
 * build_neighbors_list returns them.
 */
#ifndef TG_ORACLE_H
#define TG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Hyperparameters of one soap_turbo block (types.f90:75-134). Per-species
 * arrays have n_species entries; species_z[s] is the global species id (the
 * 1-based position in the input's species_types list) of descriptor species s. */
typedef struct {
    int n_species;
    int l_max;
    int radial_enhancement;   /* 0..2 (read_files.f90:4800-4807)            */
    int central_species;      /* 1-based descriptor species index, 0 = all  */
    const int *alpha_max;     /* radial functions per species                */
    const int *species_z;
    const double *rcut_hard;
    const double *rcut_soft;  /* already converted: rcut_hard - buffer       */
    const double *nf;
    const double *global_scaling;
    const double *atom_sigma_r;
    const double *atom_sigma_r_scaling;
    const double *atom_sigma_t;
    const double *atom_sigma_t_scaling;
    const double *amplitude_scaling;
    const double *central_weight;
    /* SOAP compression (types.f90:92-110 compress_P_*, filled at
     * read_files.f90:5166-5231). compress_nonzero = 0: uncompressed. Otherwise
     * the descriptor has compress_dim components, q_c(i) = sum over entries k
     * with compress_i[k] = i of compress_el[k] * p(compress_j[k]) (1-based; j
     * in the uncompressed order n <= n', l), and q_c is normalised after the map
     * (parity unpinned: soap_turbo is absent). */
    int compress_dim;
    int compress_nonzero;
    const int *compress_i;
    const int *compress_j;
    const double *compress_el;
} orc_soap_hypers;

/* ---- geometry: neighbors.f90 ------------------------------------------- */
void orc_get_distance(const double *posi, const double *posj, const double *a,
                      const double *b, const double *c, double *dist, double *d,
                      int *i_shift);
void orc_number_of_unit_cells(const double *a, const double *b, const double *c,
                              double rcut, int *indices);
/* Supercell replication (read_files.f90:320-380). positions(3, n_sites) in,
 * out(3, n_sites*prod(indices)); species likewise. a,b,c are the primitive box. */
void orc_make_supercell(int n_sites, const double *positions, const int *species,
                        const double *a, const double *b, const double *c,
                        const int *indices, double *positions_sc, int *species_sc);
/* build_neighbors_list (neighbors.f90:243-605). a,b,c: the (super)cell box.
 * Returns the number of pairs, or -(needed pairs) if cap is too small. */
int64_t orc_build_neighbors_list(int n_sites_supercell, const double *positions,
                                 int n_sites, double *a, double *b, double *c,
                                 double rcut_max, const int *indices,
                                 const int *species_supercell, const int *do_list,
                                 int64_t cap, int *n_neigh, int *neighbors_list,
                                 double *rjs, double *thetas, double *phis,
                                 double *xyz, int *neighbor_species);

/* ---- descriptor building blocks ----------------------------------------- */
int orc_soap_dim(const orc_soap_hypers *h);
int orc_soap_n_tot(const orc_soap_hypers *h);
/* W = S^{-1/2} of the poly3 overlap for alpha_max functions (row-major). */
void orc_poly3_W(int alpha_max, double *W);
/* Radial channel functions of one species at distance r: R_n (w folded in)
 * and dR_n/dr, n = 0..alpha_max-1. self_pair=1 evaluates the central atom. */
void orc_radial(const orc_soap_hypers *h, int s, double r, int self_pair,
                double *R, double *dR);
/* Angular factors a_l(r) = 4 pi exp(-k) i_l(k), k = r^2/sigma_t(r)^2, and d/dr. */
void orc_angular(const orc_soap_hypers *h, int s, double r, double *a, double *da);
/* Real orthonormal spherical harmonics Y_lm(u) for unit u, index l*l+l+m, and
 * the gradient of the polynomial extension (3 per entry), may be NULL. */
void orc_real_ylm(int l_max, const double *u, double *Y, double *dY);

/* get_soap (soap_turbo; called at gap_interface.f90:320-325).
 * n_neigh(n_sites), per pair: rjs, xyz(3,P), mask(P, n_species) column-major as
 * logical (int), self pair first in each list. soap(dim, n_sites) out;
 * soap_cart_der(3, dim, P) out when not NULL. Also returns |p| per site. */
void orc_get_soap(const orc_soap_hypers *h, int n_sites, const int *n_neigh,
                  int n_pairs, const int *mask, const double *rjs,
                  const double *xyz, double *soap, double *soap_cart_der,
                  double *sqrt_dot_p);

/* ---- GAP prediction: gap.f90:66-259 -------------------------------------- */
void orc_soap_energy_and_forces(int n_soap, int n_sites, const double *soap,
                                const double *soap_der, int n_sparse,
                                const double *Qs, const double *alphas,
                                double delta, double zeta0, double e0,
                                const int *n_neigh, const int *neighbors_list,
                                const double *xyz, int n_sites0, int do_forces,
                                double *energies, double *forces, double *virial);

/* ---- get_gap_soap: gap_interface.f90:41-480 ------------------------------- *
 * n_total_sites = atoms in the unit cell; the batch covers sites
 * this_i_beg..this_i_end (1-based) whose pairs are n_neigh0/neighbors_list0/
 * rjs0/xyz0 (already the batch slices). species of every unit-cell atom by
 * global species id (species_all[n_total_sites]). energies0(n_total_sites)
 * and forces0(3, n_total_sites) are ASSIGNED for touched sites. */
int orc_get_gap_soap(const orc_soap_hypers *h, int n_total_sites, int n_sites0,
                     const int *n_neigh0, const int *neighbors_list0,
                     const double *rjs0, const double *xyz0,
                     const int *species_batch, const int *species_all,
                     int n_sparse, const double *Qs, const double *alphas,
                     double delta, double zeta, int do_forces,
                     double *energies0, double *forces0, double *virial);

/* get_number_of_atom_pairs (neighbors.f90:637-778): memory-bounded batches.
 * Returns n_chunks; lists must hold n_sites entries. */
int orc_atom_pair_batches(int n_sites, const int *n_neigh, const double *rjs,
                          double rcut, int l_max, int n_max, int n_soap,
                          int n_species, double max_gbytes, int *i_beg,
                          int *i_end, int *j_beg, int *j_end);

/* ---- MD: md.f90 ------------------------------------------------------------ */
void orc_velocity_verlet(int n, double *positions, double *positions_prev,
                         double *velocities, const double *forces,
                         double *forces_prev, const double *masses, double dt,
                         double *dt_prev, int first_step);
void orc_remove_cm_vel(int n, double *vel, const double *m);
void orc_wrap_pbc(int n, double *positions, const double *a, const double *b,
                  const double *c);

/* ---- full evaluation: one structure, all blocks (turbogap.f90:1253-1378) --- */
typedef struct {
    orc_soap_hypers hypers;
    int n_sparse;
    const double *Qs;      /* (dim, n_sparse) column-major */
    const double *alphas;
    double delta, zeta;
} orc_gap_block;

/* Energies (e0 included), forces, virial of a periodic structure given the
 * unit-cell positions. Builds the supercell and neighbour list itself.
 * Returns 0 on success. n_threads <= 0 uses the OpenMP default. */
int orc_evaluate(int n_sites, const double *positions, const int *species,
                 const double *a, const double *b, const double *c,
                 int n_blocks, const orc_gap_block *blocks,
                 const double *e0_by_species, int n_species_total,
                 double neighbors_buffer, double max_gbytes,
                 double *energies, double *forces, double *virial,
                 int64_t *n_pairs_out);

/* As orc_evaluate for the sites site_beg..site_end-1 only (0-based): the work one
 * MPI rank owns in the reference (turbogap.f90:930-942). */
int orc_evaluate_range(int n_sites, const double *positions, const int *species,
                       const double *a, const double *b, const double *c, int n_blocks,
                       const orc_gap_block *blocks, const double *e0_by_species,
                       int n_species_total, double neighbors_buffer, double max_gbytes,
                       int site_beg, int site_end, double *energies, double *forces,
                       double *virial, int64_t *n_pairs_out);

int orc_set_threads(int n);

/* ---- the other GAP families: distance_2b, angle_3b, core_pot ---------- */
/* One family (types.f90 distance_2b / angle_3b / core_pot). Species are global
 * ids (1-based positions in the input's species_types). */
typedef struct {
    int kind;               /* 1 = distance_2b, 2 = angle_3b, 3 = core_pot               */
    int sp[3];              /* 2b, core_pot: species1, species2; 3b: center, 1, 2         */
    double delta;           /* 2b, 3b                                                     */
    double sigma[3];        /* 2b: sigma[0]; 3b: sigma(1:3)                               */
    double rcut;            /* 2b, 3b; core_pot uses maxval(x)                            */
    int kernel_pol;         /* 3b: 1 = kernel_type "pol", 0 = "exp"                       */
    int n;                  /* sparse points (2b, 3b) or table nodes (core_pot)           */
    const double *Qs;       /* 2b: (n); 3b: Qs(n, 3) column-major                          */
    const double *alphas;   /* (n) */
    const double *cutoff;   /* (n) */
    const double *x, *V, *y2;   /* core_pot: nodes, values, spline second derivatives     */
    double yp1, ypn;        /* core_pot end slopes (after the natural-end replacement)     */
} orc_family;

/* read_files.f90:5454-5505: spline second derivatives y2(n) of (x, V); end
 * slopes > 0.99e30 mean a natural end and are replaced by the spline's slope. */
void orc_core_pot_spline(int n, const double *x, const double *V, double *yp1, double *ypn,
                         double *y2);
/* gap.f90:400-1042 for one family over n_sites sites (n_neigh, neighbors_list,
 * rjs, xyz as build_neighbors_list returns them; species of the sites,
 * neighbor_species of the pairs). energies(n_sites) assigned; forces(3, n_sites0)
 * and virial(3, 3) zeroed and accumulated (2b and core_pot on the sites, 3b on
 * the three atoms of each triplet, by index mod n_sites0). */
void orc_family_energy_forces(const orc_family *f, int n_sites, const int *n_neigh,
                              const int *neighbors_list, const double *rjs, const double *xyz,
                              const int *species, const int *neighbor_species, int n_sites0,
                              double *energies, double *forces, double *virial);
/* orc_evaluate_range with the families added (gap_backend_cpu.f90:79-267). */
int orc_evaluate_full(int n_sites, const double *positions, const int *species, const double *a,
                      const double *b, const double *c, int n_blocks, const orc_gap_block *blocks,
                      int n_families, const orc_family *families, const double *e0_by_species,
                      int n_species_total, double neighbors_buffer, double max_gbytes,
                      int site_beg, int site_end, double *energies, double *forces,
                      double *virial, int64_t *n_pairs_out);

#ifdef __cplusplus
}
#endif
#endif
