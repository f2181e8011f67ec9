/*
 * tgb200.h -- C-ABI of the B200 SOAP-GAP backend (libtgb200.so).
 *
 * The reference (TurboGAP, Fortran) selects its backend at link time: a module
 * named gap_backend / gpu_context with identical public procedures is compiled
 * from either the CPU or the GPU source (src/gap_backend_cpu.f90:6-17,
 * src/gpu_context.f90:1-24). This header is the C side of that seam: every
 * entry point is callable from Fortran through ISO_C_BINDING (all arguments are
 * plain pointers and sizes, arrays column-major with the Fortran shapes named
 * below, neighbour indices 1-based).
 *
 * Conventions
 *   - Every call returns TG_OK (0) or a negative TG_ERR_* code; tg_last_error()
 *     returns the text of the last failure on the calling thread.
 *   - (3, n) arrays are contiguous x,y,z triples (Fortran column-major).
 *   - Host pointers are only read/written during the call; the backend owns
 *     every device buffer, stream and cached sparse set.
 *   - Not re-entrant: one host thread per context (one MPI rank per GPU in the
 *     reference's model, src/gpu_context.f90:41-58).
 */
#ifndef TGB200_H
#define TGB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    TG_OK = 0,
    TG_ERR_ARG = -1,          /* invalid argument or unsupported hyperparameter */
    TG_ERR_CUDA = -2,         /* CUDA runtime/driver error                      */
    TG_ERR_CAPACITY = -3,     /* caller buffer too small; required size returned */
    TG_ERR_STATE = -4,        /* call out of order (no context, no open block)  */
    TG_ERR_DEVICE = -5,       /* device-side error word set (see message)       */
    TG_ERR_TIMEOUT = -6,      /* a bounded device wait expired                  */
    TG_ERR_NOMEM = -7         /* device allocation failed                       */
};

/* Arithmetic of the GAP kernel GEMMs. */
enum {
    TG_PREC_BF16X3 = 3,       /* plain form: bf16 hi/lo split, 3 products, fp32 accumulate */
    TG_PREC_BF16 = 1          /* mixed form: single bf16 product, fp32 accumulate          */
};

/* One soap_turbo block's hyperparameters (type soap_turbo, src/types.f90:75-134,
 * as filled by read_gap_hypers, src/read_files.f90:4633-5236). Per-species arrays
 * hold n_species entries; rcut_soft is rcut_hard - buffer (read_files.f90:5101-5108).
 * species_z[s] is the global species id (1-based position in the input deck's
 * species_types) that descriptor species s stands for. One id may appear twice
 * (species multiplicity, gap_interface.f90:180-199): its atoms then feed both
 * descriptor species, each with its own hyperparameters. */
typedef struct {
    int32_t n_species;
    int32_t l_max;
    int32_t radial_enhancement;
    int32_t central_species;        /* 1-based descriptor species index; 0 = all */
    const int32_t *alpha_max;
    const int32_t *species_z;
    const double *rcut_hard;
    const double *rcut_soft;
    const double *nf;
    const double *global_scaling;
    const double *atom_sigma_r;
    const double *atom_sigma_r_scaling;
    const double *atom_sigma_t;
    const double *atom_sigma_t_scaling;
    const double *amplitude_scaling;
    const double *central_weight;
    /* SOAP compression: compress_P_nonzero, compress_P_i/j/el (types.f90:92-110,
     * filled at read_files.f90:5166-5231) and the compressed dim (the file's
     * header, read_files.f90:5171). compress_P_nonzero = 0 (and dim ignored)
     * leaves the descriptor uncompressed. Otherwise the descriptor has dim
     * components, q_c(i) = sum over entries k with compress_P_i[k] = i of
     * compress_P_el[k] * p(compress_P_j[k]) (1-based; p is the power spectrum in
     * the uncompressed order n <= n', l), normalised after the map; Qs then has
     * dim rows. */
    int32_t dim;
    int32_t compress_P_nonzero;
    const int32_t *compress_P_i;
    const int32_t *compress_P_j;
    const double *compress_P_el;
} tg_soap_hypers;

/* ---- device context: gpu_context_init / gpu_context_finalize
 *      (src/gpu_context.f90:41-58). n_omp is set to 1 as on the CPU path.
 *      device < 0 selects rank mod (visible devices): one MPI rank per GPU. */
int tg_context_init(int32_t rank, int32_t device, int32_t *n_omp);
int tg_context_finalize(void);

/* gpu_memory_budget_init (src/gpu_context.f90:100-162): the batch budget in GB
 * the driver uses for max_Gbytes_per_process, from the device's free memory. */
int tg_memory_budget(double *max_gbytes);

const char *tg_last_error(void);

/* ---- sparse set of one block: soap_backend_begin(hypers) / soap_backend_end()
 *      (src/gap.f90:49-64). Uploads Qs(dim, n_sparse) (column-major, one sparse
 *      point per column, src/read_files.f90:707-720) and alphas(n_sparse), builds
 *      the radial/angular tables, and makes the block current. The upload is
 *      cached by block_key: a later begin with the same key, n_sparse, precision
 *      and descriptor shape (species, alpha_max, l_max, central species,
 *      compression) reuses the device copy (the GPU branch of the reference
 *      uploads per call); another shape uploads again, and engines made on the
 *      earlier block keep it. */
int tg_soap_begin(int32_t block_key, const tg_soap_hypers *hypers, int32_t n_sparse,
                  const double *Qs, const double *alphas, double delta, double zeta,
                  int32_t precision);
int tg_soap_end(void);

/* ---- get_gap_soap (src/gap_interface.f90:41-57, live body :178-431) for the
 *      current block, prediction with forces: the remap to central sites and
 *      kept pairs, get_soap, get_soap_energy_and_forces (src/gap.f90:66-259) and
 *      the scatter to global indices.
 *   n_total_sites            atoms in the unit cell (first argument of the reference)
 *   n_sites0                 sites in this batch (this_i_end - this_i_beg + 1)
 *   n_neigh0(n_sites0), neighbors_list0(P) (1-based supercell indices),
 *   rjs0(P), xyz0(3, P)       the batch slices of build_neighbors_list's output
 *   species_batch(n_sites0)  global species id of each batch site
 *   species_all(n_total_sites) global species id of every unit-cell atom
 *   energies0(n_total_sites), forces0(3, n_total_sites): ASSIGNED for the sites
 *     this block touches, left unchanged elsewhere (gap_interface.f90:422-431);
 *   virial(3, 3): overwritten. */
int tg_get_gap_soap(int32_t n_total_sites, int32_t n_sites0, const int32_t *n_neigh0,
                    const int32_t *neighbors_list0, const double *rjs0, const double *xyz0,
                    const int32_t *species_batch, const int32_t *species_all,
                    double *energies0, double *forces0, double *virial);

/* ---- the other GAP families (src/gap_backend_cpu.f90:79-267 add_2b_contribution,
 *      add_core_pot_contribution, add_3b_contribution; kernels src/gap.f90:400-1042).
 * tg_family describes one family as read from its .gap block (types.f90
 * distance_2b / angle_3b / core_pot); species are global ids (1-based
 * positions in the input's species_types):
 *   TG_FAMILY_2B        species[0..1] = species1, species2; delta, sigma[0], rcut;
 *                       n sparse points Qs(n), alphas(n), cutoff(n)
 *   TG_FAMILY_3B        species[0..2] = species_center, species1, species2; delta,
 *                       sigma[0..2], rcut, kernel_type (TG_KERNEL_EXP / TG_KERNEL_POL);
 *                       Qs(n, 3) column-major, alphas(n), cutoff(n)
 *   TG_FAMILY_CORE_POT  species[0..1]; table x(n), V(n) after the core_pot_cutoff
 *                       taper (read_files.f90:5425-5447) and the file's end slopes
 *                       yp1, ypn (> 0.99e30: natural end); the spline second
 *                       derivatives are made here (read_files.f90:5454-5505)
 * The cutoff-function buffer of 2b and 3b is 0.5 A, as the reference passes it.
 * n is at most 4096. */
enum { TG_FAMILY_2B = 1, TG_FAMILY_3B = 2, TG_FAMILY_CORE_POT = 3 };
enum { TG_KERNEL_EXP = 0, TG_KERNEL_POL = 1 };
typedef struct {
    int32_t kind;
    int32_t species[3];
    double delta;
    double sigma[3];
    double rcut;
    int32_t kernel_type;
    int32_t n;
    const double *Qs, *alphas, *cutoff;
    const double *x, *V;
    double yp1, ypn;
} tg_family;

/* Uploads a family under key (the key space is shared with tg_soap_begin; an
 * engine created with the key evaluates the family in every step). */
int tg_family_begin(int32_t key, const tg_family *family);

/* add_*_contribution for one family and one batch, with the arguments of
 * tg_get_gap_soap (the site of each list is its self pair's index mod
 * n_total_sites). ADDS the family's energies0(n_total_sites),
 * forces0(3, n_total_sites) and virial(3, 3) to the caller's arrays, as the
 * reference adds this_energies, this_forces, this_virial to its totals. */
int tg_get_family(int32_t key, int32_t n_total_sites, int32_t n_sites0, const int32_t *n_neigh0,
                  const int32_t *neighbors_list0, const double *rjs0, const double *xyz0,
                  const int32_t *species_all, double *energies0, double *forces0,
                  double *virial);

/* local_property_predict (src/local_properties.f90:174-294) with the current
 * block holding the property model (tg_soap_begin with its sparse set, delta
 * and zeta), through the get_gap_soap remap:
 *   values(n_central)  V_i = max(0, delta^2 sum_s alpha_s K_is^zeta + v0) of
 *                      the block's central sites, in batch order;
 *   value_der(3, P)    (optional) dV_i/dr_j for every pair of those sites' lists,
 *                      in the order of neighbors_list0 (the self pair holds
 *                      dV_i/dr_i); zero for pairs the block does not see and
 *                      for every pair of a site whose value was clamped to 0.
 * The reference snaps zeta to an integer within 1e-10 here (1e-5 for energies);
 * the device snaps within 1e-5 in both. */
int tg_get_local_property(int32_t n_total_sites, int32_t n_sites0, const int32_t *n_neigh0,
                          const int32_t *neighbors_list0, const double *rjs0, const double *xyz0,
                          const int32_t *species_batch, const int32_t *species_all, double v0,
                          double *values, double *value_der, int32_t *n_central);

/* get_soap_dipole (src/gap.f90:261-398) with the current block holding a dipole
 * GAP (tg_soap_begin: its sparse set, delta and zeta), through the get_gap_soap
 * remap, with the arguments of tg_get_local_property:
 *   dipoles(3, n_central)  mu_i = dE_i/dr_i, the gradient of the block's local
 *                          fictitious energy E_i with respect to the central
 *                          atom's own position (the self pair of its list);
 *   energies(n_central)    (optional) E_i = delta^2 sum_s alpha_s K_is^zeta, no
 *                          e0 and no clamp: a fitting artefact that is never
 *                          added to the energy or its gradient to the forces.
 * Central sites in batch order; zeta snapped to an integer within 1e-5 as the
 * reference does here. The total dipole is the sum of mu_i. */
int tg_get_soap_dipole(int32_t n_total_sites, int32_t n_sites0, const int32_t *n_neigh0,
                       const int32_t *neighbors_list0, const double *rjs0, const double *xyz0,
                       const int32_t *species_batch, const int32_t *species_all,
                       double *dipoles, double *energies, int32_t *n_central);

/* get_ts_energy_and_forces (src/vdw.f90:163-493): Tkatchenko-Scheffler
 * dispersion from Hirshfeld volumes, with the reference's arguments (host
 * arrays, Fortran layouts, 1-based neighbour indices and species):
 *   hirshfeld_v(n_sites) of this batch's sites and hirshfeld_v_cart_der(3, P)
 *   per pair of their lists (tg_get_local_property gives both), n_neigh(n_sites),
 *   neighbors_list(P), neighbor_species(P), rjs(P), xyz(3, P), the neighbours'
 *   volumes hirshfeld_v_neigh(P), c6_ref/r0_ref/alpha0_ref(n_species),
 *   mbd_ts_scaling(n_sites0) by atom.
 * Outputs are assigned as the reference assigns them: energies(n_sites); with
 * do_forces, forces0(3, n_sites0), virial(3, 3) and local_virial_diag0(3,
 * n_sites0). Pairs count where rcut_inner < rjs < rcut, smoothed over the two
 * buffers. FP64 on the device. */
int tg_get_ts_energy_and_forces(int32_t n_sites, int32_t n_sites0, const double *hirshfeld_v,
                                const double *hirshfeld_v_cart_der, const int32_t *n_neigh,
                                const int32_t *neighbors_list, const int32_t *neighbor_species,
                                double rcut, double buffer, double rcut_inner, double buffer_inner,
                                const double *rjs, const double *xyz,
                                const double *hirshfeld_v_neigh, double sR, double d,
                                int32_t n_species, const double *c6_ref, const double *r0_ref,
                                const double *alpha0_ref, int32_t do_forces, double x_min,
                                double x_max, const double *mbd_ts_scaling, double *energies,
                                double *forces0, double *virial, double *local_virial_diag0);

/* Descriptor only (soap_turbo get_soap as called at gap_interface.f90:320-325,
 * through the same remap): soap(dim, n_central) of the current block's central
 * sites in batch order. The Cartesian derivative array soap_cart_der is never
 * formed on the device; forces come from the fused adjoint contraction. */
int tg_get_soap(int32_t n_total_sites, int32_t n_sites0, const int32_t *n_neigh0,
                const int32_t *neighbors_list0, const double *rjs0, const double *xyz0,
                const int32_t *species_batch, const int32_t *species_all, double *soap,
                int32_t *n_central);

/* ---- build_neighbors_list (src/neighbors.f90:243-605) with
 *      rebuild_neighbors_list = .true.: self pair first, cell list for
 *      orthorhombic boxes of at least 2 rcut, O(N * N_supercell) search
 *      otherwise; per pair rjs, xyz (MIC), thetas, phis, neighbor_species.
 *   positions(3, n_sites_supercell), species_supercell(n_sites_supercell),
 *   do_list(n_sites) (logical as int32), a/b/c_box(3) (orthorhombic boxes are
 *   snapped as the reference does). cap = capacity of the per-pair arrays; if
 *   smaller than needed, returns TG_ERR_CAPACITY with *n_pairs = required.
 *   Lists, rjs and xyz are bit-identical to the reference arithmetic; thetas
 *   and phis are within a few ulp (device acos/atan2). */
int tg_build_neighbors_list(int32_t n_sites_supercell, const double *positions,
                            int32_t n_sites, double *a_box, double *b_box, double *c_box,
                            double rcut_max, const int32_t *indices,
                            const int32_t *species_supercell, const int32_t *do_list,
                            int64_t cap, int32_t *n_neigh, int32_t *neighbors_list,
                            double *rjs, double *thetas, double *phis, double *xyz,
                            int32_t *neighbor_species, int64_t *n_pairs);

/* ---- Neighbour list that allocates nothing. No reference counterpart: the
 *   reference has no device-memory discipline to honour. It serves callers
 *   that own every device byte (an arena-managed or offload host) or may not
 *   allocate inside their time step. Same cell-list kernels as
 *   tg_build_neighbors_list, for ONE orthorhombic box of at least 2 rcut_max
 *   (no supercell, no do_list); scratch lives in a fixed file-scope device
 *   array of about 4.2 MB per GPU, so n_sites <= 131072 and at most 131072
 *   cells, else TG_ERR_CAPACITY. All pointers except the box vectors are
 *   DEVICE pointers on the current device: positions (3, n_sites);
 *   n_neigh (n_sites); pstart (n_sites + 1), pair k of site i at
 *   pstart[i] + k; neighbors_list (cap) 1-based; rjs (cap); xyz (3, cap).
 *   stream: a cudaStream_t (NULL = legacy default stream); the call
 *   synchronises it before returning. *n_pairs = pairs needed; more than cap
 *   gives TG_ERR_CAPACITY. rcut_max must be positive and finite. Make the
 *   first call on a device outside stream capture: it resolves the scratch
 *   address and, under lazy module loading, loads the module that holds the
 *   array, so the device memory it takes appears at that call, once per
 *   device. Calls that overlap on one
 *   device share the scratch and race: serialise them. Needs no
 *   tg_context_init. */
int tg_build_neighbors_list_noalloc(int32_t n_sites, const double *positions,
                                    const double *a_box, const double *b_box,
                                    const double *c_box, double rcut_max, int64_t cap,
                                    int32_t *n_neigh, int64_t *pstart,
                                    int32_t *neighbors_list, double *rjs, double *xyz,
                                    int64_t *n_pairs, void *stream);

/* ---- velocity_verlet (src/md.f90:226-283), no fixed atoms, arrays (3, n). */
int tg_velocity_verlet(int32_t n, double *positions, double *positions_prev,
                       double *velocities, const double *forces, double *forces_prev,
                       const double *masses, double dt, double *dt_prev, int32_t first_step);

/* ---- device-resident MD engine: the hot loop of the driver (turbogap.f90:664,
 *      neighbours :896-997, SOAP blocks :1274-1378, totals :1941/2009) and of
 *      compute_md's NVE path (src/turbogap_md.f90:161-297): neighbour list, every
 *      registered block, energies/forces/virial, wrap_pbc, remove_cm_vel and
 *      velocity_verlet, all on the GPU without host round trips. Each block is
 *      one tg_soap_begin'ed block_key (captured at engine creation). */
typedef struct tg_engine tg_engine;

int tg_engine_create(int32_t n_atoms, const double *positions, const int32_t *species,
                     const double *masses, const double *a_box, const double *b_box,
                     const double *c_box, int32_t n_blocks, const int32_t *block_keys,
                     const double *e0_by_species, int32_t n_species_total,
                     double neighbors_buffer, tg_engine **out);
int tg_engine_destroy(tg_engine *e);
/* Replace positions (3, n) and velocities (3, n) (velocities may be NULL). */
int tg_engine_set_state(tg_engine *e, const double *positions, const double *velocities);
/* Energies (n), forces (3, n), virial (3, 3) at the current positions. */
int tg_engine_compute(tg_engine *e, double *energies, double *forces, double *virial);
/* n_steps of NVE velocity-Verlet with time step dt (fs); graph-captured after
 * the first step. Optional outputs (NULL to skip) are read after the last step:
 * potential energy and kinetic energy (eV). */
int tg_engine_md(tg_engine *e, int32_t n_steps, double dt, double *e_pot, double *e_kin);
int tg_engine_get_state(tg_engine *e, double *positions, double *velocities, double *forces);
/* The frame of the last evaluation, as the reference writes it to its
 * trajectory (turbogap_md.f90:357-380): after an MD step, the wrapped positions
 * the forces were evaluated at (positions_prev) with the synchronous velocities;
 * after tg_engine_compute, the current positions. Any output may be NULL:
 * positions, velocities, forces (3, n), energies (n), virial (3, 3). */
int tg_engine_get_frame(tg_engine *e, double *positions, double *velocities, double *forces,
                        double *energies, double *virial);
/* Neighbour-list reuse with neighbors_buffer > 0 (src/turbogap_md.f90:451-470,
 * src/neighbors.f90:544-590): the lists are built to rcut + neighbors_buffer
 * and rebuilt only once some atom's accumulated squared displacement exceeds
 * neighbors_buffer / 2 (the reference's criterion); in between, the distances
 * of the kept pairs are recomputed. The decision is taken on the device inside
 * the captured step. A supercell (box below 2 (rcut + buffer)) rebuilds every
 * step, as in the reference. Counts of rebuilds and evaluations since
 * creation; both -1 when every evaluation rebuilds. */
int tg_engine_neighbor_stats(tg_engine *e, int64_t *n_builds, int64_t *n_evaluations);
/* CTA tiles of each block's descriptor and force passes, picked at creation by
 * the autotuner (each of 4 tiles timed on the structure itself; environment
 * TGB_AUTOTUNE=0 keeps tile 0, TGB_SOAP_TILE=t pins tile t): tiles[2k], tiles[2k+1]
 * for block k (soap_turbo
 * blocks in key order). Tile t groups 4, 4, 2, 8 sites per CTA for t = 0..3,
 * with at least 4, 3, 8, 2 CTAs resident per SM. n >= 2 * blocks; *n_blocks
 * receives the number of soap_turbo blocks. */
int tg_engine_tiles(tg_engine *e, int32_t *tiles, int32_t n, int32_t *n_blocks);

/* ---- a structure sharded over ranks (one process per GPU), as the reference
 *      splits central atoms over MPI ranks (src/turbogap.f90:930-942) and sums
 *      energies, forces and the virial (src/turbogap.f90:1876-1885).
 * tg_engine_set_site_range: this engine evaluates the central sites in
 *   [site_beg, site_end) (0-based) only; other sites' energies are zero (no e0),
 *   forces and virial hold this range's share. The neighbour search lists the
 *   range's sites only (other sites get empty lists). Default: every site.
 * tg_nccl_unique_id: 128 bytes for tg_engine_set_comm, made on one rank and
 *   sent to the others by the host (e.g. a torch.distributed broadcast).
 * tg_engine_set_comm: collective over n_ranks processes; afterwards every force
 *   evaluation ends with one grouped NCCL all-reduce (sum) of forces, energies
 *   and virial on the engine's stream (captured in the MD graph), so every rank
 *   integrates the whole structure with the full forces. NCCL is loaded at run
 *   time; initialisation and each all-reduce give up after TGB_NCCL_TIMEOUT_S
 *   (default 120) seconds with TG_ERR_TIMEOUT. id128 NULL leaves the
 *   communicator. */
int tg_engine_set_site_range(tg_engine *e, int32_t site_beg, int32_t site_end);
int tg_nccl_unique_id(void *id128);
int tg_engine_set_comm(tg_engine *e, const void *id128, int32_t n_ranks, int32_t rank);
/* Pairs in the current neighbour list. */
int tg_engine_n_pairs(tg_engine *e, int64_t *n_pairs);
/* CUDA stream the engine launches on (cudaStream_t), for timing with events. */
int tg_engine_stream(tg_engine *e, void **stream);
/* Evaluate energies+forces on the device without copying results out; the
 * bench uses this for device-resident timing. */
int tg_engine_compute_device(tg_engine *e);
/* n_steps MD steps launched eagerly with CUDA events between the passes of each
 * step on the engine's stream; ms_per_pass[7] receives the mean milliseconds per
 * step of: neighbour list, descriptor, GEMM 1, GEMM 2, forces+virial, integrate,
 * MLP ensemble + gate (every block summed into its pass). *n_passes = 7. */
int tg_engine_profile(tg_engine *e, int32_t n_steps, double dt, double *ms_per_pass,
                      int32_t *n_passes);
/* Kernel launches in one graph-captured MD step (0 before the first graph exists). */
int tg_engine_graph_kernels(tg_engine *e, int32_t *n_kernels);

/* ---- batches of independent structures (uneven sizes): energies, forces and a
 *   virial per structure for many orthorhombic cells at once, through one batched
 *   neighbour list and the same block kernels, replayed as one CUDA graph. No
 *   reference counterpart: the reference evaluates one structure per run.
 *   positions (3, N) and species (N) concatenate the structures in order;
 *   boxes[9 s .. 9 s + 8] are structure s's a, b, c rows. Neighbour lists follow
 *   the reference's pair set (every periodic image within the cutoff; boxes
 *   smaller than 2 rcut see several images of a neighbour) in their own order. */
typedef struct tg_batch tg_batch;

int tg_batch_create(int32_t n_structs, const int32_t *n_atoms, const double *positions,
                    const int32_t *species, const double *boxes, int32_t n_blocks,
                    const int32_t *block_keys, const double *e0_by_species,
                    int32_t n_species_total, tg_batch **out);
int tg_batch_destroy(tg_batch *b);
/* New positions (3, N); the pair arrays keep the capacity sized at creation
 * (+25 %): TG_ERR_DEVICE reports an overflow. */
int tg_batch_set_positions(tg_batch *b, const double *positions);
/* energies (N), forces (3, N), virials [n_structs][3][3]; any may be NULL. */
int tg_batch_compute(tg_batch *b, double *energies, double *forces, double *virials);
/* Evaluation on the device only (graph replay after the first call). */
int tg_batch_compute_device(tg_batch *b);
int tg_batch_stream(tg_batch *b, void **stream);
/* n_evals eager evaluations with CUDA events between passes; ms_per_pass[7] as
 * for tg_engine_profile (the integrate and MLP entries stay 0). */
int tg_batch_profile(tg_batch *b, int32_t n_evals, double *ms_per_pass, int32_t *n_passes);
/* Kernel launches in one evaluation's CUDA graph. */
int tg_batch_graph_kernels(tg_batch *b, int32_t *n_kernels);
/* The autotuned CTA tiles of the batch's blocks, as tg_engine_tiles. */
int tg_batch_tiles(tg_batch *b, int32_t *tiles, int32_t n, int32_t *n_blocks);
int tg_batch_n_pairs(tg_batch *b, int64_t *n_pairs);

/* ---- learned surrogate (mixed form). No reference counterpart: TurboGAP has
 *   no learned model. Per block, an ensemble of n_members MLPs
 *   dim -> hidden -> hidden -> 1 (SiLU) maps delta = q - mu of a central site
 *   (the block's internal descriptor order, as the engine holds it) to its GAP
 *   energy; dE/dq comes from the network's input gradient and goes through the
 *   same fused force contraction as the GAP path. Training runs on the GPU
 *   (bf16 GEMMs, fp32 accumulation and master weights, Adam) on (delta, E,
 *   dE/dq) samples, with the loss 1/B sum (E - y)^2 + lam/(B D) sum |dE/dx - G|^2
 *   in units normalised by sigma_x (delta scale) and sigma_e (energy scale).
 *   W1 is hidden x dim, W2 hidden x hidden, row-major FP64 on the host. */
typedef struct tg_mlp tg_mlp;

int tg_mlp_create(int32_t dim, int32_t hidden, int32_t n_members, uint64_t seed, tg_mlp **out);
int tg_mlp_destroy(tg_mlp *m);
int tg_mlp_set_member(tg_mlp *m, int32_t member, const double *W1, const double *b1,
                      const double *W2, const double *b2, const double *w3, double b3);
int tg_mlp_get_member(tg_mlp *m, int32_t member, double *W1, double *b1, double *W2, double *b2,
                      double *w3, double *b3);
/* Scales of the normalised units; unset (0) they are taken from the data set at
 * the first tg_mlp_train. */
int tg_mlp_set_normalisation(tg_mlp *m, double sigma_x, double mean_e, double sigma_e);
int tg_mlp_get_normalisation(tg_mlp *m, double *sigma_x, double *mean_e, double *sigma_e);
/* Append samples: delta (n, dim) fp32, energies (n) eV, dE/dq (n, dim) fp32. */
int tg_mlp_add_samples(tg_mlp *m, int32_t n, const float *delta, const double *energy,
                       const float *dedq);
/* Append the central sites of engine block `block` (0-based) from its last exact
 * evaluation (tg_engine_compute or an MD step), device to device. */
int tg_mlp_add_engine_samples(tg_mlp *m, tg_engine *e, int32_t block);
int tg_mlp_n_samples(tg_mlp *m, int64_t *n);
/* epochs over the shuffled data set in batches of `batch` (a multiple of 32),
 * Adam with the step size decaying from lr to lr / 20 over the epochs (cosine);
 * loss_per_epoch[epochs] receives the mean normalised loss of each epoch. */
int tg_mlp_train(tg_mlp *m, int32_t epochs, int32_t batch, double lr, double force_weight,
                 uint64_t seed, double *loss_per_epoch);
/* Ensemble mean energy (eV), its spread (population standard deviation over
 * members, eV; may be NULL) and mean dE/d(delta) (n, dim; may be NULL). */
int tg_mlp_predict(tg_mlp *m, int32_t n, const float *delta, double *energy_mean,
                   double *energy_std, double *dedq_mean);
/* Mixed form for engine block `block`: every step the ensemble evaluates all
 * central sites; sites whose spread exceeds gate_ev are evaluated by the exact
 * GAP kernel instead (compacted on the device, same CUDA graph). m = NULL
 * returns the block to the exact form. The MLP must outlive its use here. */
int tg_engine_set_mlp(tg_engine *e, int32_t block, tg_mlp *m, double gate_ev);
/* Sites of the block and how many the last step sent to the exact kernel. */
int tg_engine_mlp_stats(tg_engine *e, int32_t block, int32_t *n_gated, int32_t *n_sites);

#ifdef __cplusplus
}
#endif
#endif
