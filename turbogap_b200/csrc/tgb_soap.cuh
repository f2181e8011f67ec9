// tgb_soap.cuh -- SOAP descriptor and adjoint force kernels (interfaces).
#pragma once

#include "tgb_common.cuh"

namespace tgb {

constexpr int kMaxZ = 32;  // global species ids 1..31 map through zmap

// Everything the descriptor and force kernels need about one block.
struct SoapParams {
    int ns, amax, lmax, ntot, nlm, dim;
    int nsplit;           // 3: [hi | hi | lo] operand rows, 1: [hi]
    int K1;               // row length (elements) of the split-q GEMM operand
    int tw;               // table width: 2*amax + 2*(lmax+1) floats per node
    int n_atoms;          // unit-cell atoms (folding of supercell indices)
    signed char zmap[kMaxZ];   // global species id -> descriptor species (first match) or -1
    float rcut[kMaxSpecies];
    float tab_h[kMaxSpecies];  // node spacing (A)
    float tab_inv_h[kMaxSpecies];
    const float *table;        // [ns][kTableIntervals + 1][tw]
    const float4 *table_fd;    // [ns][kTableIntervals][functions]: (f, f') at both ends
    const float *self_R;       // [ns][amax]: central-atom contribution to c_{n,00}
    const double *mu;          // [dim]: mean of the sparse set; the GEMMs see q - mu
    const double *g0;          // [dim]: sum_s kcoef_s (q_s - mu), the K = 1 part of dE/dq
    const float *muf, *g0f;    // fp32 copies (the force pass's per-entry terms)
    double mu2, g0mu;          // mu . mu and g0 . mu (FP64)
    // 1 for a compressed block: the descriptor pass writes the raw power spectrum
    // p (FP64, all NT (NT + 1) / 2 (l_max + 1) entries, internal order) to
    // DescOut::praw and stops there, and the force pass reads ForceIn::g as dE/dp
    // in that order (separate instantiations of both kernels, every tile). The
    // compression passes between them work in the compressed space of dim.
    int raw;
    // precision of the tensor-core force tile: 3 = TF32 hi/lo split (about fp32,
    // the plain form), 1 = single TF32 products (the mixed form's budget)
    int force_prec = 3;
    // columns of the split-q row the descriptor writes (the parts, then zeros up
    // to fill_to); 0 means the whole row K1. The mixed form writes nsplit 1 and
    // fills to its network's padded input length.
    int fill_to = 0;
    // Species multiplicity (one global species in two descriptor species of the
    // block, gap_interface.f90:180-199): zmap2 gives the second match or -1, and
    // n_inst = 2 makes the pair passes run over the lists once per match.
    int n_inst = 1;
    signed char zmap2[kMaxZ];
};

// Per-launch site addressing: site i reads CSR row site_row[i] of the pair
// arrays and its results belong to atom site_atom[i].
struct SiteArgs {
    int n_sites;
    const int *site_row;
    const int *site_atom;
    const int64_t *pstart;
    const int *nbr;          // 0-based supercell index per pair
    const double *xyz;       // (3, P) MIC vectors r_j - r_i
    const int *species;      // global species id per unit-cell atom
    int ahead = 0;           // set by the launchers: sites in flight at once (L2 prefetch distance)
    // optional: the global species id of each pair's neighbour (streamed instead of
    // gathering species[neighbour])
    const signed char *nsp = nullptr;
};

// Descriptor entries on the device run in the internal order d = l * NP + pi
// (NP = NT (NT + 1) / 2 channel pairs n <= n2); the reference order is
// pi_ref * (l_max + 1) + l with pi_ref the row-major upper-triangle index. The
// sparse set, mu and g0 are stored in the internal order, so the GEMMs see a
// consistent permutation. Within one l the pairs follow the 8 x 8 Gram blocks of
// the power spectrum's tensor-core products when NT % 8 == 0: blocks (a, b),
// a <= b in row-major order; a diagonal block holds its upper triangle row by
// row (36 entries), an off-diagonal block all 64 entries in the order
// 8 (n - 8a) + (n2 - 8b). Otherwise pi is the row-major upper-triangle index.
__host__ __device__ inline int gram_block_start(int a, int b, int nb) {
    int s = 0;
    for (int i = 0; i < a; ++i) s += 36 + 64 * (nb - 1 - i);
    return s + (b == a ? 0 : 36 + 64 * (b - a - 1));
}

__host__ __device__ inline void internal_pair(int pi, int nt, int &n, int &n2) {
    if (nt % 8 == 0) {
        const int nb = nt / 8;
        for (int a = 0; a < nb; ++a)
            for (int b = a; b < nb; ++b) {
                const int size = a == b ? 36 : 64;
                const int k = pi - gram_block_start(a, b, nb);
                if (k < 0 || k >= size) continue;
                if (a != b) {
                    n = 8 * a + k / 8;
                    n2 = 8 * b + k % 8;
                } else {
                    int g = 0, rem = k;
                    while (rem >= 8 - g) { rem -= 8 - g; ++g; }
                    n = 8 * a + g;
                    n2 = 8 * a + g + rem;
                }
                return;
            }
    }
    int g = 0, rem = pi;
    while (rem >= nt - g) { rem -= nt - g; ++g; }
    n = g;
    n2 = g + rem;
}

int descriptor_ref_index(int d_internal, int nt, int nl);

struct DescOut {
    __nv_bfloat16 *qsplit;   // [n_sites][K1]: bf16 split of delta = q - mu
    float *q;                // [n_sites][dim]: delta = q - mu (fp32)
    double *qoff;            // [n_sites]: delta . mu (FP64)
    double *pnorm;           // [n_sites]
    float *c;                // [n_sites][ntot][nlm]
    double *praw = nullptr;  // compressed blocks: [n_sites][NT (NT + 1) / 2 (l_max + 1)], p
};

struct ForceIn {
    const float *g;          // sum_s (kd_s - kcoef_s)(Q_s - mu), [n_sites][dim] (GEMM 2)
    const float *q;          // delta = q - mu
    const double *pnorm;
    const float *c;
    const double *epart;     // [n_sites][n_etiles]: sum_s alpha_s K^zeta per tile
    const double *kdsum;     // [n_sites][n_etiles]: sum_s kd_s per tile
    int n_etiles;
    double delta2;
    const double *qoff;      // [n_sites]: delta . mu (FP64, from the descriptor pass)
    int ahead = 0;           // set by the launcher: sites in flight at once (L2 prefetch distance)
};

struct ForceOut {
    double *forces;          // (3, n_atoms), accumulated
    double *energies;        // (n_atoms), accumulated
    double *vpart;           // [gridDim][9]
    unsigned *err;
    // optional (batches): each site's virial is also added to vir_struct[atom_struct[atom]]
    const int *atom_struct = nullptr;
    double *vir_struct = nullptr;   // [n_structs][9]
    // optional (local properties): d E_site / d r_j per pair of the site lists,
    // (3, P) in list order; the self pair gets d E_site / d r_site. Under species
    // multiplicity a pair's matches add into it, so the caller zeroes it first.
    double *pair_grad = nullptr;
};

// Host-side construction of the FP64 tables on the device.
struct SoapHostHypers {
    int ns, lmax, radial_enhancement, central_species;
    int alpha_max[kMaxSpecies], species_z[kMaxSpecies];
    double rcut_hard[kMaxSpecies], rcut_soft[kMaxSpecies], nf[kMaxSpecies],
        global_scaling[kMaxSpecies], sigma_r[kMaxSpecies], sigma_r_scaling[kMaxSpecies],
        sigma_t[kMaxSpecies], sigma_t_scaling[kMaxSpecies], amplitude_scaling[kMaxSpecies],
        central_weight[kMaxSpecies];
};

// Floats per table node: one float4 (f, f', f'', 0) per tabulated function
// (alpha_max radial functions, then l_max + 1 angular factors).
int table_width(int amax, int lmax);

// Builds table and self_R (device buffers owned by the caller) in FP64 on the GPU,
// and, when table_fd is given, the descriptor's interval copy
// ([ns][kTableIntervals][amax + lmax + 1] float4: f, f' at both ends).
int build_soap_tables(const SoapHostHypers &h, float *table, float *self_R, cudaStream_t st,
                      float4 *table_fd = nullptr);

// Launchers; return TG_ERR_ARG for unsupported (ns, amax, lmax).
bool soap_shape_supported(int ns, int amax, int lmax);
// CTA tiles of the descriptor and force passes (the autotuner's choices):
// tile 0: 4 sites per CTA, >= 4 CTAs per SM (128 registers); 1: 4 sites, >= 3
// CTAs (168 registers); 2: 2 sites, >= 8 CTAs; 3: 8 sites, >= 2 CTAs.
constexpr int kSoapTiles = 4;
// The force pass has one more tile: the tensor-core kernel (mma.sync TF32, 4 sites
// per CTA), for alpha_max 8, l_max 8, 1 or 2 species, uncompressed blocks.
constexpr int kForceTileMma = 4;
constexpr int kForceTiles = 5;
bool soap_force_mma_supported(const SoapParams &P);
__host__ __device__ constexpr int soap_tile_warps(int t) { return t == 2 ? 2 : (t == 3 ? 8 : 4); }
__host__ __device__ constexpr int soap_tile_minb(int t) {
    return t == 1 ? 3 : (t == 2 ? 8 : (t == 3 ? 2 : 4));
}
int launch_soap_expand(const SoapParams &P, const SiteArgs &S, const DescOut &O, cudaStream_t st,
                       int tile = 0);
int launch_soap_force(const SoapParams &P, const SiteArgs &S, const ForceIn &I, const ForceOut &O,
                      int *n_vpart_blocks, cudaStream_t st, int tile = 0);
int launch_virial_reduce(const double *vpart, int nblk, double *virial_out, cudaStream_t st);

// SOAP compression (soap_turbo's compress_P_*): q = v / |v| with v = C p, C a
// sparse (dim x dimf) matrix, p the raw power spectrum in the internal order.
// Rows of C at or above the transformation's own dim are empty (zero padding to
// the GEMM row length).
struct CompressArgs {
    int dimf;                 // uncompressed entries per site (columns of C)
    const int *row_ptr;       // [dim + 1]: CSR of C by compressed index
    const int *row_col;       //   internal index of p
    const double *row_val;
    int ncols;                // columns of C with at least one entry
    const int *col_idx;       // [ncols]: their internal index of p
    const int *col_ptr;       // [ncols + 1]: CSR of C^T over those columns
    const int *col_row;       //   compressed index
    const double *col_val;
};
// praw [n_sites][dimf] -> O.q, O.qsplit, O.qoff, O.pnorm in the compressed space
// (the outputs of the uncompressed descriptor pass, same layouts, P.dim entries).
int launch_compress_forward(const SoapParams &P, const CompressArgs &C, int n_sites,
                            const double *praw, const DescOut &O, cudaStream_t st);
// dE/dq (I.g, I.kdsum, I.q, I.pnorm in the compressed space) -> dE/dp
// [n_sites][dimf] through the normalisation and C^T.
int launch_compress_adjoint(const SoapParams &P, const CompressArgs &C, int n_sites,
                            const ForceIn &I, float *gfull, cudaStream_t st);

}  // namespace tgb
