// tgb_family.cuh -- the other GAP families behind the same seam: distance_2b,
// angle_3b and core_pot (src/gap_backend_cpu.f90:79-267; kernels
// src/gap.f90:400-1042), evaluated on the device from the same neighbour
// lists as the SOAP blocks.
#pragma once

#include "tgb_common.cuh"
#include "tgb_neighbors.cuh"
#include "tgb_soap.cuh"

#include <vector>

namespace tgb {

constexpr int kFamilyMaxN = 4096;   // sparse points (2b, 3b) or table nodes (core_pot)

// Device copy of one family. Parameters are folded on the host: 2b weights
// w_s = delta^2 alpha_s cutoff_s; 3b prefactors 2 delta^2 alpha_s cutoff_s.
struct Family {
    int key = 0;
    int kind = 0;                 // TG_FAMILY_2B, TG_FAMILY_3B, TG_FAMILY_CORE_POT
    int sp[3] = {0, 0, 0};        // global species ids
    int pol = 0;                  // 3b kernel_type "pol"
    int n = 0;
    double sigma[3] = {1, 1, 1};
    double rcut = 0.0;            // core_pot: the last table node
    double yp1 = 0.0, ypn = 0.0;  // core_pot end slopes after the natural-end replacement
    double *p = nullptr;          // 2b: (Q, w) pairs; 3b: (Q1, Q2, Q3, pref); core_pot: (x, V, y2)
    Family() = default;
    Family(const Family &) = delete;
    Family &operator=(const Family &) = delete;
    ~Family() { dev_free(p); }
};

int family_create(const tg_family &f, Family &out);

// Adds the family's energies, forces and virial of the sites in S (rows of the
// neighbour list: pstart, nbr (0-based supercell), rjs, xyz) into en, fo, vir.
int evaluate_family(const Family &F, const SiteArgs &S, const double *rjs, int n_atoms, double *en,
                    double *fo, double *vir, cudaStream_t st);

// Central sites of a family among atoms [beg, end) (host species ids).
void family_sites(const Family &F, const int *species_h, int beg, int end, std::vector<int> &out);

}  // namespace tgb
