# Two soap_turbo blocks (C- and H-centred) and a pair potential, in the
# keyword layout of TurboGAP .gap files. Sparse-set files are written next to
# this file by the tests.
! a comment line of the second kind

gap_beg distance_2b
species1 = C
species2 = H
delta = 0.5
sigma = 0.8
rcut = 4.5
desc_sparse = "d2b.dat"
alphas_sparse = 'a2b.dat'
gap_end

gap_beg soap_turbo
n_species = 2
species = C H
central_species = 1
rcut = 3.7, 3.2
buffer = 0.5 0.
atom_sigma_r = 2*0.5
atom_sigma_t = 0.5d0 0.4D0
atom_sigma_r_scaling = 0. 0.
atom_sigma_t_scaling = 0. 0.
amplitude_scaling = 1. 1.
central_weight = 1. 1.
n_max = 2 2
l_max = 2
nf = 4. 4.
radial_enhancement = 1
basis = "poly3"
scaling_mode = polynomial
zeta = 4
delta = 0.2
desc_sparse = 'desc_C.dat'
alphas_sparse = 'alphas_C.dat'
gap_end

gap_beg soap_turbo
n_species = 2
species = C H
central_species = 2
rcut = 3.7 3.7
atom_sigma_r = 0.5 0.5
atom_sigma_t = 0.5 0.5
n_max = 2 2
l_max = 2
radial_enhancement = 7
desc_sparse = 'desc_H.dat'
alphas_sparse = 'alphas_H.dat'
gap_end
