"""Species multiplicity in the oracle (gap_interface.f90:180-199, the mask of
assign_species_multiplicity): a global species listed twice in a block feeds
both descriptor species. With identical hypers the two channel sets hold the
same c_{n,lm}, so the power spectrum's blocks repeat the one-species spectrum:
(a, b) and (N + a, N + b) equal it, and the cross block (a, N + b) equals it
for a < b and is sqrt(2) times it for a = b (the diagonal has no sqrt(2))."""
import numpy as np

from _util import oracle_descriptors
from turbogap_b200.hypers import SoapTurboHypers, carbon_hypers
from turbogap_b200.synth import random_structure


def _spectrum_index(n_tot, l_max):
    """(n, n2, l) -> position in the reference order pi_ref * (l_max + 1) + l."""
    idx = {}
    pi = 0
    for n in range(n_tot):
        for n2 in range(n, n_tot):
            for l in range(l_max + 1):
                idx[(n, n2, l)] = pi * (l_max + 1) + l
            pi += 1
    return idx


def test_multiplicity_repeats_the_single_species_spectrum():
    N, L = 4, 4
    st = random_structure(64, 8.5, 1.2, seed=61)
    one = carbon_hypers(n_max=N, l_max=L)
    two = SoapTurboHypers(species_z=[1, 1], alpha_max=[N, N], l_max=L)
    q1, p1, s1 = oracle_descriptors(st, one)
    q2, p2, s2 = oracle_descriptors(st, two)
    assert np.array_equal(s1, s2)
    # unnormalised spectra
    P1 = q1 * p1[:, None]
    P2 = q2 * p2[:, None]
    i1 = _spectrum_index(N, L)
    i2 = _spectrum_index(2 * N, L)
    for (a, b, l), k in i1.items():
        ref = P1[:, k]
        assert np.allclose(P2[:, i2[(a, b, l)]], ref, rtol=1e-12, atol=1e-14)
        assert np.allclose(P2[:, i2[(N + a, N + b, l)]], ref, rtol=1e-12, atol=1e-14)
        cross = P2[:, i2[(a, N + b, l)]]
        assert np.allclose(cross, ref * (np.sqrt(2.0) if a == b else 1.0), rtol=1e-12, atol=1e-14)
        if a < b:   # the lower cross entry holds the same sum
            assert np.allclose(P2[:, i2[(b, N + a, l)]], ref, rtol=1e-12, atol=1e-14)
