"""The oracle's neighbour lists against an independent pure-Python restatement of
build_neighbors_list (src/neighbors.f90:243-605) and against a brute-force
pair search (same pair sets), in the spirit of tests/mc_mpi_neighbors
(cold-rebuild comparison of lists)."""
import math

import numpy as np
import pytest

from _util import O, neighbor_data
from turbogap_b200.synth import random_structure


def f_modulo(a, p):
    r = math.fmod(a, p)
    if r != 0.0:
        if (a < 0.0) != (p < 0.0):
            r += p
    else:
        r = math.copysign(0.0, p)
    return r


def mic(pi, pj, L):
    d = [0.0, 0.0, 0.0]
    d2 = 0.0
    for q in range(3):
        v = f_modulo(pj[q] - pi[q], L[q])
        if v > L[q] / 2.0:
            v = v - L[q]
        d[q] = v
        d2 = d2 + v * v
    return d, math.sqrt(d2)


def py_build_list(pos, n_sites, L, rcut, small):
    """Line-by-line restatement (orthorhombic boxes) in pure Python."""
    pos = [list(map(float, p)) for p in pos]
    nsc = len(pos)
    nl, nn = [], [0] * n_sites
    if not small:
        mx, my, mz = int(L[0] / rcut), int(L[1] / rcut), int(L[2] / rcut)
        head = [0] * (mx * my * mz)
        nxt = [0] * (n_sites + 1)
        tol = 1e-10
        ctr = [L[0] / 2.0, L[1] / 2.0, L[2] / 2.0]

        def cell(i):
            d, _ = mic(ctr, pos[i - 1], L)
            d = [d[q] + ctr[q] for q in range(3)]
            return (int(d[0] / (L[0] + tol) * mx), int(d[1] / (L[1] + tol) * my),
                    int(d[2] / (L[2] + tol) * mz))

        for i in range(1, n_sites + 1):
            ci, cj, ck = cell(i)
            j = 1 + ci % mx + (cj % my) * mx + (ck % mz) * my * mx
            nxt[i] = head[j - 1]
            head[j - 1] = i
        for i in range(1, n_sites + 1):
            nn[i - 1] += 1
            nl.append(i)
            ci, cj, ck = cell(i)
            i2, j2, k2 = ci + 1, cj + 1, ck + 1
            for k3 in range(k2 - 1, k2 + 2):
                if mz == 1 and k3 != 1 or mz == 2 and ((k2 == 1 and k3 == 0) or (k2 == 2 and k3 == 3)):
                    continue
                for j3 in range(j2 - 1, j2 + 2):
                    if my == 1 and j3 != 1 or my == 2 and ((j2 == 1 and j3 == 0) or (j2 == 2 and j3 == 3)):
                        continue
                    for i3 in range(i2 - 1, i2 + 2):
                        if mx == 1 and i3 != 1 or mx == 2 and ((i2 == 1 and i3 == 0) or (i2 == 2 and i3 == 3)):
                            continue
                        c = 1 + (i3 - 1) % mx + ((j3 - 1) % my) * mx + ((k3 - 1) % mz) * mx * my
                        k = head[c - 1]
                        while k != 0:
                            if k != i and mic(pos[i - 1], pos[k - 1], L)[1] < rcut:
                                nn[i - 1] += 1
                                nl.append(k)
                            k = nxt[k]
    else:
        for i in range(1, n_sites + 1):
            nn[i - 1] += 1
            nl.append(i)
            for j in range(1, nsc + 1):
                if j != i and mic(pos[i - 1], pos[j - 1], L)[1] < rcut:
                    nn[i - 1] += 1
                    nl.append(j)
    return np.array(nn), np.array(nl)


@pytest.mark.parametrize("n,L,seed", [(60, 9.0, 1), (40, 8.0, 3), (70, 11.5, 5), (30, 6.0, 4),
                                      (20, 5.0, 7)])
def test_oracle_list_matches_python_restatement(n, L, seed):
    st = random_structure(n, L, 1.2, seed=seed)
    nl = neighbor_data(st, 3.7)
    small = bool(np.any(nl["indices"] > 1))
    nn, lst = py_build_list(nl["pos_sc"], st.n, nl["box_sc"].diagonal(), 3.7, small)
    assert np.array_equal(nn, nl["n_neigh"])
    assert np.array_equal(lst, nl["neighbors_list"])


def test_oracle_list_pair_set_equals_brute_force():
    st = random_structure(216, 12.91, 1.2, seed=1000)
    nl = neighbor_data(st, 3.7)
    L = st.box.diagonal()
    starts = np.concatenate([[0], np.cumsum(nl["n_neigh"])])
    d = st.positions[None, :, :] - st.positions[:, None, :]
    d -= L * np.round(d / L)
    r = np.sqrt((d ** 2).sum(-1))
    for i in range(st.n):
        got = set(nl["neighbors_list"][starts[i] + 1:starts[i + 1]] - 1)
        want = set(np.where((r[i] < 3.7) & (np.arange(st.n) != i))[0])
        assert got == want
        assert nl["neighbors_list"][starts[i]] == i + 1      # self first
        assert nl["rjs"][starts[i]] == 0.0
    # symmetric full lists, rjs consistent with xyz
    assert np.allclose(np.linalg.norm(nl["xyz"], axis=1), nl["rjs"], rtol=0, atol=1e-14)


def test_supercell_replica_order():
    """read_files.f90:347-363: replicas a-index slowest, then b, then c, then atom."""
    st = random_structure(5, 4.0, 1.0, seed=2)
    ind = np.array([2, 3, 1], np.int32)
    pos, sp = O.make_supercell(st.positions, st.species, *st.box, ind)
    k = 0
    for i2 in range(2):
        for j2 in range(3):
            for i in range(5):
                assert np.allclose(pos[k], st.positions[i] + i2 * st.box[0] + j2 * st.box[1])
                k += 1


def test_number_of_unit_cells():
    assert list(O.number_of_unit_cells(*np.eye(3) * 12.91, 3.7)) == [1, 1, 1]
    assert list(O.number_of_unit_cells(*np.eye(3) * 7.0, 3.7)) == [2, 2, 2]
    assert list(O.number_of_unit_cells(*np.diag([7.4, 8.0, 3.0]), 3.7)) == [1, 1, 3]
