"""The oracle's distance_2b, angle_3b and core_pot families (gap.f90:400-1042,
read_files.f90:5425-5505): spline set-up against scipy, and analytic forces and
virial against central finite differences of the oracle's own energy (the
tests/fd_gap methodology of the reference, strain 1e-4; h = 1e-4 A, because
the 2b Gaussians of width 0.5 A leave a 4e-4 truncation error at 1e-3 A)."""
import numpy as np
import pytest
from scipy.interpolate import CubicSpline

from _util import O, make_families
from turbogap_b200 import families as FM
from turbogap_b200.synth import random_structure

H_FD = 1e-4
STRAIN = 1e-4
L = (90 / 0.12) ** (1 / 3)


@pytest.fixture(scope="module")
def setup():
    st = random_structure(90, L, 1.0, seed=25, h_fraction=0.25)
    return st, make_families(3)


def _energy(st, fams, pos=None, box=None):
    e, _, _, _ = O.evaluate(st.positions if pos is None else pos, st.species,
                            st.box if box is None else box, [], families=fams)
    return e.sum()


def test_core_pot_spline_matches_scipy():
    x = np.array([0.5, 0.7, 1.0, 1.2, 1.6, 2.0, 2.5])
    V = 4.0 * np.exp(-1.7 * x)
    # clamped start, natural end
    y2, yp1, ypn = O.core_pot_spline(x, V, -2.0, 1e50)
    cs = CubicSpline(x, V, bc_type=((1, -2.0), (2, 0.0)))
    assert np.allclose(y2, cs(x, 2), rtol=1e-10, atol=1e-10)
    assert yp1 == -2.0 and abs(ypn - cs(x[-1], 1)) < 1e-10
    # natural start, clamped end
    y2, yp1, ypn = O.core_pot_spline(x, V, 1e50, 0.0)
    cs = CubicSpline(x, V, bc_type=((2, 0.0), (1, 0.0)))
    assert np.allclose(y2, cs(x, 2), rtol=1e-10, atol=1e-10)
    assert abs(yp1 - cs(x[0], 1)) < 1e-10 and ypn == 0.0


def test_core_pot_taper():
    x = np.linspace(0.5, 3.0, 26)
    c = FM.CorePot.from_table((1, 1), x, np.ones_like(x), 1e50, 0.0, cutoff=2.5, buffer=1.0)
    assert c.x[-1] == pytest.approx(2.5) and len(c.x) == 21
    assert np.all(c.V[c.x <= 1.5] == 1.0)
    assert c.V[-1] == pytest.approx(0.0, abs=1e-15)
    assert c.V[c.x > 1.5][0] == pytest.approx(0.5 * (np.cos(np.pi * (1.6 - 1.5)) + 1.0))


@pytest.mark.parametrize("k", [0, 1, 2, 3, None])
def test_family_forces_match_finite_differences(setup, k):
    st, fams = setup
    fams = fams if k is None else [fams[k]]
    e, f, _, _ = O.evaluate(st.positions, st.species, st.box, [], families=fams)
    assert np.abs(e).max() > 1e-4 and np.abs(f).max() > 1e-3   # the family is not idle
    for i in (0, 5, 17, 44):
        for q in range(3):
            p = st.positions.copy()
            p[i, q] += H_FD
            ep = _energy(st, fams, pos=p)
            p[i, q] -= 2 * H_FD
            em = _energy(st, fams, pos=p)
            fd = -(ep - em) / (2 * H_FD)
            assert abs(fd - f[i, q]) <= 1e-4 * max(abs(f[i, q]), 1e-3 * np.abs(f).max())


@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_family_virial_matches_strain_derivative(setup, k):
    st, fams = setup
    fams = [fams[k]]
    _, _, vir, _ = O.evaluate(st.positions, st.species, st.box, [], families=fams)
    for a, b in ((0, 0), (1, 1), (0, 1), (1, 2)):
        def strained(s):
            eps = np.eye(3)
            eps[a, b] += s
            return _energy(st, fams, pos=st.positions @ eps.T, box=st.box @ eps.T)
        dE = (strained(STRAIN) - strained(-STRAIN)) / (2 * STRAIN)
        assert abs(-dE - vir[a, b]) <= 1e-4 * np.abs(vir).max()


def test_family_sum_rules(setup):
    st, fams = setup
    e, f, v, _ = O.evaluate(st.positions, st.species, st.box, [], families=fams)
    assert np.abs(f.sum(0)).max() < 1e-10 * max(1.0, np.abs(f).max())
    assert np.abs(v - v.T).max() < 1e-12
    # the site-range split sums to the whole
    es, fs, vs = np.zeros_like(e), np.zeros_like(f), np.zeros_like(v)
    for beg, end in ((0, 31), (31, 90)):
        a, b_, c, _ = O.evaluate(st.positions, st.species, st.box, [], families=fams,
                                 site_range=(beg, end))
        es += a
        fs += b_
        vs += c
    assert np.abs(es - e).max() < 1e-12 and np.abs(fs - f).max() < 1e-12
    assert np.abs(vs - v).max() < 1e-12
