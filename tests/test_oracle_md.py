"""The oracle's MD pieces against numpy restatements of md.f90: velocity_verlet
(:226-283), remove_cm_vel (:316-344), wrap_pbc (:348-380), and the velocity draw
of randomize_velocities "maxwell" (:95-158) as done by synth.maxwell_velocities
(shape of the distribution, after tests/velocity_draw)."""
import numpy as np

from _util import O
from turbogap_b200.synth import KB_EV, maxwell_velocities


def test_velocity_verlet_matches_numpy_bitwise():
    rng = np.random.default_rng(1)
    n = 300
    x, xp, v, f, fp = (rng.normal(size=(n, 3)) for _ in range(5))
    m = rng.uniform(1, 30, n)
    for first in (1, 0):
        a = [t.copy() for t in (x, xp, v, f, fp)]
        O.velocity_verlet(a[0], a[1], a[2], a[3], a[4], m, 0.8, 0.6, first)
        vv = v.copy()
        if not first:
            vv = vv + 0.5 * (f + fp) / m[:, None] * 0.6
        xx = x + vv * 0.8 + 0.5 * f / m[:, None] * (0.8 * 0.8)
        assert np.array_equal(a[2], vv) and np.array_equal(a[0], xx)
        assert np.array_equal(a[1], x) and np.array_equal(a[4], f)


def test_remove_cm_and_wrap():
    rng = np.random.default_rng(2)
    n = 50
    v = rng.normal(size=(n, 3))
    m = rng.uniform(1, 12, n)
    O.remove_cm_vel(v, m)
    assert np.abs((m[:, None] * v).sum(0)).max() < 1e-12
    L = 7.5
    p = rng.uniform(-20, 20, size=(n, 3))
    q = p.copy()
    O.wrap_pbc(q, np.array([L, 0, 0.]), np.array([0, L, 0.]), np.array([0, 0, L]))
    assert np.all(q >= 0) and np.all(q < L)
    assert np.allclose(q, p - np.floor(p / L) * L, atol=1e-12)


def test_maxwell_velocity_distribution_shape():
    m = np.full(20000, 12.011 * 103.6426965268)
    v = maxwell_velocities(m, 300.0, seed=3)
    sig = np.sqrt(KB_EV * 300.0 / m[0])
    z = v.ravel() / sig
    assert abs(z.std() - 1) < 0.01 and abs(z.mean()) < 0.01
    # fourth moment of a Gaussian (kurtosis 3): the shape, not only the width
    assert abs((z ** 4).mean() - 3.0) < 0.1
    assert np.abs((m[:, None] * v).sum(0)).max() < 1e-9 * m.sum()


def test_wrap_triclinic_lands_in_the_cell():
    """wrap_pbc in a sheared box: the fractional coordinates end in [0, 1)."""
    rng = np.random.default_rng(3)
    box = np.array([[8.0, 0.0, 0.0], [2.4, 7.5, 0.0], [-1.1, 1.6, 9.0]])
    p = rng.uniform(-25, 25, size=(60, 3))
    q = p.copy()
    O.wrap_pbc(q, box[0], box[1], box[2])
    frac = q @ np.linalg.inv(box)
    assert frac.min() > -1e-12 and frac.max() < 1.0 + 1e-12
    # a whole-cell shift of the original
    shift = (p - q) @ np.linalg.inv(box)
    assert np.abs(shift - np.round(shift)).max() < 1e-9
