"""The training cells of the learned surrogate (turbogap_b200.learned): sizes and
temperatures log-uniform over their ranges, the target kind's density,
composition and minimum distance, and the same cells for the same seed."""
import numpy as np
from scipy.spatial import cKDTree

from turbogap_b200 import learned, synth


def test_cells_follow_the_protocol():
    for kind in ("C", "CH"):
        cells = learned.training_cells(kind, 6, seed=5, sizes=(216, 1024))
        assert len(cells) == 6
        again = learned.training_cells(kind, 6, seed=5, sizes=(216, 1024))
        for c, d in zip(cells, again):
            assert np.array_equal(c.structure.positions, d.structure.positions)
            assert c.temperature == d.temperature
        for c in cells:
            st = c.structure
            assert 216 <= st.n <= 1024 and 300.0 <= c.temperature <= 5000.0
            vol = np.linalg.det(st.box)
            if kind == "C":
                assert np.all(st.species == 1)
                assert abs(st.n / vol - synth.carbon_number_density(2.0)) < 1e-9
                dmin = 1.2
            else:
                assert abs(st.n / vol - 0.12) < 1e-9
                assert abs(np.mean(st.species == 2) - 0.25) < 1.0 / st.n
                dmin = 1.0
            tree = cKDTree(st.positions, boxsize=st.box[0, 0])
            assert len(tree.query_pairs(dmin - 1e-9)) == 0
