"""The reference's on-disk formats (turbogap_b200/formats.py) and the deck
loader, on the CPU: .gap blocks, sparse-set and compression files, extended
XYZ, thermo.log rows and input decks."""
from __future__ import annotations

import os
import shutil

import numpy as np
import pytest

from turbogap_b200 import formats as F
from turbogap_b200.hypers import GapBlock

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "formats")


def test_list_directed_tokens():
    t = F._tokens
    assert t("rcut = 3.7, 3.2") == ["rcut", "=", "3.7", "3.2"]
    assert t("x = 3*0.5 1") == ["x", "=", "0.5", "0.5", "0.5", "1"]
    assert t("f = 'a b' \"it''s\" 'q''q'") == ["f", "=", "a b", "it''s", "q'q"]
    assert t("p = dir/file") == ["p", "=", "dir"]           # slash ends the record
    assert t("k = .false.\t! note") == ["k", "=", ".false.", "!", "note"]
    assert t("n = 2* 7") == ["n", "=", "7"]                   # r* alone is r null values
    assert F._real("0.4D0") == 0.4 and F._real("1.5d-3") == 1.5e-3
    assert F._logical(".true.") and F._logical("T") and not F._logical(".F.")
    with pytest.raises(ValueError):
        F._logical("yes")


def _sparse_files(d, spec, n_sparse, seed):
    rng = np.random.default_rng(seed)
    dim = spec.uncompressed_dim
    Qs = rng.normal(size=(n_sparse, dim))
    al = rng.normal(size=n_sparse)
    with open(os.path.join(d, spec.file_alphas), "w") as fh:
        fh.writelines(f"{a!r}\n" for a in al.tolist())
    with open(os.path.join(d, spec.file_desc), "w") as fh:
        fh.writelines(f"{q!r}\n" for q in Qs.reshape(-1).tolist())
    return Qs, al


@pytest.fixture()
def gapdir(tmp_path):
    shutil.copy(os.path.join(GOLD, "ch.gap"), tmp_path / "ch.gap")
    with pytest.warns(UserWarning, match="radial_enhancement"):
        g = F.read_gap_file(str(tmp_path / "ch.gap"))
    data = [_sparse_files(str(tmp_path), s, 5 + k, 40 + k) for k, s in enumerate(g.soap_turbo)]
    return tmp_path, g, data


def test_gap_file_blocks(gapdir):
    _, g, _ = gapdir
    assert len(g.soap_turbo) == 2 and len(g.distance_2b) == 1
    assert not g.angle_3b and not g.core_pot
    c, h = g.soap_turbo
    assert c.species == ["C", "H"] and c.central_species == 1 and h.central_species == 2
    assert c.rcut_hard == [3.7, 3.2]
    assert c.buffer == [0.5, 0.0] and c.rcut_soft == [3.2, 3.2]     # buffer 0: rcut_soft = rcut
    assert c.atom_sigma_r == [0.5, 0.5] and c.atom_sigma_t == [0.5, 0.4]
    assert c.alpha_max == [2, 2] and c.l_max == 2 and c.uncompressed_dim == 30
    assert c.zeta == 4.0 and c.delta == 0.2 and c.radial_enhancement == 1
    assert (c.file_desc, c.file_alphas) == ("desc_C.dat", "alphas_C.dat")
    # defaults of the second block (types.f90:93-127, read_files.f90:4648-4667)
    assert h.zeta == 2.0 and h.delta == 1.0 and h.nf == [4.0, 4.0]
    assert h.buffer == [0.5, 0.5] and h.amplitude_scaling == [1.0, 1.0]
    assert h.radial_enhancement == 0                           # out of range: warned, reset
    assert h.basis == "poly3" and not h.compress_soap
    assert g.distance_2b[0].keywords["desc_sparse"] == ["d2b.dat"]
    assert g.rcut_max == 4.5


def test_gap_block_load_maps_species(gapdir):
    d, g, data = gapdir
    c = g.soap_turbo[0]
    blk = c.load(["H", "C"], str(d))                        # input lists H first
    assert isinstance(blk, GapBlock)
    assert blk.hypers.species_z == [2, 1]
    assert blk.hypers.central_species == 1
    assert np.array_equal(blk.Qs, data[0][0]) and np.array_equal(blk.alphas, data[0][1])
    assert blk.zeta == 4.0 and blk.delta == 0.2
    with pytest.raises(ValueError, match="not among the input species"):
        c.load(["C"], str(d))


def test_sparse_set_round_trip_and_dims(tmp_path):
    from turbogap_b200.hypers import carbon_hypers
    h = carbon_hypers(n_max=2, l_max=2)
    rng = np.random.default_rng(1)
    blk = GapBlock(h, rng.normal(size=(4, h.dim)), rng.normal(size=4), 1.0, 4.0)
    fd, fa = str(tmp_path / "d.dat"), str(tmp_path / "a.dat")
    F.write_sparse_set(blk, fd, fa)
    a, Q, cut = F.read_alphas_and_descriptors(fd, fa, "soap_turbo")
    assert cut is None
    assert np.array_equal(a, blk.alphas) and np.array_equal(Q, blk.Qs)   # exact round trip
    # distance_2b: alphas records carry a cutoff; dim must be 1
    with open(fa, "w") as fh:
        fh.write("0.5 1.0\n-0.25 0.5\n")
    with open(fd, "w") as fh:
        fh.write("1.5\n2.5\n")
    a, Q, cut = F.read_alphas_and_descriptors(fd, fa, "distance_2b")
    assert a.tolist() == [0.5, -0.25] and cut.tolist() == [1.0, 0.5] and Q.shape == (2, 1)
    with pytest.raises(ValueError, match="dim"):
        F.read_alphas_and_descriptors(fd, fa, "angle_3b")


def test_compress_file_both_forms(tmp_path):
    p = tmp_path / "c1.dat"
    p.write_text("4 4 2 3\n2\n5\n7\n")
    c = F.read_compress_file(str(p), 2)
    assert c.alpha_max == [4, 4] and c.l_max == 2 and c.dim == 3
    assert c.P_i.tolist() == [1, 2, 3] and c.P_j.tolist() == [2, 5, 7]
    M = c.matrix(10)
    assert M.shape == (3, 10) and M[1, 4] == 1.0 and M.sum() == 3.0
    p2 = tmp_path / "c2.dat"
    p2.write_text("8 8 2\nP_transformation\n1 1 0.5\n1 3 0.5\n2 2 -1.0\nend_transformation\n")
    c2 = F.read_compress_file(str(p2), 1)
    assert c2.dim == 2 and c2.P_el.tolist() == [0.5, 0.5, -1.0]
    assert c2.matrix(4).tolist() == [[0.5, 0, 0.5, 0], [0, -1.0, 0, 0]]
    spec = F.SoapTurboSpec(1, ["C"], [8], [3.7], [0.5], [4.0], [0.5], [0.5], [0.0], [0.0],
                           [1.0], [1.0], [1.0], l_max=2, compress_soap=True,
                           file_compress=p2.name)
    assert spec.compression(str(tmp_path)).dim == 2
    spec.file_compress, spec.compress_mode = "none", "trivial"
    assert spec.compression(str(tmp_path)).dim == 8 * 9 // 2 * 3 - 7 * 8 // 2 * 3
    spec.compress_mode = "0_0"
    with pytest.raises(NotImplementedError, match="get_compress_indices"):
        spec.compression(str(tmp_path))


XYZ = """3
lattice="10.0 0.0 0.0 0.0 11.0 0.0 0.0 0.0 12.0" Properties=species:S:1:pos:R:3:charge:R:1:vel:R:3:mass:R:1:fix_atom:S:3 pbc="T T T"
C  1.0 2.0 3.0   9.9   0.1 0.2 0.3   12.011  F F T
H  4.0 5.0 6.0   9.9  -0.1 0.0 0.1   1.008   F F F
C  7.0 8.0 9.5d0 9.9   0.0 0.0 0.0   12.011  T T T
2
Lattice="5.0 0.0 0.0 0.0 5.0 0.0 0.0 0.0 5.0" Properties=species:S:1:pos:R:3 step=7
H 0.5 0.5 0.5
H 1.5 0.5 0.5
"""


def test_extxyz_read_columns_and_frames(tmp_path):
    p = tmp_path / "in.xyz"
    p.write_text(XYZ)
    fr = F.read_extxyz(str(p))
    assert len(fr) == 2
    a, b = fr
    assert a.species == ["C", "H", "C"]
    assert np.allclose(a.lattice, np.diag([10.0, 11.0, 12.0]))
    assert a.positions[2].tolist() == [7.0, 8.0, 9.5]
    assert a.velocities[0].tolist() == [0.1, 0.2, 0.3]          # the charge column is skipped
    assert a.masses.tolist() == [12.011, 1.008, 12.011]
    assert a.fix_atoms[0].tolist() == [False, False, True] and a.fix_atoms[2].all()
    assert a.info["pbc"] == "T T T"
    assert a.arrays["charge"].tolist() == [9.9, 9.9, 9.9]            # other real columns
    assert b.n == 2 and b.velocities is None and b.masses is None and b.info["step"] == "7"


def test_extxyz_write_layout_and_round_trip(tmp_path):
    p = str(tmp_path / "t.xyz")
    rng = np.random.default_rng(0)
    n = 4
    pos, vel, frc = (rng.normal(size=(n, 3)) for _ in range(3))
    le = rng.normal(size=n)
    lat = np.diag([30.0, 31.0, 32.0])
    vir = np.arange(9.0).reshape(3, 3) - 4.0
    kw = dict(time=0.0, dt=0.5, temperature=3.0e8, pressure=1.5, virial=vir, velocities=vel,
              forces=frc, local_energies=le)
    F.write_extxyz(p, ["C", "H", "C", "H"], pos, lat, step=0, **kw)
    F.write_extxyz(p, ["C", "H", "C", "H"], pos + 1, lat, step=10, **kw)
    lines = open(p).read().splitlines()
    assert lines[0] == "       4"
    h = lines[1]
    assert h.startswith(" Properties=species:S:1:pos:R:3:velocities:R:3:forces:R:3:"
                        "local_energy:R:1:fix_atoms:S:3 Lattice=\"30.0000000000   ")
    assert " temperature=" + "*" * 16 + " " in h                 # F16.8 overflow
    assert " time_step=0.5000 " in h and h.endswith(" step=0")
    # the first field is left-adjusted within its 16 columns, the rest right-adjusted
    assert ' virial="-4.00000000' + " " * 10 + "-3.00000000" in h
    assert lines[2].startswith(" C        ") and lines[2].endswith(" F F F")
    fr = F.read_extxyz(p)
    assert len(fr) == 2 and fr[1].info["step"] == "10"
    assert np.allclose(fr[0].positions, pos, atol=5e-9) and np.allclose(fr[0].velocities, vel,
                                                                        atol=5e-9)
    assert np.allclose(fr[1].positions, pos + 1, atol=5e-9)
    assert np.allclose(fr[0].arrays["forces"], frc, atol=5e-9)
    assert np.allclose(fr[0].arrays["local_energy"], le, atol=5e-9)
    e = float(fr[0].info["energy"])
    assert abs(e - le.sum()) < 1e-6
    stress = np.array([float(x) for x in fr[0].info["stress"].split()]).reshape(3, 3)
    assert np.allclose(stress, -vir / (30 * 31 * 32), atol=1e-8)
    F.write_extxyz(p, ["C"], pos[:1], lat, step=-3, **{**kw, "velocities": None,
                                                        "forces": None, "local_energies": None})
    assert open(p).read().splitlines()[-2].endswith(" i_config=3")      # appended


def test_thermo_rows(tmp_path):
    r = F.thermo_row(12, 6.0, 301.25, 1.5, -1234.5678, 99.0)
    assert r == ("        12           6.0000         301.2500           1.50000000"
                 "       -1234.56780000          99.00000000")
    p = tmp_path / "thermo.log"
    p.write_text(F.THERMO_HEADER + "\n" + r + "\n" + F.thermo_row(13, 6.5, 3e13, 1, 2, 3) + "\n")
    t = F.read_thermo(str(p))
    assert t.shape == (2, 6) and t[0].tolist() == [12, 6.0, 301.25, 1.5, -1234.5678, 99.0]
    assert np.isnan(t[1, 2])                                   # overflowed field
    # T and P from E_kin and the virial (turbogap_md.f90:283-288)
    T = F.instant_temperature(1.0, 11)
    assert abs(T - 2.0 / 30.0 / F.KB_EV) < 1e-9
    P = F.instant_pressure(1.0, 11, np.eye(3) * 3.0, 1000.0)
    assert abs(P - (10 * F.KB_EV * T + 3.0) / 1000.0 * F.EV_PER_A3_TO_BAR) < 1e-6


DECK = """! species
atoms_file = 'atoms.xyz'
pot_file = 'ch.gap'
n_species = 2
Species = C H
masses = 12.011 1.008
e0 = -0.5 -0.25   ! per species
MD_nsteps = 20
md_step = 0.5
write_thermo = 5
write_xyz = 10
thermostat = none
"""


def test_input_deck(tmp_path):
    p = tmp_path / "input"
    p.write_text(DECK)
    d = F.read_input_file(str(p))
    assert d.species == ["C", "H"] and d.masses_amu == [12.011, 1.008]
    assert d.e0 == [-0.5, -0.25] and d.md_nsteps == 20 and d.md_step == 0.5
    assert d.write_thermo == 5 and d.write_xyz == 10
    assert d.t_beg == 300.0 and d.velocity_distribution == "uniform" and d.neighbors_buffer == 0
    assert d.off_path() == []
    p.write_text(DECK + "thermostat = Berendsen\nadaptive_time = .true.\n")
    assert F.read_input_file(str(p)).off_path() == ["thermostat = berendsen",
                                                    "adaptive_time = True"]


def test_deck_loader(gapdir):
    from turbogap_b200 import deck as D
    d, g, data = gapdir
    (d / "input").write_text(DECK)
    (d / "atoms.xyz").write_text(XYZ.split("2\nLattice")[0])
    (d / "a2b.dat").write_text("0.5 1.0\n-0.25 0.75\n0.125 0.5\n")
    (d / "d2b.dat").write_text("1.5\n2.0\n2.5\n")
    with pytest.warns(UserWarning):
        dk = D.Deck(str(d / "input"))
    (f2,) = dk.families
    assert f2.kind == "distance_2b" and f2.species == (1, 2)
    assert (f2.delta, f2.sigma, f2.rcut) == (0.5, 0.8, 4.5)
    assert f2.Qs.tolist() == [1.5, 2.0, 2.5] and f2.cutoff.tolist() == [1.0, 0.75, 0.5]
    assert D.family_key(f2) >= 0x40000000 > D.block_key(dk.blocks[0])
    assert [b.hypers.central_species for b in dk.blocks] == [1, 2]
    fr = dk.frames[0]
    ids = dk.species_ids(fr)
    assert ids.tolist() == [1, 2, 1]
    m = dk.masses(fr, ids)                                     # the XYZ mass column wins
    assert np.allclose(m, np.array([12.011, 1.008, 12.011]) * F.AMU_TO_EV_FS2_A2)
    assert D.block_key(dk.blocks[0]) != D.block_key(dk.blocks[1])
    assert D.block_key(dk.blocks[0]) == D.block_key(D.Deck(str(d / "input")).blocks[0])


def test_drawn_velocities():
    from turbogap_b200 import deck as D
    m = np.full(500, 12.011 * F.AMU_TO_EV_FS2_A2)
    for dist in ("uniform", "maxwell"):
        v = D.draw_velocities(m, 600.0, dist, seed=3)
        assert np.abs((m[:, None] * v).sum(0)).max() < 1e-9
        T = F.instant_temperature(0.5 * float(np.sum(m[:, None] * v * v)), len(m))
        assert abs(T - 600.0) < (1e-9 if dist == "uniform" else 60.0)
    assert not D.draw_velocities(m[:1], 600.0, "uniform", 0).any()


GAP3 = """gap_beg angle_3b
species_center = C
species1 = C
species2 = H
delta = 0.01
sigma = 4. 4. 3.
rcut = 3.5
kernel_type = "pol"
desc_sparse = 'd3b.dat'
alphas_sparse = 'a3b.dat'
gap_end

gap_beg core_pot
species1 = H
species2 = H
core_pot_file = 'cp.dat'
gap_end core_pot
"""


def test_three_body_and_core_pot_blocks(tmp_path):
    (tmp_path / "f.gap").write_text(GAP3)
    (tmp_path / "a3b.dat").write_text("0.5 1.0\n-0.25 0.5\n")
    (tmp_path / "d3b.dat").write_text("3.0\n0.25\n2.0\n4.0\n1.0\n2.5\n")
    (tmp_path / "cp.dat").write_text("4 1.0e50 0.0\n0.5 8.0\n1.0 4.0\n1.5 2.0\n2.0 0.0\n")
    g = F.read_gap_file(str(tmp_path / "f.gap"))
    f3 = g.angle_3b[0].load(["C", "H"], str(tmp_path))
    assert f3.species == (1, 1, 2) and f3.kernel_type == "pol" and f3.sigma == [4.0, 4.0, 3.0]
    assert f3.Qs.tolist() == [[3.0, 0.25, 2.0], [4.0, 1.0, 2.5]]     # 3 records per point
    assert f3.alphas.tolist() == [0.5, -0.25] and f3.cutoff.tolist() == [1.0, 0.5]
    cp = g.core_pot[0].load(["C", "H"], str(tmp_path), core_pot_cutoff=1.5, core_pot_buffer=0.5)
    assert cp.species == (2, 2) and cp.x.tolist() == [0.5, 1.0, 1.5]
    assert cp.V[:2].tolist() == [8.0, 4.0] and abs(cp.V[2]) < 1e-15   # tapered to 0 at 1.5
    assert cp.yp1 == 1e50 and cp.ypn == 0.0 and g.rcut_max == 3.5


def test_compressed_block_round_trip(tmp_path):
    """A compressed block written as .gap + sparse set + compress file loads back
    with the same transformation and descriptors."""
    from turbogap_b200.hypers import GapBlock, SoapCompression, carbon_hypers
    rng = np.random.default_rng(5)
    comp = SoapCompression(20, np.arange(1, 21).repeat(2), rng.integers(1, 325, size=40),
                           rng.normal(size=40))
    h = carbon_hypers()
    h.compress = comp
    blk = GapBlock(h, rng.normal(size=(6, 20)), rng.normal(size=6))
    F.write_sparse_set(blk, str(tmp_path / "d.dat"), str(tmp_path / "a.dat"))
    F.write_compress_file(str(tmp_path / "c.dat"), comp, h.alpha_max, h.l_max)
    with open(tmp_path / "x.gap", "w") as fh:
        F.write_soap_block(fh, F.spec_from_block(blk, ["C"], "d.dat", "a.dat", "c.dat"))
    b2 = F.read_gap_file(str(tmp_path / "x.gap")).soap_turbo[0].load(["C"], str(tmp_path))
    assert b2.hypers.dim == 20 and b2.hypers.uncompressed_dim == 324
    assert np.array_equal(b2.hypers.compress.P_i, comp.P_i)
    assert np.array_equal(b2.hypers.compress.P_j, comp.P_j)
    assert np.array_equal(b2.hypers.compress.P_el, comp.P_el)
    assert np.array_equal(b2.Qs, blk.Qs)
    with pytest.raises(ValueError, match="compress file"):
        F.spec_from_block(blk, ["C"], "d.dat", "a.dat")
