"""The reference's on-disk formats, read and written on the host.

* ``.gap`` potential files: ``gap_beg <type>`` ... ``gap_end`` blocks, parsed
  like ``read_gap_hypers`` (read_files.f90:4504-5236). soap_turbo blocks become
  typed specs; distance_2b, angle_3b and core_pot blocks keep their keywords.
* Sparse-set files ``desc_sparse`` / ``alphas_sparse``
  (``read_alphas_and_descriptors``, read_files.f90:660-768).
* SOAP compression files (read_files.f90:5166-5204).
* Extended XYZ, read like ``read_xyz`` + ``read_xyz_line`` (read_files.f90:67-318,
  xyz.f90:489-540) and written like ``write_extxyz`` (xyz.f90:169-486).
* ``thermo.log`` rows (turbogap_md.f90:299-330).
* The input deck (``read_input_file``, read_files.f90:780-1312): every
  ``keyword = values`` line, with typed access to the keywords of NVE
  molecular dynamics.

Text is split into items the way Fortran list-directed input splits it
(``_tokens``): blanks and commas separate, quotes delimit strings, an unquoted
``/`` ends the record, ``r*c`` repeats ``c`` r times, and ``1.0d0`` is a real.
"""
from __future__ import annotations

import os
import re
import warnings
from dataclasses import dataclass, field
from typing import Dict, Iterator, List, Optional, Sequence

import numpy as np

from .hypers import GapBlock, SoapCompression, SoapTurboHypers, trivial_compression

AMU_TO_EV_FS2_A2 = 103.6426965268      # read_files.f90:1301, xyz.f90:466
EV_PER_A3_TO_BAR = 1602176.6208        # turbogap.f90:95
KB_EV = 8.6173303e-5                   # md.f90:104

_REPEAT = re.compile(r"^(\d+)\*(.*)$")


def _tokens(line: str) -> List[str]:
    """Items of one record as Fortran list-directed input sees them."""
    out: List[str] = []
    i, n = 0, len(line)
    while i < n:
        c = line[i]
        if c in " \t,\r\n":
            i += 1
            continue
        if c in "'\"":
            j, buf = i + 1, []
            while j < n:
                if line[j] == c:
                    if j + 1 < n and line[j + 1] == c:   # doubled quote = one quote
                        buf.append(c)
                        j += 2
                        continue
                    break
                buf.append(line[j])
                j += 1
            out.append("".join(buf))
            i = j + 1
            continue
        if c == "/":                                     # slash ends the record
            break
        j = i
        while j < n and line[j] not in " \t,/\r\n":
            j += 1
        tok = line[i:j]
        m = _REPEAT.match(tok)
        if m and m.group(2):
            out.extend([m.group(2)] * int(m.group(1)))
        elif not m:
            out.append(tok)
        i = j
    return out


def _real(tok: str) -> float:
    return float(tok.replace("d", "e").replace("D", "e"))


def _int(tok: str) -> int:
    return int(tok)


def _logical(tok: str) -> bool:
    """Fortran logical input: optional leading '.', then T or F."""
    t = tok[1:] if tok.startswith(".") else tok
    if t[:1] in ("T", "t"):
        return True
    if t[:1] in ("F", "f"):
        return False
    raise ValueError(f"not a Fortran logical: {tok!r}")


def _values(toks: List[str], n: int, conv, key: str):
    """The n items after ``keyword =`` converted with conv."""
    vals = toks[2:2 + n]
    if len(vals) < n:
        raise ValueError(f"keyword {key!r} needs {n} value(s), got {toks[2:]}")
    return [conv(v) for v in vals]


def _records(path: str) -> List[str]:
    with open(path, "r") as fh:
        return fh.read().splitlines()


# --------------------------------------------------------------------------
# .gap files
# --------------------------------------------------------------------------

@dataclass
class CompressSpec:
    """A SOAP compression transformation: q_c(i) = sum P_el * q(j) over the
    nonzero entries (P_i, P_j), 1-based as in the file (read_files.f90:5166-5204)."""
    alpha_max: List[int]
    l_max: int
    dim: int
    P_i: np.ndarray
    P_j: np.ndarray
    P_el: np.ndarray

    def matrix(self, full_dim: int) -> np.ndarray:
        """The dense (dim, full_dim) transformation."""
        return self.compression().matrix(full_dim)

    def compression(self) -> SoapCompression:
        """The transformation as the block's hyperparameters carry it (the
        header's alpha_max and l_max are read and not used, as in the reference)."""
        return SoapCompression(self.dim, self.P_i, self.P_j, self.P_el)


def read_compress_file(path: str, n_species: int) -> CompressSpec:
    """First record: n_species alpha_max values, l_max and the compressed dim.
    Then either a ``P_transformation`` ... ``end_transformation`` list of
    ``i j value`` triples, or (the older form) dim lines of one kept index each,
    which means P_i = line number and P_el = 1."""
    recs = _records(path)
    head: List[str] = []
    k = 0
    while len(head) < n_species + 2:          # list-directed read may span records
        if k >= len(recs):
            raise ValueError(f"{path}: header needs {n_species + 2} integers")
        head += _tokens(recs[k])
        k += 1
    alpha_max = [_int(t) for t in head[:n_species]]
    l_max, dim = _int(head[n_species]), _int(head[n_species + 1])
    if k < len(recs) and recs[k].strip() == "P_transformation":
        rows = []
        k += 1
        while k < len(recs) and recs[k].strip() != "end_transformation":
            t = _tokens(recs[k])
            rows.append((_int(t[0]), _int(t[1]), _real(t[2])))
            k += 1
        if k >= len(recs):
            raise ValueError(f"{path}: P_transformation without end_transformation")
        P_i = np.array([r[0] for r in rows], dtype=np.int64)
        P_j = np.array([r[1] for r in rows], dtype=np.int64)
        P_el = np.array([r[2] for r in rows], dtype=np.float64)
    else:
        if len(recs) - k < dim:
            raise ValueError(f"{path}: {dim} kept indices expected, found {len(recs) - k}")
        P_j = np.array([_int(_tokens(recs[k + i])[0]) for i in range(dim)], dtype=np.int64)
        P_i = np.arange(1, dim + 1, dtype=np.int64)
        P_el = np.ones(dim)
    return CompressSpec(alpha_max, l_max, dim, P_i, P_j, P_el)


@dataclass
class SoapTurboSpec:
    """One ``gap_beg soap_turbo`` block as written in the file.

    Per-species lists are in the block's own species order (``species``). The
    ``buffer`` list holds what the file gives; ``rcut_soft`` applies the
    conversion done once the block closes (read_files.f90:5094-5101)."""
    n_species: int
    species: List[str]
    alpha_max: List[int]
    rcut_hard: List[float]
    buffer: List[float]
    nf: List[float]
    atom_sigma_r: List[float]
    atom_sigma_t: List[float]
    atom_sigma_r_scaling: List[float]
    atom_sigma_t_scaling: List[float]
    amplitude_scaling: List[float]
    central_weight: List[float]
    global_scaling: List[float]
    l_max: Optional[int] = None
    radial_enhancement: int = 0
    basis: str = "poly3"
    scaling_mode: str = "polynomial"
    zeta: float = 2.0
    delta: float = 1.0
    central_species: int = 0
    file_desc: Optional[str] = None
    file_alphas: Optional[str] = None
    compress_soap: bool = False
    file_compress: str = "none"
    compress_mode: str = "none"
    has_local_properties: bool = False
    other: Dict[str, List[str]] = field(default_factory=dict)

    @property
    def rcut_soft(self) -> List[float]:
        return [h if b == 0.0 else h - b for h, b in zip(self.rcut_hard, self.buffer)]

    @property
    def rcut_max(self) -> float:
        return max(self.rcut_hard)

    @property
    def n_max(self) -> int:
        return int(sum(self.alpha_max))

    @property
    def uncompressed_dim(self) -> int:
        n = self.n_max
        return n * (n + 1) // 2 * (self.l_max + 1)

    def hypers(self, species_types: Sequence[str]) -> SoapTurboHypers:
        """Hyperparameters with the block's species mapped to 1-based indices
        of the input's ``species`` list (what assign_species_multiplicity and
        get_gap_soap use to match neighbours, gap_interface.f90:195-214)."""
        if self.l_max is None:
            raise ValueError("soap_turbo block without l_max")
        for name, v in (("n_max", self.alpha_max), ("rcut", self.rcut_hard),
                        ("atom_sigma_r", self.atom_sigma_r), ("atom_sigma_t", self.atom_sigma_t)):
            if any(x is None for x in v):
                raise ValueError(f"soap_turbo block without {name}")
        z = []
        for s in self.species:
            if s not in species_types:
                raise ValueError(f"soap_turbo species {s!r} is not among the input species "
                                 f"{list(species_types)}")
            z.append(list(species_types).index(s) + 1)
        return SoapTurboHypers(
            species_z=z, alpha_max=self.alpha_max, l_max=self.l_max, rcut_hard=self.rcut_hard,
            buffer=self.buffer, nf=self.nf, atom_sigma_r=self.atom_sigma_r,
            atom_sigma_t=self.atom_sigma_t, atom_sigma_r_scaling=self.atom_sigma_r_scaling,
            atom_sigma_t_scaling=self.atom_sigma_t_scaling,
            amplitude_scaling=self.amplitude_scaling, central_weight=self.central_weight,
            global_scaling=self.global_scaling, radial_enhancement=self.radial_enhancement,
            central_species=self.central_species, basis=self.basis,
            scaling_mode=self.scaling_mode)

    def compression(self, base_dir: str = ".") -> Optional[SoapCompression]:
        """The compression transformation when compress_soap is set. A file
        takes precedence over compress_mode (read_files.f90:5162-5165). Of the
        named modes (get_compress_indices in soap_turbo, which is not part of
        the reference tree) "trivial" is built as the reference's generator of
        compress files writes it; other modes are refused."""
        if not self.compress_soap:
            return None
        if self.file_compress != "none":
            return read_compress_file(os.path.join(base_dir, self.file_compress),
                                      self.n_species).compression()
        if self.compress_mode == "trivial":
            if self.l_max is None:
                raise ValueError("soap_turbo block without l_max")
            return trivial_compression(self.alpha_max, self.l_max)
        if self.compress_mode != "none":
            raise NotImplementedError(
                f"compress_mode {self.compress_mode!r}: only \"trivial\" is available (the "
                "other recipes live in soap_turbo's get_compress_indices, which is not part "
                "of the reference tree); give a file_compress_soap instead")
        raise ValueError("compress_soap needs file_compress_soap or compress_mode")

    def load(self, species_types: Sequence[str], base_dir: str = ".") -> GapBlock:
        """The block with its sparse set, ready for soap_backend_begin.

        Paths in the file are relative to the directory the run starts in
        (``base_dir``). A compressed block carries its transformation, and its
        sparse descriptors have the compressed dim."""
        h = self.hypers(species_types)
        if self.compress_soap:
            h.compress = self.compression(base_dir)
        if self.file_desc is None or self.file_alphas is None:
            raise ValueError("soap_turbo block without desc_sparse / alphas_sparse")
        alphas, Qs, _ = read_alphas_and_descriptors(os.path.join(base_dir, self.file_desc),
                                                    os.path.join(base_dir, self.file_alphas),
                                                    "soap_turbo")
        if Qs.shape[1] != h.dim:
            raise ValueError(f"sparse descriptors have {Qs.shape[1]} components; the block's "
                             f"dim is {h.dim}")
        return GapBlock(hypers=h, Qs=Qs, alphas=alphas, delta=self.delta, zeta=self.zeta)


@dataclass
class RawGapBlock:
    """A distance_2b, angle_3b or core_pot block: its type and every
    ``keyword = values`` line; ``load`` turns it into the family the device
    evaluates (read_files.f90:5238-5505)."""
    kind: str
    keywords: Dict[str, List[str]]

    def _get(self, names, conv, default, n=1):
        for k in names:
            if k in self.keywords:
                v = _values(["", "="] + self.keywords[k], n, conv, k)
                return v if n > 1 else v[0]
        return default

    def _species(self, names, species_types):
        name = self._get(names, str, None)
        if name is None:
            raise ValueError(f"{self.kind} block without {names[-1]}")
        if name not in species_types:
            raise ValueError(f"{self.kind} species {name!r} is not among the input species "
                             f"{list(species_types)}")
        return list(species_types).index(name) + 1

    def load(self, species_types: Sequence[str], base_dir: str = ".",
             core_pot_cutoff: float = 1e10, core_pot_buffer: float = 1.0):
        from . import families as FM
        s1 = self._species(("Z1", "z1", "species1"), species_types)
        s2 = self._species(("Z2", "z2", "species2"), species_types)
        if self.kind == "core_pot":
            path = self._get(("core_pot_file",), str, None)
            if path is None:
                raise ValueError("core_pot block without core_pot_file")
            return read_core_pot_file(os.path.join(base_dir, path), (s1, s2), core_pot_cutoff,
                                      core_pot_buffer)
        fd = self._get(("desc_sparse",), str, None)
        fa = self._get(("alphas_sparse",), str, None)
        if fd is None or fa is None:
            raise ValueError(f"{self.kind} block without desc_sparse / alphas_sparse")
        rcut = self._get(("rcut",), _real, None)
        if rcut is None:
            raise ValueError(f"{self.kind} block without rcut")
        delta = self._get(("delta",), _real, 1.0)
        alphas, Qs, cut = read_alphas_and_descriptors(os.path.join(base_dir, fd),
                                                      os.path.join(base_dir, fa), self.kind)
        if self.kind == "distance_2b":
            return FM.Distance2b((s1, s2), delta, self._get(("sigma",), _real, 1.0), rcut,
                                 Qs[:, 0], alphas, cut)
        sc = self._species(("Z_center", "z_center", "species_center"), species_types)
        return FM.Angle3b((sc, s1, s2), delta, self._get(("sigma",), _real, [1.0] * 3, 3), rcut,
                          Qs, alphas, cut, self._get(("kernel_type",), str, "exp"))


def read_core_pot_file(path: str, species, cutoff: float = 1e10, buffer: float = 1.0):
    """core_pot table: a record ``n yp1 ypn`` then n records ``x V``
    (read_files.f90:5425-5447), tapered at core_pot_cutoff."""
    from . import families as FM
    recs = _records(path)
    head = _tokens(recs[0])
    n, yp1, ypn = _int(head[0]), _real(head[1]), _real(head[2])
    if len(recs) < n + 1:
        raise ValueError(f"{path}: {n} table records expected")
    xv = [_tokens(recs[1 + i]) for i in range(n)]
    x = [_real(t[0]) for t in xv]
    V = [_real(t[1]) for t in xv]
    return FM.CorePot.from_table(species, x, V, yp1, ypn, cutoff, buffer)


@dataclass
class GapFile:
    soap_turbo: List[SoapTurboSpec]
    distance_2b: List[RawGapBlock]
    angle_3b: List[RawGapBlock]
    core_pot: List[RawGapBlock]

    @property
    def rcut_max(self) -> float:
        """Largest hard cutoff over the soap_turbo blocks and the rcut of the
        others (read_files.f90:5142-5146 and the 2b/3b branches)."""
        r = [s.rcut_max for s in self.soap_turbo]
        for b in self.distance_2b + self.angle_3b:
            if "rcut" in b.keywords:
                r.append(_real(b.keywords["rcut"][0]))
        return max(r) if r else 0.0


_SOAP_LIST_REAL = {
    "nf": "nf", "rcut": "rcut_hard", "buffer": "buffer", "atom_sigma_r": "atom_sigma_r",
    "atom_sigma_t": "atom_sigma_t", "atom_sigma_r_scaling": "atom_sigma_r_scaling",
    "atom_sigma_t_scaling": "atom_sigma_t_scaling", "amplitude_scaling": "amplitude_scaling",
    "central_weight": "central_weight", "global_scaling": "global_scaling",
}


def _parse_soap_block(lines: List[List[str]]) -> SoapTurboSpec:
    # the block is pre-scanned for n_species, which sizes every per-species list
    # (read_files.f90:4633-4675)
    ns = None
    for t in lines:
        if t and t[0] == "n_species":
            ns = _values(t, 1, _int, "n_species")[0]
            break
    if ns is None or ns < 1:
        raise ValueError("soap_turbo block without n_species")
    spec = SoapTurboSpec(
        n_species=ns, species=[""] * ns, alpha_max=[None] * ns, rcut_hard=[None] * ns,
        buffer=[0.5] * ns, nf=[4.0] * ns, atom_sigma_r=[None] * ns, atom_sigma_t=[None] * ns,
        atom_sigma_r_scaling=[0.0] * ns, atom_sigma_t_scaling=[0.0] * ns,
        amplitude_scaling=[1.0] * ns, central_weight=[1.0] * ns, global_scaling=[1.0] * ns)
    for t in lines:
        if not t:
            continue
        k = t[0]
        if k in _SOAP_LIST_REAL:
            setattr(spec, _SOAP_LIST_REAL[k], _values(t, ns, _real, k))
        elif k == "n_max":
            spec.alpha_max = _values(t, ns, _int, k)
        elif k == "species":
            spec.species = _values(t, ns, str, k)
        elif k == "l_max":
            spec.l_max = _values(t, 1, _int, k)[0]
        elif k == "radial_enhancement":
            v = _values(t, 1, _int, k)[0]
            if v < 0 or v > 2:
                warnings.warn("radial_enhancement must be 0, 1 or 2; using 0")
                v = 0
            spec.radial_enhancement = v
        elif k == "basis":
            v = _values(t, 1, str, k)[0]
            if v not in ("poly3", "poly3operator", "poly3gauss"):
                warnings.warn(f"basis {v!r} not understood; using poly3")
                v = "poly3"
            spec.basis = v
        elif k == "scaling_mode":
            v = _values(t, 1, str, k)[0]
            if v != "polynomial":
                warnings.warn(f"scaling_mode {v!r} not understood; using polynomial")
                v = "polynomial"
            spec.scaling_mode = v
        elif k == "zeta":
            spec.zeta = _values(t, 1, _real, k)[0]
        elif k == "delta":
            spec.delta = _values(t, 1, _real, k)[0]
        elif k == "central_species":
            spec.central_species = _values(t, 1, _int, k)[0]
        elif k == "compress_soap":
            spec.compress_soap = _values(t, 1, _logical, k)[0]
        elif k == "file_compress_soap":
            spec.file_compress = _values(t, 1, str, k)[0]
        elif k == "compress_mode":
            spec.compress_mode = _values(t, 1, str, k)[0]
        elif k == "alphas_sparse":
            spec.file_alphas = _values(t, 1, str, k)[0]
        elif k == "desc_sparse":
            spec.file_desc = _values(t, 1, str, k)[0]
        elif k in ("has_local_properties", "has_vdw"):
            spec.has_local_properties = _values(t, 1, _logical, k)[0]
        elif k != "n_species" and len(t) >= 2 and t[1] == "=":
            spec.other[k] = t[2:]
    return spec


def read_gap_file(path: str) -> GapFile:
    """Every block of a ``.gap`` file. Lines whose first item starts with '#'
    or '!' are comments; keywords are case-sensitive, as in the reference."""
    recs = [_tokens(r) for r in _records(path)]
    out = GapFile([], [], [], [])
    i = 0
    while i < len(recs):
        t = recs[i]
        i += 1
        if not t or t[0][:1] in ("#", "!") or t[0] != "gap_beg":
            continue
        kind = t[1] if len(t) > 1 else ""
        body = []
        while i < len(recs) and not (recs[i] and recs[i][0] == "gap_end"):
            body.append(recs[i])
            i += 1
        if i >= len(recs):
            raise ValueError(f"{path}: gap_beg {kind} without gap_end")
        i += 1
        if kind == "soap_turbo":
            out.soap_turbo.append(_parse_soap_block(body))
        elif kind in ("distance_2b", "angle_3b", "core_pot"):
            kw = {b[0]: b[2:] for b in body if len(b) >= 2 and b[1] == "="}
            getattr(out, kind).append(RawGapBlock(kind, kw))
    return out


def read_alphas_and_descriptors(file_desc: str, file_alphas: str, descriptor_type: str):
    """(alphas (n_sparse,), Qs (n_sparse, dim), cutoff (n_sparse,) or None).

    n_sparse is the number of records of the alphas file and dim the number of
    records of the descriptor file over n_sparse; soap_turbo descriptors are
    stored one component per record, sparse point after sparse point
    (read_files.f90:680-721). distance_2b and angle_3b alphas records also
    carry a cutoff; their dim must be 1 and 3 (read_files.f90:722-766)."""
    ra = _records(file_alphas)
    rd = _records(file_desc)
    n_sparse = len(ra)
    if n_sparse == 0:
        raise ValueError(f"{file_alphas}: empty alphas file")
    dim = len(rd) // n_sparse

    def first(rec, path, k):
        t = _tokens(rec)
        if not t:
            raise ValueError(f"{path}: record {k + 1} is empty")
        return t

    if descriptor_type == "soap_turbo":
        alphas = np.array([_real(first(r, file_alphas, k)[0]) for k, r in enumerate(ra)])
        vals = np.array([_real(first(rd[k], file_desc, k)[0]) for k in range(n_sparse * dim)])
        return alphas, vals.reshape(n_sparse, dim), None
    want = {"distance_2b": 1, "angle_3b": 3}.get(descriptor_type)
    if want is None:
        raise ValueError(f"unknown descriptor type {descriptor_type!r}")
    if dim != want:
        raise ValueError(f"bad {descriptor_type} descriptor/alphas files: dim {dim}, expected {want}")
    a = [first(r, file_alphas, k) for k, r in enumerate(ra)]
    alphas = np.array([_real(t[0]) for t in a])
    cutoff = np.array([_real(t[1]) for t in a])
    vals = np.array([_real(first(rd[k], file_desc, k)[0]) for k in range(n_sparse * dim)])
    return alphas, vals.reshape(n_sparse, dim), cutoff


def write_sparse_set(block: GapBlock, file_desc: str, file_alphas: str) -> None:
    """Write a block's sparse set in the layout read_alphas_and_descriptors reads
    (full double precision)."""
    with open(file_alphas, "w") as fh:
        fh.writelines(f"{a!r}\n" for a in block.alphas.tolist())
    with open(file_desc, "w") as fh:
        fh.writelines(f"{q!r}\n" for q in block.Qs.reshape(-1).tolist())


def write_soap_block(fh, spec: SoapTurboSpec) -> None:
    """Write one ``gap_beg soap_turbo`` block in the reference's keyword form."""
    def line(k, v):
        fh.write(f"{k} = {v}\n")

    def lst(v):
        return " ".join(repr(float(x)) for x in v)

    fh.write("gap_beg soap_turbo\n")
    line("n_species", spec.n_species)
    line("species", " ".join(spec.species))
    line("central_species", spec.central_species)
    line("rcut", lst(spec.rcut_hard))
    line("buffer", lst(spec.buffer))
    line("atom_sigma_r", lst(spec.atom_sigma_r))
    line("atom_sigma_t", lst(spec.atom_sigma_t))
    line("atom_sigma_r_scaling", lst(spec.atom_sigma_r_scaling))
    line("atom_sigma_t_scaling", lst(spec.atom_sigma_t_scaling))
    line("amplitude_scaling", lst(spec.amplitude_scaling))
    line("central_weight", lst(spec.central_weight))
    line("global_scaling", lst(spec.global_scaling))
    line("nf", lst(spec.nf))
    line("n_max", " ".join(str(int(a)) for a in spec.alpha_max))
    line("l_max", spec.l_max)
    line("radial_enhancement", spec.radial_enhancement)
    line("basis", spec.basis)
    line("scaling_mode", spec.scaling_mode)
    line("zeta", repr(float(spec.zeta)))
    line("delta", repr(float(spec.delta)))
    if spec.compress_soap:
        line("compress_soap", ".true.")
        if spec.file_compress != "none":
            line("file_compress_soap", f"'{spec.file_compress}'")
        if spec.compress_mode != "none":
            line("compress_mode", spec.compress_mode)
    if spec.file_desc:
        line("desc_sparse", f"'{spec.file_desc}'")
    if spec.file_alphas:
        line("alphas_sparse", f"'{spec.file_alphas}'")
    fh.write("gap_end\n")


def write_compress_file(path: str, comp: SoapCompression, alpha_max: Sequence[int],
                        l_max: int) -> None:
    """A compress file in its ``P_transformation`` form, as read_files.f90:5166-5194
    reads it: alpha_max per species, l_max and dim, then one ``i j value`` line
    per entry between ``P_transformation`` and ``end_transformation``."""
    with open(path, "w") as fh:
        fh.write(" ".join(str(int(a)) for a in alpha_max) + f" {int(l_max)} {comp.dim}\n")
        fh.write("P_transformation\n")
        for i, j, v in zip(comp.P_i.tolist(), comp.P_j.tolist(), comp.P_el.tolist()):
            fh.write(f"{i} {j} {v!r}\n")
        fh.write("end_transformation\n")


def spec_from_block(block: GapBlock, species_types: Sequence[str], file_desc: str,
                    file_alphas: str, file_compress: Optional[str] = None) -> SoapTurboSpec:
    """The file form of a GapBlock whose species_z index ``species_types``. A
    compressed block names the compress file its transformation was written to
    (``write_compress_file``)."""
    h = block.hypers
    if h.compress is not None and not file_compress:
        raise ValueError("a compressed block needs the name of its compress file")
    return SoapTurboSpec(
        n_species=h.n_species, species=[species_types[z - 1] for z in h.species_z],
        alpha_max=list(h.alpha_max), rcut_hard=list(h.rcut_hard), buffer=list(h.buffer),
        nf=list(h.nf), atom_sigma_r=list(h.atom_sigma_r), atom_sigma_t=list(h.atom_sigma_t),
        atom_sigma_r_scaling=list(h.atom_sigma_r_scaling),
        atom_sigma_t_scaling=list(h.atom_sigma_t_scaling),
        amplitude_scaling=list(h.amplitude_scaling), central_weight=list(h.central_weight),
        global_scaling=list(h.global_scaling), l_max=h.l_max,
        radial_enhancement=h.radial_enhancement, basis=h.basis, scaling_mode=h.scaling_mode,
        zeta=float(block.zeta), delta=float(block.delta), central_species=h.central_species,
        file_desc=file_desc, file_alphas=file_alphas, compress_soap=h.compress is not None,
        file_compress=file_compress if h.compress is not None else "none")


# --------------------------------------------------------------------------
# extended XYZ
# --------------------------------------------------------------------------

@dataclass
class Frame:
    """One extended-XYZ structure. lattice rows are the a, b, c vectors (A);
    velocities in A/fs; masses in amu (None when the file has no mass column)."""
    species: List[str]
    positions: np.ndarray
    lattice: np.ndarray
    velocities: Optional[np.ndarray] = None
    masses: Optional[np.ndarray] = None
    fix_atoms: Optional[np.ndarray] = None
    properties: str = ""
    info: Dict[str, str] = field(default_factory=dict)
    arrays: Dict[str, np.ndarray] = field(default_factory=dict)   # other real columns

    @property
    def n(self) -> int:
        return len(self.species)


def _header_pairs(line: str) -> Dict[str, str]:
    """key=value items of a comment line; values may be double-quoted."""
    out: Dict[str, str] = {}
    for m in re.finditer(r'([A-Za-z_][\w\-]*)\s*=\s*("([^"]*)"|\S+)', line):
        out[m.group(1)] = m.group(3) if m.group(3) is not None else m.group(2)
    return out


def _columns(properties: str, with_type: bool = False):
    """(name, first column, width[, type letter]) of each property of a
    Properties string."""
    parts = properties.split(":")
    cols, c = [], 0
    for k in range(0, len(parts) - 2, 3):
        w = int(parts[k + 2])
        cols.append((parts[k].lower(), c, w, parts[k + 1].lower()) if with_type else
                    (parts[k].lower(), c, w))
        c += w
    return cols


def iter_extxyz(path: str) -> Iterator[Frame]:
    """Frames of an extended-XYZ file. Recognised columns, as in read_xyz_line:
    species; pos/positions; vel/velocities; mass/masses; fix_atoms/fix_atom
    (three logicals). Other real columns (forces, local_energy, ...) land in
    ``arrays``; the rest are skipped by their width."""
    recs = _records(path)
    k = 0
    while k < len(recs):
        if not recs[k].strip():
            k += 1
            continue
        n = int(recs[k].split()[0])
        head = recs[k + 1] if k + 1 < len(recs) else ""
        pairs = _header_pairs(head)
        low = {key.lower(): v for key, v in pairs.items()}
        if "lattice" not in low:
            raise ValueError(f"{path}: frame at line {k + 1} has no Lattice (ASE extended XYZ "
                             "is required)")
        lat = np.array([_real(x) for x in low["lattice"].split()], dtype=np.float64)
        if lat.size != 9:
            raise ValueError(f"{path}: Lattice needs 9 numbers")
        props = low.get("properties", "species:S:1:pos:R:3").lower()
        cols = _columns(props)
        species, pos = [], np.zeros((n, 3))
        vel = mass = fix = None
        known = ("species", "pos", "positions", "vel", "velocities", "mass", "masses",
                 "fix_atoms", "fix_atom")
        extra = {name: (c, w) for name, c, w, ty in _columns(props, True)
                 if ty == "r" and name not in known}
        arrays = {name: np.zeros((n, w)) for name, (c, w) in extra.items()}
        for name, c, w in cols:
            if name in ("vel", "velocities"):
                vel = np.zeros((n, 3))
            elif name in ("mass", "masses"):
                mass = np.zeros(n)
            elif name in ("fix_atoms", "fix_atom"):
                fix = np.zeros((n, 3), dtype=bool)
        for i in range(n):
            t = _tokens(recs[k + 2 + i])
            for name, c, w in cols:
                if name == "species":
                    species.append(t[c])
                elif name in ("pos", "positions"):
                    pos[i] = [_real(x) for x in t[c:c + 3]]
                elif name in ("vel", "velocities"):
                    vel[i] = [_real(x) for x in t[c:c + 3]]
                elif name in ("mass", "masses"):
                    mass[i] = _real(t[c])
                elif name in ("fix_atoms", "fix_atom"):
                    fix[i] = [_logical(x) for x in t[c:c + 3]]
            for name, (c, w) in extra.items():
                arrays[name][i] = [_real(x) for x in t[c:c + w]]
        info = {key: v for key, v in pairs.items() if key.lower() not in ("lattice", "properties")}
        arrays = {k: (v[:, 0] if v.shape[1] == 1 else v) for k, v in arrays.items()}
        yield Frame(species, pos, lat.reshape(3, 3), vel, mass, fix, props, info, arrays)
        k += 2 + n


def read_extxyz(path: str) -> List[Frame]:
    return list(iter_extxyz(path))


def _fortran_f(x: float, w: int, d: int) -> str:
    """Fortran Fw.d: right-justified, w asterisks when the number does not fit."""
    s = f"{x:{w}.{d}f}"
    return "*" * w if len(s) > w else s


def write_extxyz(path: str, species: Sequence[str], positions, lattice, *, step: int,
                 time: float, dt: float, temperature: float, pressure: float, virial,
                 velocities=None, forces=None, local_energies=None, masses_amu=None,
                 fix_atoms=None, energy_string: str = "", overwrite: bool = False) -> None:
    """Append (or, at step 0, -1 or with overwrite, start) one frame in the
    layout of write_extxyz (xyz.f90:169-486): the Properties string, then
    Lattice, temperature, pressure, time_step, time, energy, virial, stress,
    volume and step (``i_config`` for negative steps), then one line per atom.
    ``virial`` is the 3x3 tensor; masses are in amu."""
    n = len(species)
    pos = np.asarray(positions, dtype=np.float64).reshape(n, 3)
    lat = np.asarray(lattice, dtype=np.float64).reshape(3, 3)
    vir = np.asarray(virial, dtype=np.float64).reshape(3, 3)
    vel = np.zeros((n, 3)) if velocities is None else np.asarray(velocities).reshape(n, 3)
    frc = np.zeros((n, 3)) if forces is None else np.asarray(forces).reshape(n, 3)
    le = np.zeros(n) if local_energies is None else np.asarray(local_energies).reshape(n)
    fix = np.zeros((n, 3), dtype=bool) if fix_atoms is None else np.asarray(fix_atoms).reshape(n, 3)
    props = ["species:S:1", "pos:R:3", "velocities:R:3", "forces:R:3", "local_energy:R:1"]
    if masses_amu is not None:
        props.append("masses:R:1")
    props.append("fix_atoms:S:3")
    vol = float(np.dot(np.cross(lat[0], lat[1]), lat[2]))

    def tensor(key, m, fmt):
        s = [fmt(m[r, c]) for r in range(3) for c in range(3)]
        # adjustl on the first field: its blanks move behind it (xyz.f90:354)
        return f' {key}="' + s[0].lstrip().ljust(len(s[0])) + "".join(s[1:]) + '"'

    h = " Properties=" + ":".join(props)
    h += tensor("Lattice", lat, lambda x: _fortran_f(x, 16, 10))
    h += " temperature=" + _fortran_f(temperature, 16, 8).strip()
    h += " pressure=" + _fortran_f(pressure, 16, 8).strip()
    h += " time_step=" + _fortran_f(dt, 16, 4).strip()
    h += " time=" + _fortran_f(time, 16, 6).strip()
    h += " energy=" + _fortran_f(float(np.sum(le)), 16, 6).strip()
    if energy_string:
        h += " " + energy_string.strip()
    h += tensor("virial", vir, lambda x: _fortran_f(x, 16, 8))
    h += tensor("stress", -vir / vol, lambda x: _fortran_f(x, 16, 8))
    h += " volume=" + _fortran_f(vol, 16, 6).strip()
    h += f" step={step}" if step >= 0 else f" i_config={-step}"
    lines = [f"{n:8d}\n", h + "\n"]
    f3 = lambda v: " ".join(_fortran_f(x, 16, 8) for x in v)  # noqa: E731
    for i in range(n):
        s = f" {species[i]:<8s} {f3(pos[i])} {f3(vel[i])} {f3(frc[i])} {_fortran_f(le[i], 16, 8)}"
        if masses_amu is not None:
            s += " " + _fortran_f(float(masses_amu[i]), 16, 8)
        s += " " + " ".join("T" if b else "F" for b in fix[i])
        lines.append(s + "\n")
    mode = "w" if (step in (0, -1) or overwrite) else "a"
    with open(path, mode) as fh:
        fh.writelines(lines)


# --------------------------------------------------------------------------
# thermo.log
# --------------------------------------------------------------------------

THERMO_HEADER = ("#     Step             Time      Temperature                E_kin"
                 "                     E_pot             Pressure")


def thermo_row(step: int, time: float, temperature: float, e_kin: float, e_pot: float,
               pressure: float) -> str:
    """One row: (I10, 1X, F16.4, 1X, F16.4, 1X, F20.8, 1X, F20.8, 1X, F20.8)."""
    return (f"{step:10d} {_fortran_f(time, 16, 4)} {_fortran_f(temperature, 16, 4)} "
            f"{_fortran_f(e_kin, 20, 8)} {_fortran_f(e_pot, 20, 8)} {_fortran_f(pressure, 20, 8)}")


def read_thermo(path: str) -> np.ndarray:
    """Rows of a thermo.log as an (n, 6) array (step, time, T, E_kin, E_pot, P)."""
    rows = []
    for r in _records(path):
        t = r.split()
        if not t or t[0].startswith("#") or not t[0].lstrip("-").isdigit():
            continue
        rows.append([float(x) if "*" not in x else np.nan for x in t[:6]])
    return np.array(rows).reshape(-1, 6)


def instant_temperature(e_kin: float, n_sites: int) -> float:
    """T = 2 E_kin / (3 (N - 1) k_B) (turbogap_md.f90:283)."""
    return 2.0 / 3.0 / float(n_sites - 1) / KB_EV * e_kin


def instant_pressure(e_kin: float, n_sites: int, virial, volume: float) -> float:
    """Pressure in bar from the kinetic term and the virial trace
    (turbogap_md.f90:285-288)."""
    t = instant_temperature(e_kin, n_sites)
    vir = np.asarray(virial).reshape(3, 3)
    return (KB_EV * float(n_sites - 1) * t + np.trace(vir) / 3.0) / volume * EV_PER_A3_TO_BAR


# --------------------------------------------------------------------------
# input deck
# --------------------------------------------------------------------------

# keywords whose non-default value changes the dynamics beyond NVE velocity
# Verlet on soap_turbo blocks: (keyword, default, converter)
_OFF_PATH = [
    ("thermostat", "none", str), ("barostat", "none", str), ("optimize", "vv", str),
    ("adaptive_time", False, _logical), ("variable_time_step", False, _logical),
    ("electronic_stopping", False, _logical), ("nonadiabatic_processes", False, _logical),
    ("do_mc", False, _logical), ("n_nested", 0, _int), ("vdw_type", "none", str),
    ("estat_method", "none", str), ("do_exp", False, _logical),
]


@dataclass
class InputDeck:
    """A TurboGAP input file: every ``keyword = values`` line (keywords lower-cased,
    as read_input_file does), with typed access to the MD keywords."""
    keywords: Dict[str, List[str]]
    path: str = ""

    def _get(self, key, conv, default, n=1):
        t = self.keywords.get(key)
        if t is None:
            return default
        vals = _values(["", "="] + t, n, conv, key)
        return vals if n > 1 else vals[0]

    @property
    def base_dir(self) -> str:
        return os.path.dirname(os.path.abspath(self.path)) if self.path else "."

    @property
    def n_species(self) -> int:
        return self._get("n_species", _int, 1)

    @property
    def species(self) -> List[str]:
        v = self._get("species", str, None, self.n_species)
        if v is None:
            raise ValueError("input file without species")
        return [v] if isinstance(v, str) else v

    @property
    def masses_amu(self) -> Optional[List[float]]:
        v = self._get("masses", _real, None, self.n_species)
        return None if v is None else ([v] if isinstance(v, float) else v)

    @property
    def e0(self) -> List[float]:
        v = self._get("e0", _real, None, self.n_species)
        if v is None:
            return [0.0] * self.n_species
        return [v] if isinstance(v, float) else v

    atoms_file = property(lambda s: s._get("atoms_file", str, None))
    pot_file = property(lambda s: s._get("pot_file", str, None))
    md_nsteps = property(lambda s: s._get("md_nsteps", _int, 1))
    md_step = property(lambda s: s._get("md_step", _real, 1.0))
    t_beg = property(lambda s: s._get("t_beg", _real, 300.0))
    velocity_distribution = property(
        lambda s: s._get("velocity_distribution", str, "uniform").lower())
    randomize_velocities = property(lambda s: s._get("randomize_velocities", _logical, False))
    neighbors_buffer = property(lambda s: s._get("neighbors_buffer", _real, 0.0))
    write_thermo = property(lambda s: s._get("write_thermo", _int, 1))
    write_xyz = property(lambda s: s._get("write_xyz", _int, 0))
    core_pot_cutoff = property(lambda s: s._get("core_pot_cutoff", _real, 1e10))
    core_pot_buffer = property(lambda s: s._get("core_pot_buffer", _real, 1.0))
    random_seed = property(lambda s: s._get("random_seed", _int, 0))

    def off_path(self) -> List[str]:
        """Keywords set to something the device MD path does not do."""
        out = []
        for key, default, conv in _OFF_PATH:
            v = self._get(key, conv, default)
            if isinstance(v, str):
                v = v.lower()
            if v != default:
                out.append(f"{key} = {v}")
        return out


def read_input_file(path: str) -> InputDeck:
    kw: Dict[str, List[str]] = {}
    for r in _records(path):
        t = _tokens(r)
        if not t or t[0][:1] in ("#", "!"):
            continue
        if len(t) >= 2 and t[1] == "=":
            kw[t[0].lower()] = t[2:]
    return InputDeck(kw, path)
