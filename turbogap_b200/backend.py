"""Host-side mirror of TurboGAP's backend seam, running on the CUDA backend.

The procedure names and argument meanings follow the reference modules this
backend replaces (procedure -> reference):

  gpu_context_init / gpu_context_finalize   src/gpu_context.f90:41-58
  gpu_memory_budget_init                    src/gpu_context.f90:100-162
  soap_backend_begin / soap_backend_end     src/gap.f90:49-64
  get_gap_soap                              src/gap_interface.f90:41-480
  get_soap                                  soap_turbo get_soap, called at gap_interface.f90:320-325
  build_neighbors_list                      src/neighbors.f90:243-605
  velocity_verlet                           src/md.f90:226-283
  Engine (device-resident MD step)          turbogap.f90:664-2196 + turbogap_md.f90:161-297

Arrays use the reference's shapes with numpy row-major equivalents: Fortran
(3, n) is numpy (n, 3); Fortran (dim, n) is numpy (n, dim); neighbour indices
are 1-based supercell indices. Errors raise BackendError (the reference stops
or calls turbogap_abort).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import TG_PREC_BF16, TG_PREC_BF16X3, BackendError, check, lib  # noqa: F401
from .hypers import GapBlock, SoapTurboHypers


def _f64(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def _i32(x):
    return np.ascontiguousarray(x, dtype=np.int32)


# --------------------------------------------------------------------- context
def gpu_context_init(rank: int = 0, device: int = 0) -> int:
    """Bind this process to ``device``; returns n_omp (1, as on the CPU path)."""
    n = C.c_int32(0)
    check(lib().tg_context_init(int(rank), int(device), C.byref(n)))
    return int(n.value)


def gpu_context_finalize() -> None:
    check(lib().tg_context_finalize())


def gpu_memory_budget_init() -> float:
    """max_Gbytes_per_process for the SOAP batch planner."""
    g = C.c_double(0.0)
    check(lib().tg_memory_budget(C.byref(g)))
    return float(g.value)


# --------------------------------------------------------------------- blocks
class _HypersC:
    def __init__(self, h: SoapTurboHypers):
        self.keep = []
        s = _lib.TgSoapHypers()
        s.n_species = h.n_species
        s.l_max = h.l_max
        s.radial_enhancement = h.radial_enhancement
        s.central_species = h.central_species

        def iarr(v):
            a = _i32(v)
            self.keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_int32))

        def darr(v):
            a = _f64(v)
            self.keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_double))

        s.alpha_max = iarr(h.alpha_max)
        s.species_z = iarr(h.species_z)
        s.rcut_hard = darr(h.rcut_hard)
        s.rcut_soft = darr(h.rcut_soft)
        s.nf = darr(h.nf)
        s.global_scaling = darr(h.global_scaling)
        s.atom_sigma_r = darr(h.atom_sigma_r)
        s.atom_sigma_r_scaling = darr(h.atom_sigma_r_scaling)
        s.atom_sigma_t = darr(h.atom_sigma_t)
        s.atom_sigma_t_scaling = darr(h.atom_sigma_t_scaling)
        s.amplitude_scaling = darr(h.amplitude_scaling)
        s.central_weight = darr(h.central_weight)
        if h.compress is not None:
            s.dim = h.compress.dim
            s.compress_P_nonzero = len(h.compress.P_el)
            s.compress_P_i = iarr(h.compress.P_i)
            s.compress_P_j = iarr(h.compress.P_j)
            s.compress_P_el = darr(h.compress.P_el)
        self.struct = s


def soap_backend_begin(block: GapBlock, key: int, precision: int = TG_PREC_BF16X3) -> None:
    """Make ``block`` current; its sparse set is uploaded once per ``key``."""
    hc = _HypersC(block.hypers)
    # Qs(dim, n_sparse) column-major == numpy (n_sparse, dim) row-major
    check(lib().tg_soap_begin(int(key), C.byref(hc.struct), block.n_sparse, _f64(block.Qs),
                              _f64(block.alphas), float(block.delta), float(block.zeta),
                              int(precision)))


def soap_backend_end() -> None:
    check(lib().tg_soap_end())


def get_local_property(n_total_sites: int, n_neigh0, neighbors_list0, rjs0, xyz0, species_batch,
                       species_all, v0: float = 0.0, derivatives: bool = True):
    """local_property_predict with the current block as the property model:
    (values of the central sites, dV_i/dr_j per pair (P, 3) or None)."""
    n = len(n_neigh0)
    P = int(np.sum(n_neigh0))
    vals = np.zeros(n)
    der = np.zeros((P, 3)) if derivatives else None
    nc = C.c_int32(0)
    check(lib().tg_get_local_property(int(n_total_sites), n, _i32(n_neigh0), _i32(neighbors_list0),
                                      _f64(rjs0), _f64(xyz0), _i32(species_batch),
                                      _i32(species_all), float(v0), vals,
                                      der.ctypes.data if derivatives else None, C.byref(nc)))
    return vals[:nc.value], der


def get_soap_dipole(n_total_sites: int, n_neigh0, neighbors_list0, rjs0, xyz0, species_batch,
                    species_all):
    """get_soap_dipole (gap.f90:261-398) with the current block as the dipole
    model: (local dipoles mu_i = dE_i/dr_i (n_central, 3), the fictitious local
    energies E_i (n_central)) of the block's central sites."""
    n = len(n_neigh0)
    mu = np.zeros((n, 3))
    en = np.zeros(n)
    nc = C.c_int32(0)
    check(lib().tg_get_soap_dipole(int(n_total_sites), n, _i32(n_neigh0), _i32(neighbors_list0),
                                   _f64(rjs0), _f64(xyz0), _i32(species_batch), _i32(species_all),
                                   mu, en.ctypes.data, C.byref(nc)))
    return mu[:nc.value], en[:nc.value]


def get_ts_energy_and_forces(hirshfeld_v, hirshfeld_v_cart_der, n_neigh, neighbors_list,
                             neighbor_species, rcut, buffer, rcut_inner, buffer_inner, rjs, xyz,
                             hirshfeld_v_neigh, sR, d, c6_ref, r0_ref, alpha0_ref, n_sites0,
                             mbd_ts_scaling=None, do_forces=True, x_min=0.0, x_max=0.0):
    """get_ts_energy_and_forces (vdw.f90:163-493) on the device. Arrays as numpy
    (pairs-major: hirshfeld_v_cart_der and xyz (P, 3)); 1-based neighbours and
    species. Returns (energies (n_sites), forces (n_sites0, 3), virial (3, 3),
    local virial diagonal (n_sites0, 3)); the last three are None without forces."""
    n = len(n_neigh)
    sc = _f64(mbd_ts_scaling) if mbd_ts_scaling is not None else np.ones(n_sites0)
    en = np.zeros(n)
    f = np.zeros((n_sites0, 3)) if do_forces else None
    v = np.zeros(9) if do_forces else None
    lv = np.zeros((n_sites0, 3)) if do_forces else None
    vd = _f64(hirshfeld_v_cart_der) if do_forces else None
    check(lib().tg_get_ts_energy_and_forces(
        n, int(n_sites0), _f64(hirshfeld_v), vd.ctypes.data if do_forces else None, _i32(n_neigh),
        _i32(neighbors_list), _i32(neighbor_species), float(rcut), float(buffer), float(rcut_inner),
        float(buffer_inner), _f64(rjs), _f64(xyz), _f64(hirshfeld_v_neigh), float(sR), float(d),
        len(c6_ref), _f64(c6_ref), _f64(r0_ref), _f64(alpha0_ref), 1 if do_forces else 0,
        float(x_min), float(x_max), sc, en, f.ctypes.data if do_forces else None,
        v.ctypes.data if do_forces else None, lv.ctypes.data if do_forces else None))
    if not do_forces:
        return en, None, None, None
    return en, f, v.reshape(3, 3).T.copy(), lv


_FAMILY_KIND = {"distance_2b": 1, "angle_3b": 2, "core_pot": 3}


def family_begin(family, key: int) -> None:
    """Upload a distance_2b / angle_3b / core_pot family (turbogap_b200.families)
    under ``key``; engines created with the key evaluate it every step."""
    f = _lib.TgFamily()
    f.kind = _FAMILY_KIND[family.kind]
    for q, z in enumerate(family.species):
        f.species[q] = int(z)
    keep = []

    def arr(v):
        a = _f64(v)
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_double))

    if family.kind == "core_pot":
        f.n = len(family.x)
        f.x, f.V = arr(family.x), arr(family.V)
        f.yp1, f.ypn = float(family.yp1), float(family.ypn)
    else:
        f.delta = float(family.delta)
        sig = np.atleast_1d(np.asarray(family.sigma, dtype=np.float64))
        for q in range(len(sig)):
            f.sigma[q] = float(sig[q])
        f.rcut = float(family.rcut)
        f.kernel_type = 1 if getattr(family, "kernel_type", "exp") == "pol" else 0
        f.n = len(family.alphas)
        Q = np.asarray(family.Qs, dtype=np.float64)
        f.Qs = arr(Q.T.reshape(-1) if Q.ndim == 2 else Q)   # Qs(n, 3) column-major
        f.alphas, f.cutoff = arr(family.alphas), arr(family.cutoff)
    check(lib().tg_family_begin(int(key), C.byref(f)))


def get_family(key: int, n_total_sites: int, n_neigh0, neighbors_list0, rjs0, xyz0, species_all,
               energies0: Optional[np.ndarray] = None, forces0: Optional[np.ndarray] = None,
               virial: Optional[np.ndarray] = None):
    """add_*_contribution of one family for one batch: ADDS to energies0
    (n_total_sites), forces0 (n_total_sites, 3) and virial (3, 3, column-major
    order), made here when None, and returns them."""
    e = np.zeros(n_total_sites) if energies0 is None else energies0
    f = np.zeros((n_total_sites, 3)) if forces0 is None else forces0
    v = np.zeros(9) if virial is None else virial.T.reshape(-1).copy()
    check(lib().tg_get_family(int(key), int(n_total_sites), len(n_neigh0), _i32(n_neigh0),
                              _i32(neighbors_list0), _f64(rjs0), _f64(xyz0), _i32(species_all),
                              e, f, v))
    return e, f, v.reshape(3, 3).T.copy()


def get_gap_soap(n_total_sites: int, n_neigh0, neighbors_list0, rjs0, xyz0, species_batch,
                 species_all, energies0: Optional[np.ndarray] = None,
                 forces0: Optional[np.ndarray] = None):
    """Energies, forces and virial of the current block for one batch.

    ``energies0`` (n_total_sites) and ``forces0`` (n_total_sites, 3) are assigned
    for the sites the block touches and left unchanged elsewhere, as in the
    reference; fresh zero arrays are used when not given. Returns
    (energies0, forces0, virial(3,3))."""
    if energies0 is None:
        energies0 = np.zeros(n_total_sites)
    if forces0 is None:
        forces0 = np.zeros((n_total_sites, 3))
    assert energies0.dtype == np.float64 and energies0.flags.c_contiguous
    assert forces0.dtype == np.float64 and forces0.flags.c_contiguous
    vir = np.zeros(9)
    nn = _i32(n_neigh0)
    check(lib().tg_get_gap_soap(int(n_total_sites), len(nn), nn, _i32(neighbors_list0),
                                _f64(rjs0), _f64(xyz0), _i32(species_batch), _i32(species_all),
                                energies0, forces0, vir))
    return energies0, forces0, vir.reshape(3, 3).T.copy()


def get_soap(n_total_sites: int, n_neigh0, neighbors_list0, rjs0, xyz0, species_batch,
             species_all, dim: int):
    """Descriptors (n_central, dim) of the current block's central sites."""
    nn = _i32(n_neigh0)
    out = np.zeros((len(nn), dim))
    nc = C.c_int32(0)
    check(lib().tg_get_soap(int(n_total_sites), len(nn), nn, _i32(neighbors_list0), _f64(rjs0),
                            _f64(xyz0), _i32(species_batch), _i32(species_all), out,
                            C.byref(nc)))
    return out[: nc.value].copy()


# --------------------------------------------------------------------- geometry / MD
def build_neighbors_list(positions_sc, n_sites: int, a, b, c, rcut_max: float, indices,
                         species_sc, do_list=None, cap: Optional[int] = None):
    """Full neighbour lists (self first) as build_neighbors_list returns them."""
    pos = _f64(positions_sc)
    nsc = pos.shape[0]
    a, b, c = _f64(a).copy(), _f64(b).copy(), _f64(c).copy()
    dl = _i32(do_list) if do_list is not None else None
    cap = int(cap) if cap else n_sites * 48
    while True:
        nn = np.zeros(n_sites, np.int32)
        nl = np.zeros(max(cap, 1), np.int32)
        rjs = np.zeros(max(cap, 1))
        th = np.zeros(max(cap, 1))
        ph = np.zeros(max(cap, 1))
        xyz = np.zeros((max(cap, 1), 3))
        ns = np.zeros(max(cap, 1), np.int32)
        P = C.c_int64(0)
        rc = lib().tg_build_neighbors_list(nsc, pos, int(n_sites), a, b, c, float(rcut_max),
                                           _i32(indices), _i32(species_sc),
                                           dl.ctypes.data if dl is not None else None, cap, nn, nl,
                                           rjs, th, ph, xyz, ns, C.byref(P))
        if rc == -3 and P.value > cap:
            cap = int(P.value)
            continue
        check(rc)
        break
    P = int(P.value)
    return dict(n_neigh=nn, neighbors_list=nl[:P], rjs=rjs[:P], thetas=th[:P], phis=ph[:P],
                xyz=xyz[:P], neighbor_species=ns[:P], a_box=a, b_box=b, c_box=c)


def velocity_verlet(positions, positions_prev, velocities, forces, forces_prev, masses, dt,
                    dt_prev, first_step):
    """In place on (n,3) float64 arrays; returns the new dt_prev."""
    dtp = C.c_double(dt_prev)
    check(lib().tg_velocity_verlet(len(masses), positions, positions_prev, velocities,
                                   _f64(forces), forces_prev, _f64(masses), float(dt),
                                   C.byref(dtp), int(first_step)))
    return float(dtp.value)


def _tiles(fn, h):
    t = np.zeros(64, dtype=np.int32)
    nb = C.c_int32(0)
    check(fn(h, t, len(t), C.byref(nb)))
    return [(int(t[2 * k]), int(t[2 * k + 1])) for k in range(nb.value)]


class Engine:
    """Device-resident SOAP-GAP evaluator and NVE integrator for one structure.

    All blocks must have been opened with soap_backend_begin under the keys
    given here. Positions/velocities live on the GPU between calls."""

    def __init__(self, positions, species, masses, box, block_keys: Sequence[int],
                 e0_by_species=None, neighbors_buffer: float = 0.0):
        box = _f64(box)
        self.n = int(np.asarray(positions).shape[0])
        keys = _i32(block_keys)
        e0 = _f64(e0_by_species) if e0_by_species is not None else None
        h = C.c_void_p()
        check(lib().tg_engine_create(self.n, _f64(positions), _i32(species), _f64(masses),
                                     _f64(box[0]), _f64(box[1]), _f64(box[2]), len(keys), keys,
                                     e0.ctypes.data if e0 is not None else None,
                                     len(e0) if e0 is not None else 0, float(neighbors_buffer),
                                     C.byref(h)))
        self._h = h
        self._keep = e0

    def close(self):
        if getattr(self, "_h", None):
            lib().tg_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, positions=None, velocities=None):
        p = _f64(positions) if positions is not None else None
        v = _f64(velocities) if velocities is not None else None
        check(lib().tg_engine_set_state(self._h, p.ctypes.data if p is not None else None,
                                        v.ctypes.data if v is not None else None))

    def compute(self):
        """(energies (n), forces (n,3), virial (3,3)) at the current positions."""
        e = np.zeros(self.n)
        f = np.zeros((self.n, 3))
        v = np.zeros(9)
        check(lib().tg_engine_compute(self._h, e.ctypes.data, f.ctypes.data, v.ctypes.data))
        return e, f, v.reshape(3, 3).T.copy()

    def compute_device(self):
        check(lib().tg_engine_compute_device(self._h))

    def md(self, n_steps: int, dt: float, energies: bool = True):
        """n_steps NVE velocity-Verlet steps; returns (E_pot, E_kin) after them
        (None when ``energies`` is False: nothing is read back)."""
        if not energies:
            check(lib().tg_engine_md(self._h, int(n_steps), float(dt), None, None))
            return None
        ep = C.c_double(0.0)
        ek = C.c_double(0.0)
        check(lib().tg_engine_md(self._h, int(n_steps), float(dt), C.byref(ep), C.byref(ek)))
        return float(ep.value), float(ek.value)

    def graph_kernels(self) -> int:
        n = C.c_int32(0)
        check(lib().tg_engine_graph_kernels(self._h, C.byref(n)))
        return int(n.value)

    @property
    def handle(self):
        return self._h

    PASSES = ("neighbors", "descriptor", "gemm1", "gemm2", "forces", "integrate", "mlp")

    def profile(self, n_steps: int, dt: float) -> dict:
        """Mean ms per step of each pass over n_steps eager MD steps (CUDA events)."""
        ms = np.zeros(8)
        npass = C.c_int32(0)
        check(lib().tg_engine_profile(self._h, int(n_steps), float(dt), ms, C.byref(npass)))
        return {k: float(ms[i]) for i, k in enumerate(self.PASSES)}

    def get_state(self):
        p = np.zeros((self.n, 3))
        v = np.zeros((self.n, 3))
        f = np.zeros((self.n, 3))
        check(lib().tg_engine_get_state(self._h, p.ctypes.data, v.ctypes.data, f.ctypes.data))
        return p, v, f

    def get_frame(self):
        """(positions, velocities, forces, energies, virial) of the last evaluation:
        after MD steps, the positions the forces were evaluated at."""
        p = np.zeros((self.n, 3))
        v = np.zeros((self.n, 3))
        f = np.zeros((self.n, 3))
        e = np.zeros(self.n)
        w = np.zeros(9)
        check(lib().tg_engine_get_frame(self._h, p.ctypes.data, v.ctypes.data, f.ctypes.data,
                                        e.ctypes.data, w.ctypes.data))
        return p, v, f, e, w.reshape(3, 3).T.copy()

    def tiles(self):
        """[(descriptor tile, force tile)] per soap_turbo block, as autotuned."""
        return _tiles(lib().tg_engine_tiles, self._h)

    def neighbor_stats(self):
        """(list rebuilds, evaluations) since creation with neighbors_buffer > 0;
        (-1, -1) when every evaluation rebuilds its lists."""
        b, e = C.c_int64(0), C.c_int64(0)
        check(lib().tg_engine_neighbor_stats(self._h, C.byref(b), C.byref(e)))
        return int(b.value), int(e.value)

    def set_site_range(self, beg: int, end: int):
        """Evaluate only the central sites in [beg, end) (one rank's share)."""
        check(lib().tg_engine_set_site_range(self._h, int(beg), int(end)))

    def set_comm(self, nccl_id: Optional[bytes], n_ranks: int = 1, rank: int = 0):
        """Join (collectively) an NCCL communicator: each evaluation then sums
        forces, energies and virial over the ranks. None leaves it."""
        if nccl_id is None:
            check(lib().tg_engine_set_comm(self._h, None, 0, 0))
            return
        buf = C.create_string_buffer(bytes(nccl_id), 128)
        check(lib().tg_engine_set_comm(self._h, C.cast(buf, C.c_void_p), int(n_ranks), int(rank)))

    def n_pairs(self) -> int:
        n = C.c_int64(0)
        check(lib().tg_engine_n_pairs(self._h, C.byref(n)))
        return int(n.value)

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().tg_engine_stream(self._h, C.byref(s)))
        return int(s.value or 0)


def nccl_unique_id() -> bytes:
    """128 bytes naming a new NCCL communicator (make on one rank, send to all)."""
    buf = C.create_string_buffer(128)
    check(lib().tg_nccl_unique_id(C.cast(buf, C.c_void_p)))
    return buf.raw


def gemm_bf16_tn(A_bf16: np.ndarray, B_bf16: np.ndarray) -> np.ndarray:
    """Test hook: C = A . B^T through the tcgen05 GEMM (uint16 bf16 bit patterns)."""
    M, K = A_bf16.shape
    N = B_bf16.shape[0]
    out = np.zeros((M, N), np.float32)
    check(lib().tgx_gemm_bf16_tn(M, N, K, np.ascontiguousarray(A_bf16, np.uint16),
                                 np.ascontiguousarray(B_bf16, np.uint16), out))
    return out


class Mlp:
    """Ensemble of per-atom energy MLPs for one SOAP block (the learned surrogate).

    Inputs are delta = q - mu rows of the block (the device's descriptor order);
    outputs are per-atom energies (eV) and dE/d(delta). Training, inference and
    the engine's mixed form run on the GPU through libtgb200.so."""

    def __init__(self, dim: int, hidden: int = 256, n_members: int = 4, seed: int = 0):
        h = C.c_void_p()
        check(lib().tg_mlp_create(int(dim), int(hidden), int(n_members), int(seed), C.byref(h)))
        self._h = h
        self.dim, self.hidden, self.n_members = int(dim), int(hidden), int(n_members)

    def close(self):
        if self._h:
            lib().tg_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_member(self, k, W1, b1, W2, b2, w3, b3):
        check(lib().tg_mlp_set_member(self._h, int(k), _f64(W1), _f64(b1), _f64(W2), _f64(b2),
                                      _f64(w3), float(b3)))

    def get_member(self, k):
        H, D = self.hidden, self.dim
        W1, b1, W2 = np.zeros((H, D)), np.zeros(H), np.zeros((H, H))
        b2, w3, b3 = np.zeros(H), np.zeros(H), C.c_double(0.0)
        check(lib().tg_mlp_get_member(self._h, int(k), W1, b1, W2, b2, w3, C.byref(b3)))
        return W1, b1, W2, b2, w3, float(b3.value)

    def set_normalisation(self, sigma_x, mean_e, sigma_e):
        check(lib().tg_mlp_set_normalisation(self._h, float(sigma_x), float(mean_e), float(sigma_e)))

    def normalisation(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        check(lib().tg_mlp_get_normalisation(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def add_samples(self, delta, energy, dedq):
        delta = np.ascontiguousarray(delta, np.float32)
        check(lib().tg_mlp_add_samples(self._h, delta.shape[0], delta, _f64(energy),
                                       np.ascontiguousarray(dedq, np.float32)))

    def add_engine_samples(self, engine: "Engine", block: int):
        check(lib().tg_mlp_add_engine_samples(self._h, engine.handle, int(block)))

    def n_samples(self) -> int:
        n = C.c_int64(0)
        check(lib().tg_mlp_n_samples(self._h, C.byref(n)))
        return int(n.value)

    def train(self, epochs: int, batch: int = 512, lr: float = 1e-3, force_weight: float = 1.0,
              seed: int = 0) -> np.ndarray:
        loss = np.zeros(max(int(epochs), 1))
        check(lib().tg_mlp_train(self._h, int(epochs), int(batch), float(lr), float(force_weight),
                                 int(seed), loss))
        return loss[:int(epochs)]

    def predict(self, delta):
        delta = np.ascontiguousarray(delta, np.float32)
        n = delta.shape[0]
        em, es, g = np.zeros(n), np.zeros(n), np.zeros((n, self.dim))
        check(lib().tg_mlp_predict(self._h, n, delta, em, es, g))
        return em, es, g

    def layout(self):
        o = np.zeros(9, np.int64)
        check(lib().tgx_mlp_layout(self._h, o))
        return dict(zip(("D", "Dp", "H", "W1", "b1", "W2", "b2", "w3", "b3"), map(int, o)))

    def batch_grads(self, member, x, y, gref, lam):
        """Test hook: loss, flat gradients, E and G of one normalised batch."""
        L = self.layout()
        B = x.shape[0]
        n = L["b3"] + 1
        n = (n + 63) // 64 * 64
        grads = np.zeros(n)
        loss = C.c_double(0.0)
        E = np.zeros(B, np.float32)
        G = np.zeros((B, L["Dp"]), np.float32)
        check(lib().tgx_mlp_batch_grads(self._h, int(member), B, np.ascontiguousarray(x, np.float32),
                                        np.ascontiguousarray(y, np.float32),
                                        np.ascontiguousarray(gref, np.float32), float(lam), grads,
                                        C.byref(loss), E, G))
        return float(loss.value), grads, E, G


def engine_set_mlp(engine: "Engine", block: int, mlp: Optional[Mlp], gate_ev: float = 0.005):
    """Run engine block `block` in the mixed form (MLP ensemble, exact GAP where
    the ensemble spread exceeds gate_ev); mlp=None restores the exact form."""
    check(lib().tg_engine_set_mlp(engine.handle, int(block), mlp.handle if mlp else None,
                                  float(gate_ev)))


def engine_mlp_stats(engine: "Engine", block: int):
    g, n = C.c_int32(0), C.c_int32(0)
    check(lib().tg_engine_mlp_stats(engine.handle, int(block), C.byref(g), C.byref(n)))
    return int(g.value), int(n.value)


class Batch:
    """Many independent orthorhombic structures evaluated together (energies,
    forces, per-structure virials), e.g. cells of uneven size."""

    def __init__(self, structures, block_keys: Sequence[int], e0_by_species=None):
        self.n_atoms = np.array([s.n for s in structures], np.int32)
        self.n = int(self.n_atoms.sum())
        self.ns = len(structures)
        pos = np.ascontiguousarray(np.concatenate([s.positions for s in structures]), np.float64)
        sp = np.ascontiguousarray(np.concatenate([s.species for s in structures]), np.int32)
        boxes = np.ascontiguousarray(np.stack([np.asarray(s.box, np.float64).reshape(9)
                                               for s in structures]))
        keys = _i32(block_keys)
        e0 = _f64(e0_by_species) if e0_by_species is not None else None
        h = C.c_void_p()
        check(lib().tg_batch_create(self.ns, self.n_atoms, pos, sp, boxes, len(keys), keys,
                                    e0.ctypes.data if e0 is not None else None,
                                    len(e0) if e0 is not None else 0, C.byref(h)))
        self._h = h
        self._keep = e0

    def tiles(self):
        """[(descriptor tile, force tile)] per soap_turbo block, as autotuned."""
        return _tiles(lib().tg_batch_tiles, self._h)

    def close(self):
        if self._h:
            lib().tg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_positions(self, positions):
        check(lib().tg_batch_set_positions(self._h, _f64(positions)))

    def compute(self):
        e = np.zeros(self.n)
        f = np.zeros((self.n, 3))
        v = np.zeros((self.ns, 3, 3))
        check(lib().tg_batch_compute(self._h, e.ctypes.data, f.ctypes.data, v.ctypes.data))
        return e, f, v

    def compute_device(self):
        check(lib().tg_batch_compute_device(self._h))

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().tg_batch_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def n_pairs(self) -> int:
        n = C.c_int64(0)
        check(lib().tg_batch_n_pairs(self._h, C.byref(n)))
        return int(n.value)

    def graph_kernels(self) -> int:
        n = C.c_int32(0)
        check(lib().tg_batch_graph_kernels(self._h, C.byref(n)))
        return int(n.value)

    def profile(self, n_evals: int) -> dict:
        """Mean ms per evaluation of each pass (eager, CUDA events)."""
        ms = np.zeros(8)
        npass = C.c_int32(0)
        check(lib().tg_batch_profile(self._h, int(n_evals), ms, C.byref(npass)))
        return {k: float(ms[i]) for i, k in enumerate(Engine.PASSES)}
