"""ctypes front-end of the FP64 CPU oracle (oracle/tg_oracle.cpp).

TEST INFRASTRUCTURE ONLY: it is the checker the CUDA backend is compared with.
Arrays follow the Fortran layout of the reference: ``(3, n)`` arrays are passed
as numpy ``(n, 3)`` C-order (identical memory), neighbour indices are 1-based.

Parity status: geometry, neighbour lists, get_gap_soap remap, GAP kernel and
velocity-Verlet restate the reference Fortran; the SOAP descriptor restates the
published method because the soap_turbo submodule is absent from the
reference tree -- descriptor values are parity unpinned (see tg_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libtg_oracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, OpenMP)."""
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(
            os.path.join(_HERE, "tg_oracle.cpp")):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


class _Hypers(C.Structure):
    _fields_ = [
        ("n_species", C.c_int), ("l_max", C.c_int), ("radial_enhancement", C.c_int),
        ("central_species", C.c_int),
        ("alpha_max", C.POINTER(C.c_int)), ("species_z", C.POINTER(C.c_int)),
        ("rcut_hard", C.POINTER(C.c_double)), ("rcut_soft", C.POINTER(C.c_double)),
        ("nf", C.POINTER(C.c_double)), ("global_scaling", C.POINTER(C.c_double)),
        ("atom_sigma_r", C.POINTER(C.c_double)), ("atom_sigma_r_scaling", C.POINTER(C.c_double)),
        ("atom_sigma_t", C.POINTER(C.c_double)), ("atom_sigma_t_scaling", C.POINTER(C.c_double)),
        ("amplitude_scaling", C.POINTER(C.c_double)), ("central_weight", C.POINTER(C.c_double)),
        ("compress_dim", C.c_int), ("compress_nonzero", C.c_int),
        ("compress_i", C.POINTER(C.c_int)), ("compress_j", C.POINTER(C.c_int)),
        ("compress_el", C.POINTER(C.c_double)),
    ]


class _Block(C.Structure):
    _fields_ = [("hypers", _Hypers), ("n_sparse", C.c_int), ("Qs", C.POINTER(C.c_double)),
                ("alphas", C.POINTER(C.c_double)), ("delta", C.c_double), ("zeta", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_distance.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip]
        L.orc_number_of_unit_cells.argtypes = [_dp, _dp, _dp, C.c_double, _ip]
        L.orc_make_supercell.argtypes = [C.c_int, _dp, _ip, _dp, _dp, _dp, _ip, _dp, _ip]
        L.orc_build_neighbors_list.restype = C.c_int64
        L.orc_build_neighbors_list.argtypes = [C.c_int, _dp, C.c_int, _dp, _dp, _dp, C.c_double,
                                               _ip, _ip, _ip, C.c_int64, _ip, _ip, _dp, _dp, _dp,
                                               _dp, _ip]
        L.orc_soap_dim.argtypes = [C.POINTER(_Hypers)]
        L.orc_poly3_W.argtypes = [C.c_int, _dp]
        L.orc_radial.argtypes = [C.POINTER(_Hypers), C.c_int, C.c_double, C.c_int, _dp, _dp]
        L.orc_angular.argtypes = [C.POINTER(_Hypers), C.c_int, C.c_double, _dp, _dp]
        L.orc_real_ylm.argtypes = [C.c_int, _dp, _dp, C.c_void_p]
        L.orc_get_soap.argtypes = [C.POINTER(_Hypers), C.c_int, _ip, C.c_int, _ip, _dp, _dp, _dp,
                                   C.c_void_p, C.c_void_p]
        L.orc_soap_energy_and_forces.argtypes = [C.c_int, C.c_int, _dp, C.c_void_p, C.c_int, _dp,
                                                 _dp, C.c_double, C.c_double, C.c_double, _ip, _ip,
                                                 _dp, C.c_int, C.c_int, _dp, _dp, _dp]
        L.orc_get_gap_soap.argtypes = [C.POINTER(_Hypers), C.c_int, C.c_int, _ip, _ip, _dp, _dp,
                                       _ip, _ip, C.c_int, _dp, _dp, C.c_double, C.c_double,
                                       C.c_int, _dp, _dp, _dp]
        L.orc_atom_pair_batches.argtypes = [C.c_int, _ip, _dp, C.c_double, C.c_int, C.c_int,
                                            C.c_int, C.c_int, C.c_double, _ip, _ip, _ip, _ip]
        L.orc_velocity_verlet.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double,
                                          _dp, C.c_int]
        L.orc_remove_cm_vel.argtypes = [C.c_int, _dp, _dp]
        L.orc_wrap_pbc.argtypes = [C.c_int, _dp, _dp, _dp, _dp]
        L.orc_evaluate.argtypes = [C.c_int, _dp, _ip, _dp, _dp, _dp, C.c_int, C.POINTER(_Block),
                                   C.c_void_p, C.c_int, C.c_double, C.c_double, _dp, _dp, _dp,
                                   C.POINTER(C.c_int64)]
        L.orc_evaluate_range.argtypes = [C.c_int, _dp, _ip, _dp, _dp, _dp, C.c_int,
                                         C.POINTER(_Block), C.c_void_p, C.c_int, C.c_double,
                                         C.c_double, C.c_int, C.c_int, _dp, _dp, _dp,
                                         C.POINTER(C.c_int64)]
        L.orc_core_pot_spline.argtypes = [C.c_int, _dp, _dp, C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), _dp]
        L.orc_family_energy_forces.argtypes = [C.POINTER(_Family), C.c_int, _ip, _ip, _dp, _dp,
                                               _ip, _ip, C.c_int, _dp, _dp, _dp]
        L.orc_evaluate_full.argtypes = [C.c_int, _dp, _ip, _dp, _dp, _dp, C.c_int,
                                        C.POINTER(_Block), C.c_int, C.POINTER(_Family),
                                        C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int,
                                        C.c_int, _dp, _dp, _dp, C.POINTER(C.c_int64)]
    return _lib


def set_threads(n: int) -> int:
    return lib().orc_set_threads(int(n))


def _f64(x):
    return np.ascontiguousarray(x, dtype=np.float64)


class _Family(C.Structure):
    _pd = C.POINTER(C.c_double)
    _fields_ = [("kind", C.c_int), ("sp", C.c_int * 3), ("delta", C.c_double),
                ("sigma", C.c_double * 3), ("rcut", C.c_double), ("kernel_pol", C.c_int),
                ("n", C.c_int), ("Qs", _pd), ("alphas", _pd), ("cutoff", _pd), ("x", _pd),
                ("V", _pd), ("y2", _pd), ("yp1", C.c_double), ("ypn", C.c_double)]


def core_pot_spline(x, V, yp1, ypn):
    """read_files.f90:5454-5505: (y2, yp1, ypn) of the core_pot table."""
    x, V = _f64(x), _f64(V)
    y2 = np.zeros(len(x))
    a, b = C.c_double(yp1), C.c_double(ypn)
    lib().orc_core_pot_spline(len(x), x, V, C.byref(a), C.byref(b), y2)
    return y2, a.value, b.value


class FamilyC:
    """Keeps the buffers behind an ``orc_family`` alive. ``f`` has ``kind``
    ("distance_2b", "angle_3b" or "core_pot"), ``species`` (global ids) and the
    family's parameters (turbogap_b200.families)."""

    KINDS = {"distance_2b": 1, "angle_3b": 2, "core_pot": 3}

    def __init__(self, f):
        s = _Family()
        s.kind = self.KINDS[f.kind]
        for q, z in enumerate(f.species):
            s.sp[q] = int(z)
        self.keep = []

        def arr(v):
            a = _f64(v)
            self.keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_double))

        if f.kind == "core_pot":
            y2, yp1, ypn = core_pot_spline(f.x, f.V, f.yp1, f.ypn)
            s.n = len(f.x)
            s.x, s.V, s.y2 = arr(f.x), arr(f.V), arr(y2)
            s.yp1, s.ypn = yp1, ypn
        else:
            s.delta = float(f.delta)
            sig = np.atleast_1d(np.asarray(f.sigma, dtype=np.float64))
            for q in range(len(sig)):
                s.sigma[q] = float(sig[q])
            s.rcut = float(f.rcut)
            s.kernel_pol = int(getattr(f, "kernel_type", "exp") == "pol")
            s.n = len(f.alphas)
            # angle_3b Qs (n, 3) row-major numpy is Qs(n, 3) column-major transposed
            Q = np.asarray(f.Qs, dtype=np.float64)
            s.Qs = arr(Q.T.reshape(-1) if Q.ndim == 2 else Q)
            s.alphas, s.cutoff = arr(f.alphas), arr(f.cutoff)
        self.struct = s


def family_energy_forces(f, n_neigh, neighbors_list, rjs, xyz, species, neighbor_species,
                         n_sites0):
    """gap.f90:400-1042 for one family: energies (n_sites), forces (n_sites0, 3),
    virial (3, 3)."""
    fc = FamilyC(f)
    n = len(n_neigh)
    e = np.zeros(n)
    fo = np.zeros((n_sites0, 3))
    v = np.zeros(9)
    lib().orc_family_energy_forces(C.byref(fc.struct), n, _i32(n_neigh), _i32(neighbors_list),
                                   _f64(rjs), _f64(xyz), _i32(species), _i32(neighbor_species),
                                   int(n_sites0), e, fo, v)
    return e, fo, v.reshape(3, 3).T.copy()


def _i32(x):
    return np.ascontiguousarray(x, dtype=np.int32)


class HypersC:
    """Keeps the numpy buffers behind an ``orc_soap_hypers`` alive.

    ``h`` is any object with the soap_turbo hyperparameter attributes
    (``n_species, l_max, radial_enhancement, central_species, alpha_max,
    species_z, rcut_hard, rcut_soft, nf, global_scaling, atom_sigma_r,
    atom_sigma_r_scaling, atom_sigma_t, atom_sigma_t_scaling,
    amplitude_scaling, central_weight``, and optionally ``compress`` with
    ``dim, P_i, P_j, P_el``: 1-based compression entries)."""

    _dfields = ("rcut_hard", "rcut_soft", "nf", "global_scaling", "atom_sigma_r",
                "atom_sigma_r_scaling", "atom_sigma_t", "atom_sigma_t_scaling",
                "amplitude_scaling", "central_weight")

    def __init__(self, h):
        self.keep = {}
        s = _Hypers()
        s.n_species = int(h.n_species)
        s.l_max = int(h.l_max)
        s.radial_enhancement = int(h.radial_enhancement)
        s.central_species = int(h.central_species)
        for name in ("alpha_max", "species_z"):
            a = _i32(getattr(h, name))
            self.keep[name] = a
            setattr(s, name, a.ctypes.data_as(C.POINTER(C.c_int)))
        for name in self._dfields:
            a = _f64(getattr(h, name))
            self.keep[name] = a
            setattr(s, name, a.ctypes.data_as(C.POINTER(C.c_double)))
        comp = getattr(h, "compress", None)
        if comp is not None and len(comp.P_el) > 0:
            s.compress_dim = int(comp.dim)
            s.compress_nonzero = int(len(comp.P_el))
            for name, arr, ct in (("compress_i", _i32(comp.P_i), C.c_int),
                                  ("compress_j", _i32(comp.P_j), C.c_int),
                                  ("compress_el", _f64(comp.P_el), C.c_double)):
                self.keep[name] = arr
                setattr(s, name, arr.ctypes.data_as(C.POINTER(ct)))
        self.struct = s
        self.dim = lib().orc_soap_dim(C.byref(s))

    @property
    def ref(self):
        return C.byref(self.struct)


def get_distance(posi, posj, a, b, c):
    dist = np.zeros(3)
    d = np.zeros(1)
    ish = np.zeros(3, np.int32)
    lib().orc_get_distance(_f64(posi), _f64(posj), _f64(a), _f64(b), _f64(c), dist, d, ish)
    return dist, float(d[0]), ish


def number_of_unit_cells(a, b, c, rcut):
    ind = np.zeros(3, np.int32)
    lib().orc_number_of_unit_cells(_f64(a), _f64(b), _f64(c), float(rcut), ind)
    return ind


def make_supercell(positions, species, a, b, c, indices):
    n = positions.shape[0]
    nrep = int(np.prod(indices))
    pos = np.zeros((n * nrep, 3))
    spc = np.zeros(n * nrep, np.int32)
    lib().orc_make_supercell(n, _f64(positions), _i32(species), _f64(a), _f64(b), _f64(c),
                             _i32(indices), pos, spc)
    return pos, spc


def build_neighbors_list(positions_sc, n_sites, a, b, c, rcut_max, indices, species_sc,
                         do_list=None):
    """neighbors.f90:243-605. Returns dict of n_neigh, neighbors_list (1-based),
    rjs, thetas, phis, xyz (P,3), neighbor_species."""
    nsc = positions_sc.shape[0]
    if do_list is None:
        do_list = np.ones(n_sites, np.int32)
    a, b, c = _f64(a).copy(), _f64(b).copy(), _f64(c).copy()
    cap = n_sites * 48
    while True:
        n_neigh = np.zeros(n_sites, np.int32)
        nl = np.zeros(cap, np.int32)
        rjs = np.zeros(cap)
        th = np.zeros(cap)
        ph = np.zeros(cap)
        xyz = np.zeros((cap, 3))
        ns = np.zeros(cap, np.int32)
        np_ = lib().orc_build_neighbors_list(nsc, _f64(positions_sc), n_sites, a, b, c,
                                             float(rcut_max), _i32(indices), _i32(species_sc),
                                             _i32(do_list), cap, n_neigh, nl, rjs, th, ph, xyz, ns)
        if np_ >= 0:
            break
        cap = -np_
    P = int(np_)
    return dict(n_neigh=n_neigh, neighbors_list=nl[:P], rjs=rjs[:P], thetas=th[:P],
                phis=ph[:P], xyz=xyz[:P], neighbor_species=ns[:P])


def poly3_W(alpha_max):
    W = np.zeros((alpha_max, alpha_max))
    lib().orc_poly3_W(int(alpha_max), W)
    return W


def radial(hc: HypersC, s, r, self_pair=False):
    am = int(hc.keep["alpha_max"][s])
    R = np.zeros(am)
    dR = np.zeros(am)
    lib().orc_radial(hc.ref, int(s), float(r), int(self_pair), R, dR)
    return R, dR


def angular(hc: HypersC, s, r):
    L = hc.struct.l_max
    a = np.zeros(L + 1)
    da = np.zeros(L + 1)
    lib().orc_angular(hc.ref, int(s), float(r), a, da)
    return a, da


def real_ylm(l_max, u, with_grad=False):
    L2 = (l_max + 1) ** 2
    Y = np.zeros(L2)
    dY = np.zeros((L2, 3)) if with_grad else None
    lib().orc_real_ylm(int(l_max), _f64(u), Y, dY.ctypes.data if with_grad else None)
    return (Y, dY) if with_grad else Y


def get_soap(hc: HypersC, n_neigh, mask, rjs, xyz, derivatives=True):
    """soap(n_sites, dim) [row per site], soap_cart_der(P, dim, 3), |p|(n_sites)."""
    n_sites = len(n_neigh)
    P = len(rjs)
    dim = hc.dim
    soap = np.zeros((n_sites, dim))
    sdp = np.zeros(n_sites)
    der = np.zeros((P, dim, 3)) if derivatives else None
    mask_cm = _i32(np.asarray(mask, dtype=np.int32).T.copy())  # (n_species, P) = Fortran (P, ns)
    lib().orc_get_soap(hc.ref, n_sites, _i32(n_neigh), P, mask_cm, _f64(rjs), _f64(xyz), soap,
                       der.ctypes.data if derivatives else None, sdp.ctypes.data)
    return soap, der, sdp


def soap_energy_and_forces(soap, soap_der, Qs, alphas, delta, zeta, e0, n_neigh,
                           neighbors_list, xyz, n_sites0, do_forces=True):
    """gap.f90:66-259. soap (n_sites, D), Qs (M, D), soap_der (P, D, 3)."""
    n_sites, D = soap.shape
    M = Qs.shape[0]
    en = np.zeros(n_sites)
    f = np.zeros((n_sites0, 3))
    vir = np.zeros(9)
    sd = _f64(soap_der) if do_forces else None
    lib().orc_soap_energy_and_forces(D, n_sites, _f64(soap), sd.ctypes.data if do_forces else None,
                                     M, _f64(Qs), _f64(alphas), float(delta), float(zeta),
                                     float(e0), _i32(n_neigh), _i32(neighbors_list), _f64(xyz),
                                     int(n_sites0), int(do_forces), en, f, vir)
    return en, f, vir.reshape(3, 3).T


def get_gap_soap(hc: HypersC, n_total_sites, n_neigh0, neighbors_list0, rjs0, xyz0,
                 species_batch, species_all, Qs, alphas, delta, zeta, do_forces=True):
    """gap_interface.f90:41-480; energies0/forces0 assigned for touched sites."""
    e = np.zeros(n_total_sites)
    f = np.zeros((n_total_sites, 3))
    vir = np.zeros(9)
    lib().orc_get_gap_soap(hc.ref, int(n_total_sites), len(n_neigh0), _i32(n_neigh0),
                           _i32(neighbors_list0), _f64(rjs0), _f64(xyz0), _i32(species_batch),
                           _i32(species_all), Qs.shape[0], _f64(Qs), _f64(alphas), float(delta),
                           float(zeta), int(do_forces), e, f, vir)
    return e, f, vir.reshape(3, 3).T


def atom_pair_batches(n_neigh, rjs, rcut, l_max, n_max, n_soap, n_species, max_gbytes):
    n = len(n_neigh)
    ib, ie, jb, je = (np.zeros(max(n, 1), np.int32) for _ in range(4))
    k = lib().orc_atom_pair_batches(n, _i32(n_neigh), _f64(rjs), float(rcut), int(l_max),
                                    int(n_max), int(n_soap), int(n_species), float(max_gbytes),
                                    ib, ie, jb, je)
    return ib[:k], ie[:k], jb[:k], je[:k]


def velocity_verlet(positions, positions_prev, velocities, forces, forces_prev, masses, dt,
                    dt_prev, first_step):
    """md.f90:226-283, in place on the (n,3) arrays; returns new dt_prev."""
    dtp = np.array([dt_prev], dtype=np.float64)
    lib().orc_velocity_verlet(len(masses), positions, positions_prev, velocities, _f64(forces),
                              forces_prev, _f64(masses), float(dt), dtp, int(first_step))
    return float(dtp[0])


def remove_cm_vel(vel, masses):
    lib().orc_remove_cm_vel(len(masses), vel, _f64(masses))


def wrap_pbc(positions, a, b, c):
    lib().orc_wrap_pbc(positions.shape[0], positions, _f64(a), _f64(b), _f64(c))


def evaluate(positions, species, box, blocks, e0=None, neighbors_buffer=0.0, max_gbytes=1.0,
             site_range=None, families=()):
    """Energies (n), forces (n,3), virial (3,3) of one periodic structure.

    ``blocks``: sequence of objects with ``hypers`` (attributes as HypersC),
    ``Qs`` (M, D), ``alphas`` (M), ``delta``, ``zeta``. ``site_range`` = (beg, end)
    restricts the work to those sites (one MPI rank's share)."""
    n = positions.shape[0]
    box = _f64(box)
    keep = []
    arr = (_Block * len(blocks))()
    for i, b in enumerate(blocks):
        hc = HypersC(b.hypers)
        Qs = _f64(b.Qs)
        al = _f64(b.alphas)
        keep += [hc, Qs, al]
        arr[i].hypers = hc.struct
        arr[i].n_sparse = Qs.shape[0]
        arr[i].Qs = Qs.ctypes.data_as(C.POINTER(C.c_double))
        arr[i].alphas = al.ctypes.data_as(C.POINTER(C.c_double))
        arr[i].delta = float(b.delta)
        arr[i].zeta = float(b.zeta)
    e0a = _f64(e0) if e0 is not None else None
    en = np.zeros(n)
    f = np.zeros((n, 3))
    vir = np.zeros(9)
    npairs = C.c_int64(0)
    beg, end = site_range if site_range is not None else (0, n)
    fams = [FamilyC(q) for q in families]
    farr = (_Family * max(len(fams), 1))()
    for i, q in enumerate(fams):
        farr[i] = q.struct
    rc = lib().orc_evaluate_full(n, _f64(positions), _i32(species), _f64(box[0]), _f64(box[1]),
                                 _f64(box[2]), len(blocks), arr, len(fams), farr,
                                 e0a.ctypes.data if e0a is not None else None,
                                 len(e0a) if e0a is not None else 0, float(neighbors_buffer),
                                 float(max_gbytes), int(beg), int(end), en, f, vir,
                                 C.byref(npairs))
    if rc != 0:
        raise RuntimeError(f"oracle evaluate failed: {rc}")
    return en, f, vir.reshape(3, 3).T, int(npairs.value)


def local_property_predict(soap, Qs, alphas, V0, delta, zeta, soap_cart_der, n_neigh):
    """local_properties.f90:174-294 in numpy. soap (n_sites, D) and Qs (M, D) in
    the same descriptor order; soap_cart_der (P, D, 3) per kept pair, site after
    site (n_neigh). Returns V (n_sites) and V_der (P, 3), zero for clamped sites."""
    K = soap @ Qs.T
    zi = int(round(zeta))
    z = zi if abs(zi - zeta) < 1e-10 else zeta
    Kd = z * K ** (z - 1) * alphas[None, :]
    V = delta ** 2 * (K ** z) @ alphas + V0
    V = np.where(V < 0.0, 0.0, V)
    Qss = delta ** 2 * Kd @ Qs
    der = np.zeros((soap_cart_der.shape[0], 3))
    k = 0
    for i, nn in enumerate(n_neigh):
        for _ in range(nn):
            if V[i] != 0.0:
                der[k] = Qss[i] @ soap_cart_der[k]
            k += 1
    return V, der


def soap_dipole(soap, soap_cart_der, Qs, alphas, delta, zeta, n_neigh):
    """get_soap_dipole (gap.f90:261-398) in numpy: zeta snapped within 1e-5;
    energies = delta^2 K^zeta . alphas (no e0); Qss = zeta delta^2 (K^(zeta-1)
    alphas) Qs; mu_i = Qss_i . soap_cart_der of the site's first (self) pair.
    soap (n_sites, D), Qs (M, D), soap_cart_der (P, D, 3) per kept pair, site
    after site (n_neigh). Returns (dipoles (n_sites, 3), energies (n_sites))."""
    zi = int(zeta)
    z = float(zi) if abs(zeta - zi) < 1e-5 else zeta
    K = soap @ Qs.T
    energies = delta ** 2 * (K ** z) @ alphas
    Qss = z * delta ** 2 * (K ** (z - 1.0) * alphas[None, :]) @ Qs
    mu = np.zeros((soap.shape[0], 3))
    k = 0
    for i, nn in enumerate(n_neigh):
        mu[i] = Qss[i] @ soap_cart_der[k]
        k += nn
    return mu, energies


def poly_cut(x, x_min, x_max):
    """misc.f90:479-494."""
    if x < x_min:
        return 0.0
    if x >= x_max:
        return 1.0
    c = x - (x_max + x_min) / 2.0
    w = x_max - x_min
    return 0.5 + 1.5 * c / w - 2.0 * c ** 3 / w ** 3


def ts_energy_and_forces(hirshfeld_v, hirshfeld_v_cart_der, n_neigh, neighbors_list,
                         neighbor_species, rcut, buffer, rcut_inner, buffer_inner, rjs, xyz,
                         hirshfeld_v_neigh, sR, d, c6_ref, r0_ref, alpha0_ref, n_sites0,
                         mbd_ts_scaling, x_min=0.0, x_max=0.0):
    """get_ts_energy_and_forces (vdw.f90:163-493), statement by statement in
    Python loops (FP64). Pairs-major arrays (xyz, hirshfeld_v_cart_der (P, 3)),
    1-based neighbours and species. Returns (energies, forces (n_sites0, 3),
    virial (3, 3), local virial diagonal (n_sites0, 3))."""
    n_sites = len(n_neigh)
    P = len(neighbors_list)
    rjs = np.asarray(rjs, float)
    # buffer flags (:259-280)
    in_buf = np.zeros(P, bool)
    if buffer > 0.0 or buffer_inner > 0.0:
        for k in range(P):
            if (rcut - buffer < rjs[k] < rcut) or (rcut_inner < rjs[k] < rcut_inner + buffer_inner):
                in_buf[k] = True
    with np.errstate(divide="ignore", invalid="ignore"):
        r6 = 1.0 / rjs ** 6
        r6_der = -6.0 / rjs * r6
    for k in np.nonzero(in_buf)[0]:                  # :287-300, from the unsmoothed r6
        if rjs[k] <= rcut_inner + buffer_inner:
            rb = -(rjs[k] - rcut_inner - buffer_inner) / buffer_inner
            r6_der[k] += 6.0 * r6[k] / (-buffer_inner) * (-rb + rb ** 2)
        else:
            rb = (rjs[k] - rcut + buffer) / buffer
            r6_der[k] += 6.0 * r6[k] / buffer * (-rb + rb ** 2)
    for k in np.nonzero(in_buf)[0]:                  # :302-310
        if rjs[k] <= rcut_inner + buffer_inner:
            rb = (rjs[k] - rcut_inner - buffer_inner) / (-buffer_inner)
        else:
            rb = (rjs[k] - rcut + buffer) / buffer
        r6[k] *= 1.0 - 3.0 * rb ** 2 + 2.0 * rb ** 3
    sp = np.asarray(neighbor_species) - 1
    vn = np.asarray(hirshfeld_v_neigh, float)
    c6_ii_n = np.asarray(c6_ref)[sp] * vn ** 2       # :329-332
    r0_ii_n = np.asarray(r0_ref)[sp] * vn ** (1.0 / 3.0)
    a0_n = np.asarray(alpha0_ref)[sp] * vn
    c6_ij = np.zeros(P)
    r0_ij = np.zeros(P)
    k = 0
    for i in range(n_sites):                         # :341-367
        i2 = (neighbors_list[k] - 1) % n_sites0
        c6_ii = c6_ii_n[k] * mbd_ts_scaling[i2]
        r0_i, a0_i = r0_ii_n[k], a0_n[k]
        c6_ij[k], r0_ij[k] = c6_ii, r0_i
        k += 1
        for _ in range(1, n_neigh[i]):
            j2 = (neighbors_list[k] - 1) % n_sites0
            c6_jj = c6_ii_n[k] * mbd_ts_scaling[j2]
            a0_j = a0_n[k]
            if c6_ii == 0.0 or c6_jj == 0.0:
                c6_ij[k] = 0.0
            else:
                c6_ij[k] = 2.0 * c6_ii * c6_jj / (a0_j / a0_i * c6_ii + a0_i / a0_j * c6_jj)
            r0_ij[k] = r0_i + r0_ii_n[k]
            k += 1
    energies = np.zeros(n_sites)
    f_damp = np.zeros(P)
    exp_damp = np.zeros(P)
    k = 0
    for i in range(n_sites):                         # :375-388
        k += 1
        for _ in range(1, n_neigh[i]):
            if rcut_inner < rjs[k] < rcut:
                with np.errstate(divide="ignore", over="ignore"):
                    exp_damp[k] = np.exp(-d * (rjs[k] / (sR * r0_ij[k]) - 1.0))
                f_damp[k] = 1.0 / (1.0 + exp_damp[k])
                energies[i] += c6_ij[k] * r6[k] * f_damp[k]
            k += 1
    energies *= -0.5
    forces = np.zeros((n_sites0, 3))
    virial = np.zeros((3, 3))
    lvir = np.zeros((n_sites0, 3))
    pf1 = np.zeros(n_sites)
    pf2 = np.zeros(n_sites)
    k = 0
    for i in range(n_sites):                         # :402-421
        i2s = sp[k]
        k += 1
        for _ in range(1, n_neigh[i]):
            if rcut_inner < rjs[k] < rcut:
                pf1[i] += c6_ij[k] * f_damp[k] * r6[k]
                pf2[i] -= (c6_ij[k] * f_damp[k] ** 2 * rjs[k] * r6[k] * exp_damp[k] * d / sR
                           / r0_ij[k] ** 2)
            k += 1
        if hirshfeld_v[i] == 0.0:
            pf1[i] = pf2[i] = 0.0
        else:
            pf1[i] = pf1[i] / hirshfeld_v[i]
            pf2[i] = pf2[i] * r0_ref[i2s] / 3.0 / hirshfeld_v[i] ** (2.0 / 3.0)
    vd = np.asarray(hirshfeld_v_cart_der, float)
    x = np.asarray(xyz, float)
    k = 0
    for i in range(n_sites):                         # :422-486
        i2 = (neighbors_list[k] - 1) % n_sites0
        for _ in range(n_neigh[i]):
            j2 = (neighbors_list[k] - 1) % n_sites0
            if rcut_inner < rjs[k] < rcut:
                pc = poly_cut(rjs[k], x_min, x_max)
                if not np.all(vd[k] == 0.0):
                    f = vd[k] * (pf1[i] + pf2[i])
                    forces[j2] += f
                    lvir[j2] += f * x[k] * pc
                    virial += 0.5 * (np.outer(f, x[k]) + np.outer(x[k], f))
                if r0_ij[k] == 0.0:
                    f = np.zeros(3)
                else:
                    f = (c6_ij[k] / rjs[k] * x[k] * f_damp[k]
                         * (-r6_der[k] - r6[k] * f_damp[k] * exp_damp[k] * d / sR / r0_ij[k]))
                if j2 != i2:
                    forces[i2] += f
                lvir[j2] -= 0.5 * f * x[k] * pc
                virial -= 0.25 * (np.outer(f, x[k]) + np.outer(x[k], f))
            k += 1
    return energies, forces, virial, lvir
