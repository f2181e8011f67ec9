"""Loader of libtgb200.so, the CUDA backend, with ctypes signatures.

The library is built in-tree (``python -m turbogap_b200.build``). There is no
fallback: if the library or a CUDA device is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtgb200.so")

dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
u16p = np.ctypeslib.ndpointer(dtype=np.uint16, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")

TG_OK = 0
TG_ERR = {-1: "TG_ERR_ARG", -2: "TG_ERR_CUDA", -3: "TG_ERR_CAPACITY", -4: "TG_ERR_STATE",
          -5: "TG_ERR_DEVICE", -6: "TG_ERR_TIMEOUT", -7: "TG_ERR_NOMEM"}
TG_PREC_BF16X3 = 3
TG_PREC_BF16 = 1


class BackendError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{TG_ERR.get(code, code)}: {msg}")
        self.code = code


class TgSoapHypers(C.Structure):
    _fields_ = [
        ("n_species", C.c_int32), ("l_max", C.c_int32), ("radial_enhancement", C.c_int32),
        ("central_species", C.c_int32),
        ("alpha_max", C.POINTER(C.c_int32)), ("species_z", C.POINTER(C.c_int32)),
        ("rcut_hard", C.POINTER(C.c_double)), ("rcut_soft", C.POINTER(C.c_double)),
        ("nf", C.POINTER(C.c_double)), ("global_scaling", C.POINTER(C.c_double)),
        ("atom_sigma_r", C.POINTER(C.c_double)), ("atom_sigma_r_scaling", C.POINTER(C.c_double)),
        ("atom_sigma_t", C.POINTER(C.c_double)), ("atom_sigma_t_scaling", C.POINTER(C.c_double)),
        ("amplitude_scaling", C.POINTER(C.c_double)), ("central_weight", C.POINTER(C.c_double)),
        ("dim", C.c_int32), ("compress_P_nonzero", C.c_int32),
        ("compress_P_i", C.POINTER(C.c_int32)), ("compress_P_j", C.POINTER(C.c_int32)),
        ("compress_P_el", C.POINTER(C.c_double)),
    ]


class TgFamily(C.Structure):
    _pd = C.POINTER(C.c_double)
    _fields_ = [("kind", C.c_int32), ("species", C.c_int32 * 3), ("delta", C.c_double),
                ("sigma", C.c_double * 3), ("rcut", C.c_double), ("kernel_type", C.c_int32),
                ("n", C.c_int32), ("Qs", _pd), ("alphas", _pd), ("cutoff", _pd), ("x", _pd),
                ("V", _pd), ("yp1", C.c_double), ("ypn", C.c_double)]


# (name, restype, argtypes) of every C-ABI entry point in include/tgb200.h and
# include/tgb200_test.h.
_vp = C.c_void_p
SIGNATURES = [
    ("tg_last_error", C.c_char_p, []),
    ("tg_context_init", C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    ("tg_context_finalize", C.c_int, []),
    ("tg_memory_budget", C.c_int, [C.POINTER(C.c_double)]),
    ("tg_soap_begin", C.c_int, [C.c_int32, C.POINTER(TgSoapHypers), C.c_int32, dp, dp,
                                C.c_double, C.c_double, C.c_int32]),
    ("tg_soap_end", C.c_int, []),
    ("tg_get_gap_soap", C.c_int, [C.c_int32, C.c_int32, ip, ip, dp, dp, ip, ip, dp, dp, dp]),
    ("tg_get_soap", C.c_int, [C.c_int32, C.c_int32, ip, ip, dp, dp, ip, ip, dp,
                              C.POINTER(C.c_int32)]),
    ("tg_get_local_property", C.c_int, [C.c_int32, C.c_int32, ip, ip, dp, dp, ip, ip, C.c_double,
                                        dp, _vp, C.POINTER(C.c_int32)]),
    ("tg_get_soap_dipole", C.c_int, [C.c_int32, C.c_int32, ip, ip, dp, dp, ip, ip, dp, _vp,
                                     C.POINTER(C.c_int32)]),
    ("tg_get_ts_energy_and_forces", C.c_int, [C.c_int32, C.c_int32, dp, _vp, ip, ip, ip, C.c_double,
                                              C.c_double, C.c_double, C.c_double, dp, dp, dp,
                                              C.c_double, C.c_double, C.c_int32, dp, dp, dp,
                                              C.c_int32, C.c_double, C.c_double, dp, dp, _vp, _vp,
                                              _vp]),
    ("tg_family_begin", C.c_int, [C.c_int32, C.POINTER(TgFamily)]),
    ("tg_get_family", C.c_int, [C.c_int32, C.c_int32, C.c_int32, ip, ip, dp, dp, ip, dp, dp, dp]),
    ("tg_build_neighbors_list", C.c_int, [C.c_int32, dp, C.c_int32, dp, dp, dp, C.c_double, ip,
                                          ip, _vp, C.c_int64, ip, ip, dp, dp, dp, dp, ip,
                                          C.POINTER(C.c_int64)]),
    ("tg_build_neighbors_list_noalloc", C.c_int, [C.c_int32, _vp, dp, dp, dp, C.c_double,
                                                  C.c_int64, _vp, _vp, _vp, _vp, _vp,
                                                  C.POINTER(C.c_int64), _vp]),
    ("tg_velocity_verlet", C.c_int, [C.c_int32, dp, dp, dp, dp, dp, dp, C.c_double,
                                     C.POINTER(C.c_double), C.c_int32]),
    ("tg_engine_create", C.c_int, [C.c_int32, dp, ip, dp, dp, dp, dp, C.c_int32, ip, _vp,
                                   C.c_int32, C.c_double, C.POINTER(_vp)]),
    ("tg_engine_destroy", C.c_int, [_vp]),
    ("tg_engine_set_state", C.c_int, [_vp, _vp, _vp]),
    ("tg_engine_compute", C.c_int, [_vp, _vp, _vp, _vp]),
    ("tg_engine_md", C.c_int, [_vp, C.c_int32, C.c_double, C.POINTER(C.c_double),
                               C.POINTER(C.c_double)]),
    ("tg_engine_get_state", C.c_int, [_vp, _vp, _vp, _vp]),
    ("tg_engine_get_frame", C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    ("tg_engine_set_site_range", C.c_int, [_vp, C.c_int32, C.c_int32]),
    ("tg_engine_neighbor_stats", C.c_int, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("tg_engine_tiles", C.c_int, [_vp, ip, C.c_int32, C.POINTER(C.c_int32)]),
    ("tg_batch_tiles", C.c_int, [_vp, ip, C.c_int32, C.POINTER(C.c_int32)]),
    ("tg_nccl_unique_id", C.c_int, [_vp]),
    ("tg_engine_set_comm", C.c_int, [_vp, _vp, C.c_int32, C.c_int32]),
    ("tg_engine_n_pairs", C.c_int, [_vp, C.POINTER(C.c_int64)]),
    ("tg_engine_stream", C.c_int, [_vp, C.POINTER(_vp)]),
    ("tg_engine_compute_device", C.c_int, [_vp]),
    ("tg_engine_profile", C.c_int, [_vp, C.c_int32, C.c_double, dp, C.POINTER(C.c_int32)]),
    ("tg_engine_graph_kernels", C.c_int, [_vp, C.POINTER(C.c_int32)]),
    ("tg_mlp_create", C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(_vp)]),
    ("tg_mlp_destroy", C.c_int, [_vp]),
    ("tg_mlp_set_member", C.c_int, [_vp, C.c_int32, dp, dp, dp, dp, dp, C.c_double]),
    ("tg_mlp_get_member", C.c_int, [_vp, C.c_int32, dp, dp, dp, dp, dp, C.POINTER(C.c_double)]),
    ("tg_mlp_set_normalisation", C.c_int, [_vp, C.c_double, C.c_double, C.c_double]),
    ("tg_mlp_get_normalisation", C.c_int, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]),
    ("tg_mlp_add_samples", C.c_int, [_vp, C.c_int32, f32p, dp, f32p]),
    ("tg_mlp_add_engine_samples", C.c_int, [_vp, _vp, C.c_int32]),
    ("tg_mlp_n_samples", C.c_int, [_vp, C.POINTER(C.c_int64)]),
    ("tg_mlp_train", C.c_int, [_vp, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_uint64,
                               dp]),
    ("tg_mlp_predict", C.c_int, [_vp, C.c_int32, f32p, dp, dp, dp]),
    ("tg_engine_set_mlp", C.c_int, [_vp, C.c_int32, _vp, C.c_double]),
    ("tg_engine_mlp_stats", C.c_int, [_vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("tg_batch_create", C.c_int, [C.c_int32, ip, dp, ip, dp, C.c_int32, ip, _vp, C.c_int32,
                                  C.POINTER(_vp)]),
    ("tg_batch_destroy", C.c_int, [_vp]),
    ("tg_batch_set_positions", C.c_int, [_vp, dp]),
    ("tg_batch_compute", C.c_int, [_vp, _vp, _vp, _vp]),
    ("tg_batch_compute_device", C.c_int, [_vp]),
    ("tg_batch_stream", C.c_int, [_vp, C.POINTER(_vp)]),
    ("tg_batch_n_pairs", C.c_int, [_vp, C.POINTER(C.c_int64)]),
    ("tg_batch_profile", C.c_int, [_vp, C.c_int32, dp, C.POINTER(C.c_int32)]),
    ("tg_batch_graph_kernels", C.c_int, [_vp, C.POINTER(C.c_int32)]),
    ("tgx_gemm_bf16_tn", C.c_int, [C.c_int32, C.c_int32, C.c_int32, u16p, u16p, f32p]),
    ("tgx_gemm_stall_probe", C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_uint32)]),
    ("tgx_comm_probe", C.c_int, [_vp, C.c_int32, C.c_int32]),
    ("tgx_mlp_batch_grads", C.c_int, [_vp, C.c_int32, C.c_int32, f32p, f32p, f32p, C.c_double, dp,
                                      C.POINTER(C.c_double), f32p, f32p]),
    ("tgx_mlp_layout", C.c_int, [_vp, i64p]),
]

_lib = None


def lib() -> C.CDLL:
    """The loaded backend; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BackendError(-4, f"{LIB_PATH} is missing: build it with "
                                   "`python -m turbogap_b200.build` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != TG_OK:
        msg = lib().tg_last_error()
        raise BackendError(rc, msg.decode() if msg else "")
