"""Failure detection on the GPU without a GPU fault.

Every mbarrier wait of the tcgen05 GEMM is bounded (2 s); when one runs out the
role sets a timeout bit in the device error word, stops issuing and lets the CTA
free its tensor memory and return. The probe silences the GEMM's TMA producer (a
flag that nothing else sets), so the MMA issuer's first wait runs out: the call
must come back with TG_ERR_TIMEOUT and the MMA timeout bit, and the context must
still run a correct GEMM afterwards."""
import ctypes as C

import numpy as np
import pytest

from turbogap_b200._lib import lib

pytestmark = pytest.mark.gpu

TG_ERR_TIMEOUT = -6
DEV_ERR_TIMEOUT_MMA = 1 << 2


def _bf16(x):
    u = np.asarray(x, np.float32).view(np.uint32)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def _f32(u):
    return (u.astype(np.uint32) << 16).view(np.float32)


def test_gemm_wait_runs_out_and_the_context_survives(gpu):
    err = C.c_uint32(0)
    rc = lib().tgx_gemm_stall_probe(256, 256, 128, C.byref(err))
    assert rc == TG_ERR_TIMEOUT, lib().tg_last_error()
    assert err.value & DEV_ERR_TIMEOUT_MMA
    assert b"timed out" in lib().tg_last_error()
    # the same context, the normal path: correct products
    rng = np.random.default_rng(3)
    A = _bf16(rng.normal(size=(300, 128)))
    B = _bf16(rng.normal(size=(260, 128)))
    Cm = gpu.gemm_bf16_tn(A, B)
    ref = _f32(A).astype(np.float64) @ _f32(B).astype(np.float64).T
    assert np.abs(Cm - ref).max() < 4e-6 * np.sqrt(128) * 8
