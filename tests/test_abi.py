"""The C ABI without a GPU: the library loads and exports every declared symbol."""

import re
from pathlib import Path

import numpy as np
import pytest

from solprop_b200 import _lib
from solprop_b200.record import load_record

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols() -> set[str]:
    text = "\n".join(p.read_text() for p in (ROOT / "include").glob("*.h"))
    return set(re.findall(r"\b(sp_[a-z0-9_]+)\s*\(", text))


def test_header_declares_the_bound_functions():
    assert declared_symbols() == set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = _lib.library()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_version_and_error_buffer():
    lib = _lib.library()
    assert b"sm_100a" in lib.sp_version()


def test_problem_descriptor_round_trip_and_refusals():
    rec = load_record(ROOT / "tests" / "golden" / "cap1_ar.problem.npz")
    desc, keep = _lib.problem_desc(rec)
    assert desc.n_to == rec.n_to and desc.n_phi_terms == 1 and desc.band == 1
    assert desc.n_taps == rec.taps.size
    # the problem object validates and copies on the host; no device needed
    problem = _lib.Problem(rec)
    problem.close()
    # the envelope GNLSE with Raman is taken with one mode or two; above 4096 samples, or
    # with plasma, it is refused by name
    env = load_record(ROOT / "tests" / "golden" / "gnlse_raman.problem.npz")
    _lib.Problem(env).close()
    env.n_modes = 2
    env.synthesis = np.ones((1, 2))
    env.projection = np.ones((2, 1))
    env.phi_terms = np.repeat(env.phi_terms, 2, axis=1)
    env.prefactor_terms = np.repeat(env.prefactor_terms, 2, axis=1)
    env.field0 = np.repeat(env.field0, 2, axis=0)
    _lib.Problem(env).close()
    env.plasma_enabled = True
    env.rate_coefficients = np.zeros((4, 1))
    with pytest.raises(_lib.BackendRefusal, match="envelope plasma"):
        _lib.Problem(env)


def test_invalid_descriptor_is_an_argument_error():
    rec = load_record(ROOT / "tests" / "golden" / "cap1_ar.problem.npz")
    rec.n_to = 1000  # not a power of two
    with pytest.raises(_lib.NativeError, match="power of two"):
        _lib.Problem(rec)


def test_batched_tensor_core_product_refuses_what_it_cannot_take():
    """sp_mlp_gemm_tc_batch's argument checks run before any device work: a product count
    outside 1..8, tiles the shapes do not fill, output pitches or operand addresses that its
    16-byte loads and stores cannot take."""
    import ctypes as C

    lib = _lib.library()
    fake = C.c_void_p(0x10000)  # never dereferenced: every call below is refused first
    one = (C.c_void_p * 1)(fake)

    def call(count=1, A=one, W=one, Cout=one, ldc=512, C16=None, ldc16=0, M=128, N=512, K=64,
             lda=64, ldw=64):
        return lib.sp_mlp_gemm_tc_batch(count, A, lda, W, ldw, Cout, ldc, C16, ldc16, M, N, K, None, 1,
                                        fake, None)

    assert call(count=0) == 1 and call(count=9) == 1
    assert call(N=500) == 1 and call(K=96) == 1 and call(lda=60) == 1
    assert call(ldc=510) == 1  # FP32 rows leave as 16-byte stores
    assert call(Cout=None, C16=one, ldc16=500) == 1  # BF16 rows likewise
    odd = (C.c_void_p * 1)(C.c_void_p(0x10008))
    assert call(A=odd) == 1 and call(Cout=odd) == 1
