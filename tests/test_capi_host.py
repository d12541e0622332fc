"""Host-side checks of the C ABI (no GPU needed): every declared symbol is exported,
argument validation reports the reference's error codes before any device work, and the
host-computed pieces (alpha, layouts, the default resample_poly design) equal the oracle."""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    from zkx_dev_b200 import _lib
    try:
        _lib.lib()
    except ImportError as e:
        pytest.skip(str(e))
    return _lib


def header_symbols():
    text = open(os.path.join(ROOT, "include", "zkx_rd.h")).read()
    return sorted(set(re.findall(r"ZKX_API\s+[\w\s\*]+?\b(zkx_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported(L):
    syms = header_symbols()
    assert len(syms) >= 19
    lib = ctypes.CDLL(L.LIB_PATH)
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in include/zkx_rd.h but not exported"
    assert set(syms) <= set(L.SIGNATURES), "ctypes signatures missing for some symbols"


def test_pulse_compression_validation_codes(L):
    lib = L.lib()
    p = ctypes.c_void_p(16)  # never dereferenced: validation fails first
    assert lib.zkx_pulse_compression_c64(p, 0, 16, p, 4, -1, 1, 0, None, p, None) == L.INVALID_SHAPE
    assert lib.zkx_pulse_compression_c64(p, 2, 16, p, 0, -1, 1, 0, None, p, None) == L.INVALID_SHAPE
    assert lib.zkx_pulse_compression_c64(p, 2, 16, p, 4, -1, 1, 7, None, p, None) == L.INVALID_ARGUMENT
    assert lib.zkx_pulse_compression_c64(p, 2, 16, p, 4, -1, 1, 3, None, p, None) == L.INVALID_ARGUMENT
    assert lib.zkx_pulse_compression_c64(p, 2, 16, p, 4, -1, 1, 0, p, p, None) == L.INVALID_ARGUMENT
    # powers of two up to 65536 and any other length up to 32768 are supported
    assert lib.zkx_pulse_compression_c64(p, 2, 40000, p, 4, -1, 1, 0, None, p, None) == L.UNSUPPORTED_OPERATION
    assert b"32768" in lib.zkx_last_error()
    assert lib.zkx_pulse_compression_c64(p, 2, 16, p, 4, 1 << 17, 1, 0, None, p, None) == L.UNSUPPORTED_OPERATION
    assert b"65536" in lib.zkx_last_error()
    assert lib.zkx_fft_c2c_c64(p, 2, 1 << 17, 0, p, None) == L.UNSUPPORTED_OPERATION
    assert lib.zkx_fft_c2c_c64(p, 2, 32769, 0, p, None) == L.UNSUPPORTED_OPERATION
    assert lib.zkx_pulse_compression_c64(None, 2, 16, p, 4, -1, 1, 0, None, p, None) == L.INVALID_ARGUMENT
    assert lib.zkx_pulse_compression_c64(p, 1 << 16, 1 << 16, p, 4, -1, 1, 0, None, p, None) == L.INVALID_SHAPE
    assert b"pulse_compression" in lib.zkx_last_error()


def test_doppler_and_cfar_validation_codes(L):
    lib = L.lib()
    p = ctypes.c_void_p(16)
    assert lib.zkx_pulse_doppler_c64(p, 0, 8, -1, 0, None, p, None, None) == L.INVALID_SHAPE
    assert lib.zkx_pulse_doppler_c64(p, 8, 8, 40000, 0, None, p, None, None) == L.UNSUPPORTED_OPERATION
    assert lib.zkx_pulse_doppler_c64(p, 8, 8, 1 << 17, 0, None, p, None, None) == L.UNSUPPORTED_OPERATION
    assert lib.zkx_pulse_doppler_c64(p, 8, 8, -1, 2, p, p, None, None) == L.INVALID_ARGUMENT
    # window too large for the input: rows <= 2 * (guard + train)
    assert lib.zkx_ca_cfar_f32(p, 2, 20, 100, 2, 2, 8, 8, 1e-3, 0, p, p, None) == L.INVALID_SHAPE
    assert lib.zkx_ca_cfar_f32(p, 2, 100, 100, 2, 2, 0, 8, 1e-3, 0, p, p, None) == L.INVALID_ARGUMENT
    assert lib.zkx_ca_cfar_f32(p, 2, 100, 100, 2, 2, 8, 8, 0.0, 0, p, p, None) == L.INVALID_ARGUMENT
    assert lib.zkx_ca_cfar_f32(p, 2, 100, 100, 2, 2, 8, 8, 1.5, 0, p, p, None) == L.INVALID_ARGUMENT
    assert lib.zkx_ca_cfar_f32(p, 3, 100, 100, 2, 2, 8, 8, 1e-3, 0, p, p, None) == L.INVALID_SHAPE
    assert lib.zkx_ca_cfar_f32(p, 2, 100, 100, 2, 2, 8, 8, 1e-3, 9, p, p, None) == L.INVALID_ARGUMENT


def test_filter_validation_codes(L):
    lib = L.lib()
    p = ctypes.c_void_p(16)
    assert lib.zkx_fir_f32(p, 0, p, 1, 10, None, p, None, None) == L.INVALID_ARGUMENT
    assert lib.zkx_fir_f32(p, 3, p, 0, 10, None, p, None, None) == L.INVALID_SHAPE
    assert lib.zkx_upfirdn_f32(p, 0, p, 1, 10, 1, 1, p, None) == L.INVALID_ARGUMENT
    assert lib.zkx_upfirdn_f32(p, 3, p, 1, 10, 0, 1, p, None) == L.INVALID_ARGUMENT
    lay = L.ResampleLayout()
    assert lib.zkx_resample_poly_layout(10, 0, 1, 0, 0, ctypes.byref(lay)) == L.INVALID_ARGUMENT


@pytest.mark.parametrize("pfa,n", [(1e-6, 416), (1e-3, 128), (0.5, 1), (1.0, 16384), (1e-9, 2)])
def test_cfar_alpha_matches_oracle(L, pfa, n):
    a = ctypes.c_double()
    assert L.lib().zkx_cfar_alpha(pfa, n, ctypes.byref(a)) == 0
    assert a.value == O.cfar_alpha(pfa, n)


@pytest.mark.parametrize("n,nh,up,down", [(100, 5, 2, 1), (1024, 7, 3, 2), (100, 9, 2, 3), (1, 1, 1, 1),
                                          (0, 4, 3, 2), (1 << 20, 127, 3, 2)])
def test_upfirdn_length_matches_oracle(L, n, nh, up, down):
    assert L.lib().zkx_upfirdn_length(n, nh, up, down) == O.upfirdn_length(n, nh, up, down)


@pytest.mark.parametrize("n,up,down", [(100, 3, 2), (10, 2, 1), (100, 2, 3), (1000, 1, 4), (77, 5, 3),
                                       (32, 2, 2), (1 << 20, 3, 2), (50, 6, 4)])
def test_resample_layout_and_design_match_oracle(L, n, up, down):
    lay = L.ResampleLayout()
    assert L.lib().zkx_resample_poly_layout(n, up, down, 0, 0, ctypes.byref(lay)) == 0
    ref = O.resample_poly_layout(n, up, down)
    for f, _ in L.ResampleLayout._fields_:
        assert getattr(lay, f) == getattr(ref, f), f
    if not lay.identity:
        taps = np.zeros(lay.coefficient_count)
        assert L.lib().zkx_resample_poly_design(ctypes.byref(lay), 5.0, taps.ctypes.data) == 0
        np.testing.assert_array_equal(taps, O.resample_poly_design(n, up, down, 5.0))


def test_reference_design_matches_restatement(reference_lib):
    """The reference's own resample_poly on a small case equals the restatement."""
    x = np.random.default_rng(0).standard_normal((2, 300)).astype(np.float32)
    got, is64 = O.ref_resample_poly(x, 3, 2)
    assert is64
    np.testing.assert_array_equal(got, O.resample_poly(x, 3, 2))


def test_reference_doppler_phase_error_grows_with_pulses():
    """The reference's CPU pulse_doppler uses the float-rounded pi inside a double phase
    (radartools_typed.cpp:14,742); the restatement reproduces it (pinned by the published
    digests) and its distance to the exact DFT grows linearly with the pulse count."""
    rng = np.random.default_rng(4)
    errs = []
    for P in (128, 512, 2048):
        x = (rng.standard_normal((P, 8)) + 1j * rng.standard_normal((P, 8))).astype(np.complex64)
        a = O.pulse_doppler_direct(x)
        b, _ = O.pulse_doppler_fft64(x)
        errs.append(np.linalg.norm(a - b) / np.linalg.norm(b))
    assert 3e-6 < errs[0] < 1.5e-5
    assert errs[2] > 8 * errs[0]


def test_wait_timeout_selftest_checks_its_limit(L):
    """The failure-path self-test refuses limits outside 1000 .. 2^31 clocks before any
    device work (so this runs without a GPU)."""
    for bad in (0, 999, (1 << 31) + 1):
        assert L.lib().zkx_selftest_wait_timeout(bad, None) == L.INVALID_ARGUMENT


def test_worklist_and_tuning_validation_codes(L):
    """The work list and the plan-tuning entries reject null and out-of-range arguments with
    the reference's codes before any device work."""
    lib = L.lib()
    h = ctypes.c_void_p()
    assert lib.zkx_rd_worklist_create(None, 1, ctypes.byref(h)) == L.INVALID_ARGUMENT
    items = (L.WorkItem * 1)()
    assert lib.zkx_rd_worklist_create(items, 1, None) == L.INVALID_ARGUMENT
    assert lib.zkx_rd_worklist_create(items, 0, ctypes.byref(h)) == L.INVALID_SHAPE
    assert lib.zkx_rd_worklist_create(items, 70000, ctypes.byref(h)) == L.INVALID_SHAPE
    assert lib.zkx_rd_worklist_launch(None, None) == L.INVALID_ARGUMENT
    assert lib.zkx_rd_worklist_info(None, None, None, None) == L.INVALID_ARGUMENT
    assert lib.zkx_rd_worklist_destroy(None) == L.SUCCESS
    t = L.RdTuning()
    assert lib.zkx_rd_plan_set_tuning(None, ctypes.byref(t)) == L.INVALID_ARGUMENT
    assert lib.zkx_rd_plan_get_tuning(None, ctypes.byref(t)) == L.INVALID_ARGUMENT
