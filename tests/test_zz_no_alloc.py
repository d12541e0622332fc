"""The allocation-free pulse compression entry point (zkx_pulse_compression_c64_noalloc).

It serves callers that cannot let the library allocate device memory (loops that must
not call cudaMalloc/cudaFree while running, hosts whose device memory belongs to another
allocator): its scratch is a fixed device array, so this test checks, through the C ABI,
that two calls in a row give the same result as the allocating entry point and that
calls after the first leave the device's free memory unchanged.  The file is named to be
collected last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL_L2 = 1e-5


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zkx_dev_b200 import _lib
    _lib.lib()
    return _lib


def _call(L, fn, x, t, nfft, window):
    P, N = x.shape
    y = torch.empty((P, nfft), dtype=torch.complex64, device=x.device)
    rc = getattr(L.lib(), fn)(x.data_ptr(), P, N, t.data_ptr(), t.numel(), nfft, 1, window, None,
                              y.data_ptr(), L.stream_handle())
    L.check(rc)
    return y


def _rel(a, b):
    return (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()


def test_noalloc_matches_allocating_entry_twice(L):
    rng = np.random.default_rng(2026)
    cases = [(64, 4096, 256, 4096, L.WINDOW_HAMMING), (32, 16384, 1024, 16384, L.WINDOW_HANN)]
    for P, N, Lr, nfft, win in cases:  # two calls in a row, different transform lengths
        x = torch.as_tensor((rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))).astype(np.complex64)).cuda()
        t = torch.as_tensor((rng.standard_normal(Lr) + 1j * rng.standard_normal(Lr)).astype(np.complex64)).cuda()
        ref = _call(L, "zkx_pulse_compression_c64", x, t, nfft, win)
        got = _call(L, "zkx_pulse_compression_c64_noalloc", x, t, nfft, win)
        torch.cuda.synchronize()
        assert _rel(got, ref) <= REL_L2


def test_noalloc_repeated_calls_allocate_nothing(L):
    rng = np.random.default_rng(7)
    x = torch.as_tensor((rng.standard_normal((16, 2048)) + 1j * rng.standard_normal((16, 2048))).astype(np.complex64)).cuda()
    t = torch.as_tensor((rng.standard_normal(64) + 1j * rng.standard_normal(64)).astype(np.complex64)).cuda()
    y = torch.empty((16, 2048), dtype=torch.complex64, device="cuda")
    lib, sh = L.lib(), L.stream_handle()
    L.check(lib.zkx_pulse_compression_c64_noalloc(x.data_ptr(), 16, 2048, t.data_ptr(), 64, -1, 1,
                                                  L.WINDOW_NONE, None, y.data_ptr(), sh))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        L.check(lib.zkx_pulse_compression_c64_noalloc(x.data_ptr(), 16, 2048, t.data_ptr(), 64, -1, 1,
                                                      L.WINDOW_NONE, None, y.data_ptr(), sh))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_transforms_beyond_its_scratch(L):
    p = ctypes.c_void_p(16)
    rc = L.lib().zkx_pulse_compression_c64_noalloc(p, 2, 32768, p, 8, -1, 1, 0, None, p, None)
    assert rc == L.INVALID_ARGUMENT
    assert b"16384" in L.lib().zkx_last_error()


def test_noalloc_rejects_lengths_that_are_not_powers_of_two(L):
    """The allocating entry point handles other lengths by the chirp-z transform, which
    needs a workspace; this one refuses them (nfft = -1 takes the pulse length, 1000)."""
    p = ctypes.c_void_p(16)
    rc = L.lib().zkx_pulse_compression_c64_noalloc(p, 2, 1000, p, 8, -1, 1, 0, None, p, None)
    assert rc == L.UNSUPPORTED_OPERATION
    assert b"power of two" in L.lib().zkx_last_error()
