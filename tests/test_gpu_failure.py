"""Failure detection on the GPU without a fault: every bulk-copy wait in the library's
kernels is bounded, and a CTA whose wait runs out records code 1 in the device error word
and returns instead of spinning.  zkx_selftest_wait_timeout makes one such wait run out on
purpose (a barrier armed for bytes that no copy delivers, a limit of 2^20 SM clocks); the
test checks that the kernel returned, that the host reads the code through
zkx_kernel_status, and that the context stays usable afterwards."""
from __future__ import annotations

import time

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zkx_dev_b200 import _lib
    _lib.lib()
    return _lib


def test_bounded_wait_runs_out_and_is_reported(L):
    assert L.kernel_status(clear=True) == 0
    t0 = time.perf_counter()
    L.check(L.lib().zkx_selftest_wait_timeout(1 << 20, None))
    code = L.kernel_status(clear=True)  # synchronises: the kernel has returned
    elapsed = time.perf_counter() - t0
    assert code == 1
    assert elapsed < 5.0
    assert L.kernel_status(clear=True) == 0  # cleared


def test_context_usable_after_a_timeout(L):
    import zkx_dev_b200 as z
    L.check(L.lib().zkx_selftest_wait_timeout(1 << 16, None))
    assert L.kernel_status(clear=True) == 1
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((8, 4096)) + 1j * rng.standard_normal((8, 4096))).astype(np.complex64)
    t = (rng.standard_normal(64) + 1j * rng.standard_normal(64)).astype(np.complex64)
    got = z.pulse_compression(torch.as_tensor(x).cuda(), torch.as_tensor(t).cuda(), normalize=True).cpu().numpy()
    ref = O.pulse_compression_fft64(x, t, -1, True)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-5
    assert L.kernel_status(clear=True) == 0
