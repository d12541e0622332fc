"""Tensor-core range compression (tcgen05 DFT passes on split hi + lo FP16 / BF16
operands, FP32 accumulation) against the FP64 oracle, and the precision comparison of the
512 x 8192 CPI with near-threshold targets: plain FP32, TC-FP16 and TC-BF16 against FP64,
relative errors and detection masks."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# relative L2 tolerances against the FP64 oracle (the FP32 path is held to 1e-5)
TOL = {"tc_f16": 2e-6, "tc_bf16": 5e-5}
PREC = {"fp32": 0, "tc_f16": 1, "tc_bf16": 2}


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.fixture(scope="module")
def z():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zkx_dev_b200
    return zkx_dev_b200


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def compress(z, x, t, nfft, precision, window="hamming"):
    from zkx_dev_b200 import _lib as L
    xd = dev(x)
    spec = z.replica_spectrum(dev(t), nfft, normalize=True, window=window)
    y = torch.empty((x.shape[0], nfft), dtype=torch.complex64, device="cuda")
    L.check(L.lib().zkx_pulse_compression_spectrum_ex_c64(xd.data_ptr(), x.shape[0], x.shape[1], nfft,
                                                          spec.data_ptr(), PREC[precision], y.data_ptr(),
                                                          L.stream_handle()))
    return y.cpu().numpy()


@pytest.mark.parametrize("precision", ["tc_f16", "tc_bf16"])
@pytest.mark.parametrize("P,N,L,nfft", [(6, 4096, 256, 4096), (5, 8192, 512, 8192), (3, 16384, 1024, 16384),
                                        (4, 5000, 300, 8192), (3, 20000, 700, 16384), (300, 4096, 64, 4096)])
def test_tc_compression_vs_fp64(z, precision, P, N, L, nfft):
    rng = np.random.default_rng(P + N + L)
    x = (rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))).astype(np.complex64)
    t = (rng.standard_normal(L) + 1j * rng.standard_normal(L)).astype(np.complex64)
    ref = O.pulse_compression_fft64(x, t, nfft, True, O.radar_window_f32("hamming", L))
    got = compress(z, x, t, nfft, precision)
    assert rel_l2(got, ref) <= TOL[precision]


@pytest.mark.parametrize("precision", ["tc_f16", "tc_bf16"])
def test_tc_compression_extreme_magnitudes(z, precision):
    """Per-pulse range scaling: a zero pulse, a pulse of 1e-20 values and one of 1e6 values
    keep their relative accuracy (the FP16 range is 6e-5 .. 65504)."""
    rng = np.random.default_rng(3)
    base = (rng.standard_normal((3, 4096)) + 1j * rng.standard_normal((3, 4096)))
    x = (base * np.array([0.0, 1e-20, 1e6])[:, None]).astype(np.complex64)
    t = (rng.standard_normal(100) + 1j * rng.standard_normal(100)).astype(np.complex64)
    ref = O.pulse_compression_fft64(x, t, 4096, True, O.radar_window_f32("hamming", 100))
    got = compress(z, x, t, 4096, precision)
    assert np.all(got[0] == 0)
    for p in (1, 2):
        assert rel_l2(got[p], ref[p]) <= TOL[precision]


def test_tc_rejects_unsupported_length(z):
    from zkx_dev_b200 import _lib as L
    x = torch.zeros((2, 2048), dtype=torch.complex64, device="cuda")
    rc = L.lib().zkx_pulse_compression_spectrum_ex_c64(x.data_ptr(), 2, 2048, 2048, x.data_ptr(), 1,
                                                       x.data_ptr(), None)
    assert rc == L.UNSUPPORTED_OPERATION


def test_c3_precision_chain(z):
    """512 x 8192 CPI, 40 targets (5% at 0-3 dB), 512-sample chirp: the chain with each
    compression arithmetic against the FP64 oracle.  Every mask equals the FP64 CFAR of
    its own power; FP32 and TC-FP16 compressed cubes stay within 1e-5 of FP64."""
    from zkx_dev_b200.synth import make_cpi, seed_for
    cpi = make_cpi(512, 8192, 40, 512, seed_for(3), low_snr_fraction=0.05)
    w_r = O.radar_window_f32("hamming", 512)
    w_d = O.radar_window_f32("hamming", 512)
    comp64 = O.pulse_compression_fft64(cpi.x, cpi.replica, -1, True, w_r)
    rd64, pow64 = O.pulse_doppler_fft64(comp64, -1, w_d)
    _, m64 = O.ca_cfar_f64(pow64.astype(np.float32), (2, 2), (8, 8), 1e-6)
    errors = {}
    for name in ("fp32", "tc_f16", "tc_bf16"):
        chain = z.RangeDopplerChain(z.ChainConfig(512, 8192, 512, precision=name), dev(cpi.replica))
        out = chain(dev(cpi.x))
        torch.cuda.synchronize()
        comp = out["compressed"].cpu().numpy()
        power = out["power"].cpu().numpy()
        det = out["detections"].cpu().numpy()
        errors[name] = (rel_l2(comp, comp64), rel_l2(out["rd"].cpu().numpy(), rd64),
                        int(np.sum(det != m64)))
        _, m_own = O.ca_cfar_f64(power, (2, 2), (8, 8), 1e-6)
        np.testing.assert_array_equal(det, m_own)
    assert errors["fp32"][0] <= 1e-5 and errors["tc_f16"][0] <= 1e-5
    assert errors["tc_bf16"][0] <= TOL["tc_bf16"]
    print("C3 errors (compressed rel L2, rd rel L2, mask cells differing from FP64):", errors)
