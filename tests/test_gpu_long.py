"""Range transforms of 32768 and 65536 points (thread-block clusters of two and four
CTAs): batched FFT rows against numpy's FP64 FFT, pulse compression against the FP64
oracle (zero padding and truncation included), and the whole chain at 64 x 32768."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL_L2 = 1e-5        # FP32 path vs FP64 oracle, relative L2
FFT_REL_L2 = 2e-6    # one FP32 transform vs FP64


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.fixture(scope="module")
def z():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zkx_dev_b200
    return zkx_dev_b200


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def cplx(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


@pytest.mark.parametrize("n", [32768, 65536])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft_rows_long(z, n, inverse):
    rng = np.random.default_rng(n + inverse)
    x = cplx(rng, 3, n)
    got = z.fft(dev(x), inverse=inverse).cpu().numpy()
    ref = np.fft.ifft(x.astype(np.complex128), axis=1) if inverse else np.fft.fft(x.astype(np.complex128), axis=1)
    assert rel_l2(got, ref) <= FFT_REL_L2


@pytest.mark.parametrize("n", [32768, 65536])
def test_fft_rows_long_in_place_round_trip(z, n):
    rng = np.random.default_rng(3)
    x = dev(cplx(rng, 5, n))
    y = x.clone()
    z.fft(y, out=y)
    z.fft(y, inverse=True, out=y)
    assert (torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x)).item() <= FFT_REL_L2


@pytest.mark.parametrize("P,N,L,nfft", [(3, 32768, 2048, -1), (2, 65536, 4096, -1),
                                        (2, 40000, 1000, 65536), (2, 70000, 333, 32768),
                                        (1, 20000, 64, 32768)])
@pytest.mark.parametrize("window", ["none", "hamming"])
def test_pulse_compression_long(z, P, N, L, nfft, window):
    rng = np.random.default_rng(P + N + L)
    x, t = cplx(rng, P, N), cplx(rng, L)
    w = O.radar_window_f32(window, L) if window != "none" else None
    ref = O.pulse_compression_fft64(x, t, nfft, True, w)
    got = z.pulse_compression(dev(x), dev(t), normalize=True,
                              window=None if window == "none" else window,
                              nfft=None if nfft == -1 else nfft).cpu().numpy()
    assert got.shape == ref.shape
    assert rel_l2(got, ref) <= REL_L2


def test_pulse_compression_long_spectrum_path(z):
    """A resident spectrum (cluster order) gives the same result as the one-call form."""
    rng = np.random.default_rng(9)
    x, t = dev(cplx(rng, 4, 65536)), dev(cplx(rng, 4096))
    spec = z.replica_spectrum(t, 65536, normalize=True, window="hann")
    a = z.pulse_compression(x, t, normalize=True, window="hann")
    b = z.pulse_compression(x, None, spectrum=spec, nfft=65536)
    assert torch.equal(a, b)


@pytest.mark.parametrize("n", [32768, 65536])
def test_pulse_compression_long_identity_replica(z, n):
    """Size-independent property on 256 pulses: a unit replica leaves every pulse unchanged."""
    rng = np.random.default_rng(n)
    x = dev(cplx(rng, 256, n))
    one = dev(np.array([1.0 + 0j], dtype=np.complex64))
    y = z.pulse_compression(x, one, normalize=True)
    assert (torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x)).item() <= 1e-6


def test_chain_long_range_against_fp64(z):
    """64 x 32768 CPI with a 2048-sample chirp through the chain (batched, two CPIs):
    every stage against the FP64 oracle and the mask against an FP64 CFAR of the GPU's
    own power."""
    from zkx_dev_b200.synth import make_cpi
    cpis = [make_cpi(64, 32768, 12, 2048, seed=41 + b) for b in range(2)]
    chain = z.RangeDopplerChain(z.ChainConfig(64, 32768, 2048), dev(cpis[0].replica))
    out = chain.run_batch(dev(np.stack([c.x for c in cpis])))
    torch.cuda.synchronize()
    w_r = O.radar_window_f32("hamming", 2048)
    w_d = O.radar_window_f32("hamming", 64)
    for b, cpi in enumerate(cpis):
        comp64 = O.pulse_compression_fft64(cpi.x, cpi.replica, -1, True, w_r)
        rd64, pow64 = O.pulse_doppler_fft64(comp64, -1, w_d)
        assert rel_l2(out["compressed"][b].cpu().numpy(), comp64) <= REL_L2
        assert rel_l2(out["rd"][b].cpu().numpy(), rd64) <= REL_L2
        power = out["power"][b].cpu().numpy()
        assert rel_l2(power, pow64) <= REL_L2
        _, m64 = O.ca_cfar_f64(power, (2, 2), (8, 8), 1e-6)
        np.testing.assert_array_equal(out["detections"][b].cpu().numpy(), m64)
