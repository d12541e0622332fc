"""Device-side input synthesis: the Task1 waveform and echo against the oracle (noise
bit-identical to the reference's hash, phases within FP32 rounding of FP64) and the CPI
model against numpy FP64 (targets) and a numpy restatement of its counter-based noise; a
device-made CPI runs through the chain and its targets are detected."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def z():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zkx_dev_b200
    return zkx_dev_b200


def test_lfm_waveform(z):
    from zkx_dev_b200 import synth
    L, fs, B = 1000, 2.0e6, 0.8e6
    got = synth.device_lfm(L, fs, B).cpu().numpy()
    T = L / fs
    t = np.arange(L) / fs - 0.5 * T
    ref = np.exp(1j * np.pi * (B / T) * t * t)
    assert np.max(np.abs(got - ref)) <= 2e-7


@pytest.mark.parametrize("P,N,L,delay", [(16, 1024, 128, 300), (33, 700, 64, 0), (8, 512, 512, 0)])
def test_task1_echo_matches_oracle(z, P, N, L, delay):
    from zkx_dev_b200 import synth
    fs, prf, B = 1.0e6, 1.0e4, 0.4e6
    w = synth.device_lfm(L, fs, B)
    fd = 3.0 * prf / P
    noiseless, noise, echo = synth.device_task1_echo(w, P, N, delay, fd, 20260101, prf, fs, 2.5, 0.3)
    ref_clean, ref_noise = O.task1_echo(w.cpu().numpy(), P, N, delay, fd, 20260101, prf, fs, 2.5, 0.3)
    np.testing.assert_array_equal(noise.cpu().numpy(), ref_noise)
    assert np.max(np.abs(noiseless.cpu().numpy() - ref_clean)) <= 2.5 * 3e-7
    e = echo.cpu().numpy()
    c = noiseless.cpu().numpy()
    np.testing.assert_array_equal(e.real, (c.real + ref_noise.real).astype(np.float32))
    np.testing.assert_array_equal(e.imag, (c.imag + ref_noise.imag).astype(np.float32))


def splitmix64(z):
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
    return z ^ (z >> np.uint64(31))


def noise_model(seed, count, power):
    """numpy restatement of the generator's CN(0, power) noise (splitmix64, Box-Muller)."""
    with np.errstate(over="ignore"):
        e = np.arange(count, dtype=np.uint64)
        golden = np.uint64(0x9e3779b97f4a7c15)
        base = np.uint64(seed) + (np.uint64(2) * e + np.uint64(1)) * golden
        a, b = splitmix64(base), splitmix64(base + golden)
    u1 = ((a >> np.uint64(11)).astype(np.float64) + 1.0) * 2.0 ** -53
    u2 = (b >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    r = np.sqrt(-2.0 * np.log(u1)) * np.sqrt(0.5 * power)
    return r * np.cos(2 * np.pi * u2) + 1j * r * np.sin(2 * np.pi * u2)


def test_cpi_model_targets_and_noise(z):
    from zkx_dev_b200 import synth
    P, N, Lc = 64, 4096, 256
    tg = synth.draw_targets(P, N, 12, Lc, seed=77)
    clean = synth.device_cpi(P, N, tg, Lc, seed=5, noise_power=0.0).cpu().numpy()
    s = synth.lfm_chirp(Lc)
    ref = np.zeros((P, N), complex)
    p = np.arange(P)
    for t in tg:
        ramp = 10 ** (t.snr_db / 20) * np.exp(1j * (2 * np.pi * t.doppler_bin * p / P + t.phase))
        ref[:, t.delay:t.delay + Lc] += np.outer(ramp, s)
    assert np.max(np.abs(clean - ref)) / np.max(np.abs(ref)) <= 1e-6
    noise = synth.device_cpi(P, N, [], Lc, seed=5, noise_power=2.0).cpu().numpy()
    model = noise_model(5, P * N, 2.0).reshape(P, N)
    assert np.max(np.abs(noise - model)) <= 1e-5
    assert abs(np.mean(np.abs(noise) ** 2) - 2.0) < 0.05
    both = synth.device_cpi(P, N, tg, Lc, seed=5, noise_power=2.0).cpu().numpy()
    assert np.max(np.abs(both - (ref + model))) <= 1e-4


def test_device_cpi_through_chain_detects_targets(z):
    """A 256 x 8192 CPI made on the device, 20 targets at 15-30 dB: the chain finds every
    target at its (Doppler, range) cell."""
    from zkx_dev_b200 import synth
    P, N, Lc = 256, 8192, 512
    tg = synth.draw_targets(P, N, 20, Lc, seed=3, snr_db=(15.0, 30.0))
    x = synth.device_cpi(P, N, tg, Lc, seed=11)
    rep = torch.as_tensor(synth.lfm_chirp(Lc).astype(np.complex64)).cuda()
    chain = z.RangeDopplerChain(z.ChainConfig(P, N, Lc), rep)
    det = chain(x)["detections"].cpu().numpy()
    assert all(det[t.doppler_bin, t.delay] for t in tg)
