"""Transforms of any length through libzkx_rd.so: lengths that are not powers of two (the
chirp-z path, which the reference's FFT backend also switches to for such lengths,
backends/fft/fft_thrust.cu:702-765) and power-of-two Doppler transforms above the
single-CTA kernel, against FP64 DFTs, the oracle and the reference's own CPU functions.

Tolerance: relative L2 <= 1e-5 against the exact FP64 transform, the FP32 path's parity
bar; CFAR masks exactly equal to an FP64 CFAR of the GPU's own power."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL_L2 = 1e-5


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


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


# ------------------------------------------------------------------ batched FFT

@pytest.mark.parametrize("rows,n", [(3, 3), (2, 5), (4, 6), (4, 12), (7, 100), (2, 1000), (3, 3000),
                                    (1, 12345), (2, 20000), (1, 32767), (33, 17), (2, 24576)])
def test_fft_any_length(z, rows, n):
    rng = np.random.default_rng(rows * 100003 + n)
    x = cplx(rng, rows, n)
    x64 = x.astype(np.complex128)
    got = z.fft(dev(x)).cpu().numpy()
    assert rel_l2(got, np.fft.fft(x64, axis=1)) <= REL_L2
    inv = z.fft(dev(x), inverse=True).cpu().numpy()
    assert rel_l2(inv, np.fft.ifft(x64, axis=1)) <= REL_L2


def test_fft_any_length_in_place_round_trip(z):
    rng = np.random.default_rng(9)
    x = cplx(rng, 64, 1500)
    t = dev(x)
    z.fft(t, out=t)
    z.fft(t, inverse=True, out=t)
    assert rel_l2(t.cpu().numpy(), x) <= REL_L2


def test_fft_any_length_many_rows_span_passes(z):
    """Rows beyond one 256 MB workspace pass (n = 20000 -> 65536-point convolutions,
    512 rows per pass): sampled rows against FP64, every row through a round trip."""
    rng = np.random.default_rng(11)
    x = cplx(rng, 1200, 20000)
    t = dev(x)
    y = z.fft(t)
    rows = [0, 1, 511, 512, 1023, 1024, 1199]
    assert rel_l2(y[rows].cpu().numpy(), np.fft.fft(x[rows].astype(np.complex128), axis=1)) <= REL_L2
    back = z.fft(y, inverse=True).cpu().numpy()
    assert rel_l2(back, x) <= REL_L2


# ------------------------------------------------------------ pulse compression

@pytest.mark.parametrize("P,N,L,nfft", [(4, 1000, 100, -1), (3, 3000, 64, 5000), (2, 20000, 200, -1),
                                        (5, 100, 128, -1), (2, 4096, 64, 6000), (3, 5000, 50, 3000),
                                        (1, 30000, 300, -1), (6, 7, 3, -1)])
@pytest.mark.parametrize("window", ["none", "hamming"])
def test_pulse_compression_any_length(z, P, N, L, nfft, window):
    rng = np.random.default_rng(P * 1000 + N + L)
    x, t = cplx(rng, P, N), cplx(rng, L)
    ref = O.pulse_compression_direct(x, t, nfft, True, window)
    got = z.pulse_compression(dev(x), dev(t), normalize=True,
                              window=None if window == "none" else window,
                              nfft=None if nfft == -1 else nfft).cpu().numpy()
    assert got.shape == ref.shape
    assert rel_l2(got, ref) <= REL_L2


def test_pulse_compression_any_length_against_reference_cpu(z):
    if O.reference() is None:
        pytest.skip("reference CPU library not built")
    rng = np.random.default_rng(5)
    x, t = cplx(rng, 3, 1500), cplx(rng, 90)
    ref, _ = O.ref_pulse_compression(x, t, 2500, True, "hann")
    got = z.pulse_compression(dev(x), dev(t), normalize=True, window="hann", nfft=2500).cpu().numpy()
    assert rel_l2(got, ref) <= REL_L2


# ------------------------------------------------------------------ Doppler

def doppler64(x, nfft, window):
    P = x.shape[0]
    w = np.ones(P) if window == "none" else O.radar_window_f32(window, P).astype(np.float64)
    nf = P if nfft == -1 else nfft
    return np.fft.fft(x.astype(np.complex128) * w[:, None], n=nf, axis=0)


@pytest.mark.parametrize("P,N,nfft", [(100, 64, -1), (48, 33, 100), (300, 20, 250), (3, 5, -1),
                                      (1000, 7, -1), (8192, 4, -1), (5000, 3, -1), (20000, 2, -1),
                                      (64, 40, 6000), (65536, 1, -1), (96, 1000, -1)])
@pytest.mark.parametrize("window", ["none", "hamming"])
def test_pulse_doppler_any_length(z, P, N, nfft, window):
    rng = np.random.default_rng(P + 7 * N)
    x = cplx(rng, P, N)
    exact = doppler64(x, nfft, window)
    got, power = z.pulse_doppler(dev(x), window=None if window == "none" else window,
                                 nfft=None if nfft == -1 else nfft, return_power=True)
    got = got.cpu().numpy()
    assert got.shape == exact.shape
    assert rel_l2(got, exact) <= REL_L2
    assert rel_l2(power.cpu().numpy(), np.abs(got.astype(np.complex128)) ** 2) <= 1e-6
    if P <= 128 and (nfft == -1 or nfft <= 128):
        # the reference's restated CPU function (float-rounded pi in the phase)
        assert rel_l2(got, O.pulse_doppler_direct(x, nfft, window)) <= REL_L2


# ------------------------------------------------------------------ chain

@pytest.mark.parametrize("P,N,batch", [(100, 1000, 1), (96, 3000, 3), (24, 500, 2)])
def test_chain_any_length_against_fp64(z, P, N, batch):
    """The range-Doppler chain with both transform lengths not powers of two: every stage
    against FP64 and the mask against an FP64 CFAR of the GPU's own power, one launch per
    stage over the batch."""
    from zkx_dev_b200.synth import make_cpi
    cpis = [make_cpi(P, N, 6, 64, seed=100 + b) for b in range(batch)]
    replica = cpis[0].replica
    chain = z.RangeDopplerChain(z.ChainConfig(P, N, 64, guard_cells=(1, 2), reference_cells=(4, 8)),
                                dev(replica))
    out = chain.run_batch(dev(np.stack([c.x for c in cpis])))
    torch.cuda.synchronize()
    for b, c in enumerate(cpis):
        comp64 = O.pulse_compression_direct(c.x, replica, -1, True, "hamming")
        rd64 = doppler64(comp64, -1, "hamming")
        comp = out["compressed"][b].cpu().numpy()
        rd = out["rd"][b].cpu().numpy()
        power = out["power"][b].cpu().numpy()
        assert rel_l2(comp, comp64) <= REL_L2
        assert rel_l2(rd, rd64) <= REL_L2
        _, m64 = O.ca_cfar_f64(power, (1, 2), (4, 8), 1e-6)
        np.testing.assert_array_equal(out["detections"][b].cpu().numpy(), m64)


def test_serving_any_length_equals_alone(z):
    """A non-power-of-two CPI submitted to the serving loop next to power-of-two ones gives
    the result of the same CPI through the chain alone."""
    from zkx_dev_b200.synth import make_cpi
    shapes = [(100, 1000), (64, 1024), (100, 1000), (48, 3000)]
    cpis = [make_cpi(P, N, 5, N // 16, seed=300 + i) for i, (P, N) in enumerate(shapes)]
    replicas = {}
    with z.RdServer(z.ServerConfig()) as server:
        tickets = []
        for (P, N), c in zip(shapes, cpis):
            if (P, N) not in replicas:
                replicas[(P, N)] = dev(c.replica)
            det = torch.empty((P, N), dtype=torch.uint8, device="cuda")
            t = server.submit(dev(c.x), replicas[(P, N)], waveform_id=P * 100000 + N, detections=det)
            tickets.append((t, det))
        for t, _ in tickets:
            server.wait(t)
    for ((P, N), c), (_, det) in zip(zip(shapes, cpis), tickets):
        chain = z.RangeDopplerChain(z.ChainConfig(P, N, N // 16), replicas[(P, N)])
        ref = chain.run(dev(c.x))["detections"]
        torch.cuda.synchronize()
        assert torch.equal(det.cpu(), ref.cpu())


def test_graph_replay_any_length_matches_eager(z):
    """The captured chain (stream-ordered workspace allocations inside the graph) replays
    to exactly the eager result."""
    from zkx_dev_b200.synth import make_cpi
    cpis = [make_cpi(100, 1000, 6, 64, seed=17 + b) for b in range(2)]
    chain = z.RangeDopplerChain(z.ChainConfig(100, 1000, 64), dev(cpis[0].replica))
    x = dev(np.stack([c.x for c in cpis]))
    ref = {k: v.clone() for k, v in chain.run_batch(x).items()}
    out = chain.allocate_outputs(batch=2)
    graph = chain.capture(x, out)
    for v in out.values():
        v.zero_()
    for _ in range(2):
        graph.launch()
    torch.cuda.synchronize()
    for key in ref:
        assert torch.equal(out[key], ref[key]), key
    graph.close()
