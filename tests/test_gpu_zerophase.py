"""firfilter2 (zero-phase FIR) and hilbert (analytic signal) on the GPU against the oracle
restatements (pinned bit-exact to the reference's published digests) and FP64 transforms.

Tolerance: relative L2 <= 1e-5 (the FP32 path's bar); the odd-pad rounding of half and
integer element types is checked where it changes the padded values."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL_L2 = 1e-5


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
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


def hilbert64(x, nfft):
    X = np.fft.fft(np.asarray(x, dtype=np.float64), n=nfft, axis=-1)
    w = np.zeros(nfft)
    w[0] = 1.0
    w[1:(nfft + 1) // 2] = 2.0
    if nfft % 2 == 0:
        w[nfft // 2] = 1.0
    return np.fft.ifft(X * w, axis=-1)


# ------------------------------------------------------------------ firfilter2

@pytest.mark.parametrize("nb,lines,n", [(3, 2, 100), (127, 4, 20000), (1, 3, 50), (16, 1, 4096),
                                        (17, 2, 4097), (64, 5, 12345), (255, 1, 9000), (33, 300, 257),
                                        (1000, 2, 10000), (4096, 1, 20000)])
@pytest.mark.parametrize("padtype", ["odd", "even", "constant", "none"])
def test_firfilter2_matches_restatement(z, nb, lines, n, padtype):
    rng = np.random.default_rng(nb * 31 + n)
    b = (rng.standard_normal(nb) / np.sqrt(nb)).astype(np.float32)
    x = rng.standard_normal((lines, n)).astype(np.float32)
    ref = O.firfilter2(b, x, padtype)
    got = z.firfilter2(dev(b), dev(x), padtype=padtype).cpu().numpy()
    assert rel_l2(got, ref) <= REL_L2


@pytest.mark.parametrize("nb,n,padlen", [(7, 8, 7), (5, 100, 0), (9, 50, 49), (3, 5, 1), (31, 100, -4)])
def test_firfilter2_padlen_edges(z, nb, n, padlen):
    """Explicit padlen down to the limit n - 1, zero and negative (no padding)."""
    rng = np.random.default_rng(n + padlen)
    b = rng.standard_normal(nb).astype(np.float32)
    x = rng.standard_normal((3, n)).astype(np.float32)
    for padtype in ("odd", "even", "constant"):
        ref = O.firfilter2(b, x, padtype, padlen)
        got = z.firfilter2(dev(b), dev(x), padtype=padtype, padlen=padlen).cpu().numpy()
        assert rel_l2(got, ref) <= REL_L2, padtype


def test_firfilter2_taps_longer_than_line(z):
    """No padding and more taps than samples: both initial conditions cover whole lines."""
    rng = np.random.default_rng(4)
    b = rng.standard_normal(40).astype(np.float32)
    x = rng.standard_normal((2, 9)).astype(np.float32)
    got = z.firfilter2(dev(b), dev(x), padtype=None).cpu().numpy()
    assert rel_l2(got, O.firfilter2(b, x, "none")) <= REL_L2


def test_firfilter2_axis0_and_rank3(z):
    rng = np.random.default_rng(5)
    b = rng.standard_normal(9).astype(np.float32)
    x = rng.standard_normal((300, 7)).astype(np.float32)
    got = z.firfilter2(dev(b), dev(x), axis=0).cpu().numpy()
    assert rel_l2(got, O.firfilter2(b, x.T.copy()).T) <= REL_L2
    x3 = rng.standard_normal((2, 3, 500)).astype(np.float32)
    got3 = z.firfilter2(dev(b), dev(x3)).cpu().numpy()
    assert rel_l2(got3, O.firfilter2(b, x3.reshape(6, 500)).reshape(2, 3, 500)) <= REL_L2


@pytest.mark.parametrize("dtype,rounding", [(np.int8, 2), (np.int16, 3), (np.float16, 1)])
def test_firfilter2_odd_pad_rounding_of_element_types(z, dtype, rounding):
    """Odd reflection of values near the type's range wraps (integers) or rounds (half) as
    the reference's element type does; the GPU follows with the same rounding code and
    matches the reference's own CPU function where it is built."""
    rng = np.random.default_rng(6)
    if dtype == np.float16:
        x = (rng.standard_normal((2, 64)) * 4e3).astype(np.float16)  # 2 x0 - r stays finite
    else:
        info = np.iinfo(dtype)
        x = rng.integers(info.min, info.max, (2, 64), endpoint=True).astype(dtype)
    b = np.array([1, 2, 3, 2, 1], dtype=dtype)
    xf, bf = x.astype(np.float32), b.astype(np.float32)
    ref = O.firfilter2(bf, xf, "odd", 10, rounding)
    plain = O.firfilter2(bf, xf, "odd", 10, 0)
    got = z.firfilter2(dev(bf), dev(xf), padlen=10, pad_rounding=rounding).cpu().numpy()
    assert rel_l2(got, ref) <= REL_L2
    if dtype != np.float16:
        assert rel_l2(plain, ref) > 1e-3  # the wrap changes the result: the case is meaningful
    if O.reference() is not None:
        r, _ = O.ref_firfilter2(b, x, -1, "odd", 10)
        assert rel_l2(got, r) <= REL_L2


def test_firfilter2_full_size_sampled_lines(z):
    """16 x 2^20 with 127 taps: sampled lines against the restatement."""
    rng = np.random.default_rng(7)
    b = (rng.standard_normal(127) / 11).astype(np.float32)
    x = rng.standard_normal((16, 1 << 20)).astype(np.float32)
    got = z.firfilter2(dev(b), dev(x)).cpu().numpy()
    for line in (0, 7, 15):
        assert rel_l2(got[line], O.firfilter2(b, x[line:line + 1])[0]) <= REL_L2


def test_firfilter2_errors(z):
    b = dev(np.ones(3, np.float32))
    with pytest.raises(z.ZkxValueError):
        z.firfilter2(b, dev(np.ones((2, 9), np.float32)))          # n <= 3 * nb
    with pytest.raises(ValueError):
        z.firfilter2(b, dev(np.ones((2, 100), np.float32)), method="gust")
    with pytest.raises(z.ZkxError):
        z.firfilter2(dev(np.ones(5000, np.float32)), dev(np.ones((1, 20000), np.float32)), padtype=None)


# ------------------------------------------------------------------ hilbert

@pytest.mark.parametrize("lines,n,N", [(3, 16, None), (2, 1000, 1024), (5, 4096, None), (1, 16384, None),
                                       (4, 100, 64), (2, 5000, None), (3, 777, 1000), (1, 32768, None),
                                       (1, 65536, None), (64, 1, None), (2, 1, 8), (7, 3, None),
                                       (2, 20000, 30000)])
def test_hilbert_matches_fp64(z, lines, n, N):
    rng = np.random.default_rng(lines * 7 + n)
    x = rng.standard_normal((lines, n)).astype(np.float32)
    nf = n if N is None else N
    got = z.hilbert(dev(x), N=N).cpu().numpy()
    assert got.shape == (lines, nf)
    assert rel_l2(got, hilbert64(x, nf)) <= REL_L2
    if nf <= 64:
        assert rel_l2(got, O.hilbert(x, nf)) <= REL_L2


def test_hilbert_real_part_is_the_input(z):
    """For N = n the real part of the analytic signal is x itself."""
    rng = np.random.default_rng(8)
    x = rng.standard_normal((8, 4096)).astype(np.float32)
    got = z.hilbert(dev(x)).cpu().numpy()
    assert np.max(np.abs(got.real - x)) <= 1e-5 * np.max(np.abs(x)) * 10


def test_hilbert_axis0_and_empty(z):
    rng = np.random.default_rng(9)
    x = rng.standard_normal((512, 6)).astype(np.float32)
    got = z.hilbert(dev(x), axis=0).cpu().numpy()
    assert rel_l2(got, hilbert64(x.T, 512).T) <= REL_L2
    empty = z.hilbert(dev(np.zeros((3, 0), np.float32)), N=8).cpu().numpy()
    assert empty.shape == (3, 8) and not np.any(empty)
    with pytest.raises(ValueError):
        z.hilbert(dev(np.zeros((3, 0), np.float32)))


@pytest.mark.parametrize("nb,lines,n,padtype,padlen", [(127, 4, 20000, "odd", None), (16, 3, 5000, "even", None),
                                                       (255, 1, 9000, "constant", 300), (64, 5, 4000, "odd", 64),
                                                       (1000, 2, 10000, "odd", None), (2000, 1, 30000, "even", None),
                                                       (4096, 1, 20000, "odd", 5000), (33, 300, 257, "odd", None),
                                                       (127, 3, 382, "odd", None)])
def test_firfilter2_fft_evaluation(z, nb, lines, n, padtype, padlen):
    """One overlap-save convolution with the taps' autocorrelation (padding >= taps) equals the
    two-pass definition: against the restatement and the direct kernel."""
    rng = np.random.default_rng(nb * 3 + n)
    b = (rng.standard_normal(nb) / np.sqrt(nb)).astype(np.float32)
    x = rng.standard_normal((lines, n)).astype(np.float32)
    ref = O.firfilter2(b, x, padtype, padlen)
    got = z.firfilter2(dev(b), dev(x), padtype=padtype, padlen=padlen, evaluation="fft").cpu().numpy()
    direct = z.firfilter2(dev(b), dev(x), padtype=padtype, padlen=padlen, evaluation="direct").cpu().numpy()
    assert rel_l2(got, ref) <= REL_L2
    assert rel_l2(direct, ref) <= REL_L2


def test_firfilter2_fft_needs_padding_as_long_as_the_filter(z):
    b = dev(np.ones(9, np.float32))
    x = dev(np.ones((1, 100), np.float32))
    with pytest.raises(z.ZkxError):
        z.firfilter2(b, x, padlen=4, evaluation="fft")
    # the automatic choice falls back to the direct passes
    got = z.firfilter2(b, x, padlen=4).cpu().numpy()
    assert rel_l2(got, O.firfilter2(np.ones(9, np.float32), np.ones((1, 100), np.float32), "odd", 4)) <= REL_L2


def test_hilbert_of_a_cosine_is_the_complex_exponential(z):
    """For a cosine on an exact bin, the analytic signal is exp(i w n): real part the cosine,
    imaginary part the sine (cuSignal's hilbert contract)."""
    n = np.arange(4096)
    for k in (1, 17, 1000, 2047):
        x = np.cos(2 * np.pi * k * n / 4096).astype(np.float32)
        got = z.hilbert(dev(x[None, :])).cpu().numpy()[0]
        ref = np.exp(1j * 2 * np.pi * k * n / 4096)
        assert rel_l2(got, ref) <= REL_L2, k


def test_firfilter2_has_zero_phase(z):
    """A passband sinusoid comes out of the zero-phase filter with no delay: the output equals
    the input times |H(w)|^2 away from the line ends."""
    from zkx_dev_b200.synth import firwin_kaiser
    b = firwin_kaiser(63, 0.3, 8.0).astype(np.float32)
    n = np.arange(20000)
    w = 2 * np.pi * 0.05
    x = np.cos(w * n + 0.3).astype(np.float32)
    got = z.firfilter2(dev(b), dev(x[None, :])).cpu().numpy()[0]
    gain = np.abs(np.sum(b.astype(np.float64) * np.exp(-1j * w * np.arange(63)))) ** 2
    mid = slice(2000, 18000)
    assert rel_l2(got[mid], gain * x[mid].astype(np.float64)) <= 1e-4
