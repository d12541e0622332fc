"""ambgfun on the GPU (fused per-row FFT for the 2-D cut, power-of-two correlation for the
Doppler cut) against the oracle's restatement of ambgfun_typed_cpu (pinned bit-exact to the
reference) at small sizes, and against numpy FP64 transforms at large ones.  Tolerance:
relative L2 1e-5 (the FP32 path against FP64)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL_L2 = 1e-5


def rel(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.fixture(scope="module")
def z():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zkx_dev_b200
    return zkx_dev_b200


def cplx(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("nx,ny", [(16, None), (20, 7), (5, 33), (1, None), (64, 64), (100, 37)])
@pytest.mark.parametrize("cut,cut_value", [("2d", 0.0), ("delay", 0.3), ("delay", 7.25), ("doppler", 0.3),
                                           ("doppler", -0.11)])
def test_ambgfun_matches_oracle(z, nx, ny, cut, cut_value):
    rng = np.random.default_rng(nx * 100 + (ny or 0))
    x = cplx(rng, nx)
    y = None if ny is None else cplx(rng, ny)
    ref = O.ambgfun(x, y, fs=2.0, cut=cut, cut_value=cut_value)
    got = z.ambgfun(dev(x), 2.0, 1.0, y=None if y is None else dev(y), cut=cut, cutValue=cut_value)
    assert tuple(got.shape) == ref.shape
    assert rel(got.cpu().numpy(), ref) <= REL_L2


def test_ambgfun_high_rank_prefix(z):
    """A [8, 3] input: only its first extent (8 samples) enters the sums, the norm runs over
    all 24 values (the reference's 2-D rule)."""
    x = cplx(np.random.default_rng(2), 8, 3)
    ref = O.ambgfun(x.ravel(), nx=8)
    got = z.ambgfun(dev(x), 1.0, 1.0).cpu().numpy()
    assert rel(got, ref) <= REL_L2


def test_ambgfun_zero_norm_is_nan(z):
    got = z.ambgfun(torch.zeros(12, dtype=torch.complex64, device="cuda"), 1.0, 1.0).cpu().numpy()
    assert np.all(np.isnan(got))


def numpy_2d_rows(x, y, rows_wanted):
    x = x.astype(np.complex128); y = y.astype(np.complex128)
    xn, yn = x / np.linalg.norm(x), y / np.linalg.norm(y)
    nx, ny = x.size, y.size
    rows = nx + ny - 1
    nf = 1 << int(np.ceil(np.log2(rows)))
    out = []
    c = np.arange(ny)
    for r in rows_wanted:
        xc = c - (nx - 1) + r
        ok = (xc >= 0) & (xc < nx)
        p = np.zeros(nf, complex)
        p[c[ok]] = yn[c[ok]] * np.conj(xn[xc[ok]])
        out.append(np.roll(np.abs(nf * np.fft.ifft(p)), nf // 2))
    return np.array(out)


@pytest.mark.parametrize("nx,ny", [(2048, 2048), (3000, 1000), (12000, 5000)])
def test_ambgfun_2d_large_sampled_rows(z, nx, ny):
    """Fused per-row path (nfreq 4096) and the general path through the clustered
    transforms (nfreq 32768): sampled delay rows against numpy FP64."""
    rng = np.random.default_rng(nx + ny)
    x, y = cplx(rng, nx), cplx(rng, ny)
    got = z.ambgfun(dev(x), 1.0, 1.0, y=dev(y))
    rows = nx + ny - 1
    pick = sorted({0, 1, rows // 3, rows // 2, rows - 2, rows - 1, nx - 1})
    g = got[torch.as_tensor(pick, device="cuda")].cpu().numpy()
    assert rel(g, numpy_2d_rows(x, y, pick)) <= REL_L2


def test_ambgfun_cuts_large(z):
    rng = np.random.default_rng(4)
    nx, ny, fs = 5000, 3000, 4.0
    x, y = cplx(rng, nx), cplx(rng, ny)
    xn = x.astype(np.complex128) / np.linalg.norm(x.astype(np.complex128))
    yn = y.astype(np.complex128) / np.linalg.norm(y.astype(np.complex128))
    rows = nx + ny - 1
    nf = 1 << int(np.ceil(np.log2(rows)))
    # delay cut
    tau = 13.5
    X = np.fft.fft(xn, nf) * np.exp(2j * np.pi * (-fs / 2 + fs * np.arange(nf) / nf) * tau)
    xs = np.fft.ifft(X)
    prod = np.zeros(nf, complex)
    prod[:ny] = yn * np.conj(xs[:ny])
    tr = np.fft.ifft(prod)
    ref = nf * np.abs(tr[(np.arange(nf) + nf // 2) % nf])
    got = z.ambgfun(dev(x), fs, 1.0, y=dev(y), cut="delay", cutValue=tau).cpu().numpy()
    assert rel(got, ref) <= REL_L2
    # Doppler cut
    fd = 0.37
    xm = xn * np.exp(2j * np.pi * fd * np.arange(nx) / fs)
    c = np.fft.ifft(np.fft.fft(yn, rows) * np.conj(np.fft.fft(xm, rows)))
    ref = np.abs(c[(np.arange(rows) - rows // 2 + rows) % rows])
    got = z.ambgfun(dev(x), fs, 1.0, y=dev(y), cut="doppler", cutValue=fd).cpu().numpy()
    assert rel(got, ref) <= REL_L2
