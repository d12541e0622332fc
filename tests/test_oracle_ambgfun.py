"""The ambgfun restatement in oracle/ (rt.cpp:330-463) against the reference's own
ambgfun_typed_cpu<float> compiled from its sources: bit-identical on every cut, on unequal
lengths, on a high-rank prefix and on a zero-norm input (NaN)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O


def cplx(rng, n):
    return (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)


CASES = [
    ("x only", lambda r: dict(x=cplx(r, 16))),
    ("y shorter", lambda r: dict(x=cplx(r, 20), y=cplx(r, 7))),
    ("y longer", lambda r: dict(x=cplx(r, 5), y=cplx(r, 33))),
    ("zero norm", lambda r: dict(x=np.zeros(9, np.complex64))),
]


@pytest.mark.parametrize("name,make", CASES)
@pytest.mark.parametrize("cut,cut_value", [("2d", 0.0), ("delay", 0.3), ("delay", 2.5), ("doppler", 0.3),
                                           ("doppler", -0.05)])
def test_restatement_matches_reference(reference_lib, name, make, cut, cut_value):
    kw = make(np.random.default_rng(len(name)))
    ours = O.ambgfun(cut=cut, fs=2.0, cut_value=cut_value, **kw)
    ref, is64 = O.ref_ambgfun(cut=cut, fs=2.0, cut_value=cut_value, **kw)
    assert is64 == (cut != "2d")
    if not is64:
        ours = ours.astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(ours, ref)


def test_high_rank_prefix_matches_reference(reference_lib):
    x = cplx(np.random.default_rng(5), 24)
    ours = O.ambgfun(x, nx=8).astype(np.float32)
    ref, _ = O.ref_ambgfun(x, nx=8)
    np.testing.assert_array_equal(ours, ref)


def test_restatement_against_fft_definition():
    """The 2-D cut equals the magnitude of the shifted inverse DFT of each delayed product
    (numpy FP64), the reference's device formulation (radartools_typed.cu:63-75)."""
    rng = np.random.default_rng(9)
    x, y = cplx(rng, 12), cplx(rng, 9)
    got = O.ambgfun(x, y, cut="2d")
    xn = x.astype(np.complex128) / np.linalg.norm(x.astype(np.complex128))
    yn = y.astype(np.complex128) / np.linalg.norm(y.astype(np.complex128))
    rows, nf = got.shape
    for r in range(rows):
        p = np.zeros(nf, complex)
        for c in range(9):
            xc = c - 11 + r
            if 0 <= xc < 12:
                p[c] = yn[c] * np.conj(xn[xc])
        np.testing.assert_allclose(got[r], np.roll(np.abs(nf * np.fft.ifft(p)), nf // 2), rtol=1e-12, atol=1e-13)
