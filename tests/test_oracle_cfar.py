"""The banded, separable FP64 CA-CFAR used for full-plane mask checks equals the direct
FP64 ring sum (same geometry, border rule and test) and the reference's own CFAR
semantics on the cuSignal all-ones known answer."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O


@pytest.mark.parametrize("shape,guard,train,band", [((300, 400), (2, 2), (8, 8), 7),
                                                     ((61, 97), (1, 2), (3, 5), 64),
                                                     ((40, 33), (0, 0), (1, 1), 1),
                                                     ((128, 4096), (2, 2), (8, 8), 64)])
def test_banded_fp64_cfar_equals_direct(shape, guard, train, band):
    rng = np.random.default_rng(shape[0] + shape[1])
    p = rng.exponential(size=shape).astype(np.float32)
    p[rng.integers(0, shape[0], 20), rng.integers(0, shape[1], 20)] *= 80.0
    t1, m1 = O.ca_cfar_f64(p, guard, train, 1e-3)
    t2, m2 = O.ca_cfar_f64_bands(p, guard, train, 1e-3, threads=3, band_rows=band)
    np.testing.assert_array_equal(m1, m2)
    np.testing.assert_allclose(t2, t1, rtol=1e-13, atol=0)


def test_banded_fp64_cfar_all_ones():
    """cuSignal's known answer (test_radartools.py): threshold alpha inside, 0 at the
    borders; so on a constant plane only the border cells (x > 0 = T) detect."""
    x = np.ones((64, 96), dtype=np.float32)
    thr, det = O.ca_cfar_f64_bands(x, (2, 2), (8, 8), 1e-3, threads=2, band_rows=5)
    alpha = O.cfar_alpha(1e-3, O.reference_count_2d((2, 2), (8, 8)))
    assert np.allclose(thr[10:-10, 10:-10], alpha, rtol=1e-14)
    assert not thr[:10].any() and not thr[:, :10].any() and not thr[-10:].any() and not thr[:, -10:].any()
    assert not det[10:-10, 10:-10].any()
    assert det[:10].all() and det[:, :10].all() and det[-10:].all() and det[:, -10:].all()
