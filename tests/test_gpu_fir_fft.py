"""The overlap-save FIR (two real lines per complex transform) against the FP64 oracle and
the direct-sum kernel: every block boundary, line pairing (odd line counts), filters longer
than the line, initial state, and the transform sizes for 512 / 1024 / 4096 taps.

Tolerance: relative L2 <= 1e-5 against FP64 (the FP32 path's bar)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL_L2 = 1e-5


def rel(a, b) -> float:
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def z():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zkx_dev_b200
    return zkx_dev_b200


@pytest.mark.parametrize("nb,lines,n", [(1, 2, 5000), (7, 3, 100), (64, 1, 4096), (127, 16, 20000),
                                        (127, 5, 3970), (127, 2, 3971), (128, 3, 50), (255, 4, 12345),
                                        (511, 2, 9000), (512, 2, 8000), (513, 3, 20000), (1000, 2, 30000),
                                        (1024, 1, 8193), (1025, 2, 40000), (4096, 2, 50000), (33, 1, 1)])
def test_fir_fft_matches_fp64(z, nb, lines, n):
    rng = np.random.default_rng(nb * 13 + lines * 7 + n)
    b = (rng.standard_normal(nb) / np.sqrt(nb)).astype(np.float32)
    x = rng.standard_normal((lines, n)).astype(np.float32)
    ref = O.firfilter(b, x)
    tb, tx = torch.as_tensor(b).cuda(), torch.as_tensor(x).cuda()
    got = z.firfilter(tb, tx, method="fft").cpu().numpy()
    assert rel(got, ref) <= REL_L2
    direct = z.firfilter(tb, tx, method="direct").cpu().numpy()
    assert rel(got, direct) <= REL_L2


@pytest.mark.parametrize("nb,lines,n", [(127, 3, 10000), (200, 2, 150)])
def test_fir_fft_with_initial_state(z, nb, lines, n):
    rng = np.random.default_rng(nb + n)
    b = rng.standard_normal(nb).astype(np.float32)
    x = rng.standard_normal((lines, n)).astype(np.float32)
    zi = rng.standard_normal((lines, nb - 1)).astype(np.float32)
    ref_y, ref_zf = O.firfilter(b, x, zi)
    y, zf = z.firfilter(torch.as_tensor(b).cuda(), torch.as_tensor(x).cuda(), zi=torch.as_tensor(zi).cuda(),
                        method="fft")
    assert rel(y.cpu().numpy(), ref_y) <= REL_L2
    assert rel(zf.cpu().numpy(), ref_zf) <= REL_L2


def test_fir_fft_full_size_front_end(z):
    """The bench's front end (16 x 2^20, 127-tap Kaiser lowpass): sampled lines vs FP64."""
    from zkx_dev_b200.synth import firwin_kaiser, make_front_end
    b = firwin_kaiser(127, 0.45, 8.0).astype(np.float32)
    x = make_front_end(16, 1 << 20, 5)
    got = z.firfilter(torch.as_tensor(b).cuda(), torch.as_tensor(x).cuda(), method="fft").cpu().numpy()
    for line in (0, 9, 15):
        assert rel(got[line], O.firfilter(b, x[line:line + 1])[0]) <= REL_L2


def test_fir_auto_uses_a_valid_method_and_rejects_unknown(z):
    b = torch.ones(3, device="cuda")
    x = torch.ones(1, 100, device="cuda")
    with pytest.raises(ValueError):
        z.firfilter(b, x, method="winograd")
    with pytest.raises(z.ZkxError):
        z.firfilter(torch.ones(5000, device="cuda"), torch.ones(1, 10000, device="cuda"), method="fft")
