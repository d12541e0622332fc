"""The autotuner (zkx_rd_plan_autotune): every kernel choice it can make gives the same
chain results bit for bit, the chosen values are valid, and later plans of the same shape
start from them."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def z():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zkx_dev_b200
    return zkx_dev_b200


def set_tuning(chain, variant, columns):
    from zkx_dev_b200 import _lib as L
    t = L.RdTuning(variant, columns)
    L.check(L.lib().zkx_rd_plan_set_tuning(chain._plan, ctypes.byref(t)))


@pytest.mark.parametrize("P,N,L", [(512, 8192, 512), (1024, 4096, 256), (128, 16384, 1024)])
def test_every_choice_gives_identical_results(z, P, N, L):
    from zkx_dev_b200.synth import draw_targets, device_cpi, lfm_chirp
    x = device_cpi(P, N, draw_targets(P, N, 10, L, seed=1), L, seed=2)
    chain = z.RangeDopplerChain(z.ChainConfig(P, N, L), torch.as_tensor(lfm_chirp(L).astype(np.complex64)).cuda())
    outs = []
    for variant in (1, 2):
        for columns in (8, 16):
            set_tuning(chain, variant, columns)
            o = chain(x)
            torch.cuda.synchronize()
            outs.append({k: v.clone() for k, v in o.items()})
    for o in outs[1:]:
        for key in outs[0]:
            assert torch.equal(o[key], outs[0][key]), key


def test_autotune_choice_is_valid_and_shared(z):
    from zkx_dev_b200.synth import draw_targets, device_cpi, lfm_chirp
    P, N, L = 256, 8192, 512
    x = device_cpi(P, N, draw_targets(P, N, 5, L, seed=3), L, seed=4)
    rep = torch.as_tensor(lfm_chirp(L).astype(np.complex64)).cuda()
    chain = z.RangeDopplerChain(z.ChainConfig(P, N, L), rep)
    chosen = chain.autotune(x)
    assert chosen["compression_variant"] in (1, 2) and chosen["doppler_columns"] in (8, 16)
    assert chain.tuning == chosen
    again = z.RangeDopplerChain(z.ChainConfig(P, N, L), rep)
    assert again.tuning == chosen
    out = again(x)
    torch.cuda.synchronize()
    assert out["detections"].sum().item() > 0
