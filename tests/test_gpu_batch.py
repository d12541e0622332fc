"""Batched chain execution and CUDA-graph replay: every CPI's result in a batch equals the
same CPI processed alone (the kernels are identical, so the outputs are bit-equal)."""
from __future__ import annotations

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


@pytest.mark.parametrize("P,N,L,nd,mode", [(64, 1024, 64, -1, "accurate"), (48, 2048, 100, 64, "accurate"),
                                           (32, 512, 32, -1, "compat")])
def test_batch_equals_single(z, P, N, L, nd, mode):
    from zkx_dev_b200.synth import make_cpi
    B = 3
    cpis = [make_cpi(P, N, 4, L, seed=100 + b) for b in range(B)]
    replica = torch.as_tensor(cpis[0].replica).cuda()
    cfg = z.ChainConfig(P, N, L, doppler_nfft=nd, cfar_mode=mode, guard_cells=(2, 2), reference_cells=(4, 4),
                        pfa=1e-4)
    chain = z.RangeDopplerChain(cfg, replica)
    x = torch.as_tensor(np.stack([c.x for c in cpis])).cuda()
    out = chain.run_batch(x)
    for b in range(B):
        one = chain.run(x[b])
        torch.cuda.synchronize()
        for key in ("compressed", "rd", "power", "threshold", "detections"):
            assert torch.equal(out[key][b], one[key]), (b, key)


def test_graph_replay_matches_eager(z):
    from zkx_dev_b200.synth import make_cpi
    cpis = [make_cpi(128, 4096, 8, 256, seed=7 + b) for b in range(2)]
    chain = z.RangeDopplerChain(z.ChainConfig(128, 4096, 256), torch.as_tensor(cpis[0].replica).cuda())
    x = torch.as_tensor(np.stack([c.x for c in cpis])).cuda()
    ref = chain.run_batch(x)
    ref = {k: v.clone() for k, v in ref.items()}
    out = chain.allocate_outputs(batch=2)
    graph = chain.capture(x, out)
    for v in out.values():
        v.zero_()
    graph.launch()
    torch.cuda.synchronize()
    for key in ref:
        assert torch.equal(out[key], ref[key]), key
    graph.close()
