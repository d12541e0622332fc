"""The work list (zkx_rd_worklist_*): CPIs of mixed shapes run with one launch per stage,
and every CPI's power, threshold and detections equal the same CPI executed alone with
its plan, bit for bit -- on the work-list kernels and on the plans' own kernels that take
the stages the work-list kernels do not cover (long and non-power-of-two transforms,
four-step compression, compat-mode and half-tile CFAR)."""
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


def set_tuning(chain, variant, columns, cfar_tile=0):
    from zkx_dev_b200 import _lib as L
    t = L.RdTuning(variant, columns, cfar_tile)
    L.check(L.lib().zkx_rd_plan_set_tuning(chain._plan, ctypes.byref(t)))


def make_items(z, specs, seed):
    """specs: (P, N, copies, options) -> [(chain, x, outputs)] plus the plans."""
    from zkx_dev_b200.synth import make_cpi
    items, chains = [], []
    for k, (P, N, copies, opts) in enumerate(specs):
        L = max(16, N // 16)
        cpis = [make_cpi(P, N, 6, L, seed=seed * 1000 + 10 * k + c) for c in range(copies)]
        cfg = z.ChainConfig(P, N, L, cfar_mode=opts.get("cfar_mode", "accurate"),
                            doppler_nfft=opts.get("doppler_nfft", -1),
                            guard_cells=opts.get("guard", (2, 2)), reference_cells=opts.get("train", (8, 8)))
        chain = z.RangeDopplerChain(cfg, torch.as_tensor(cpis[0].replica).cuda())
        if "tuning" in opts:
            set_tuning(chain, *opts["tuning"])
        chains.append(chain)
        shape = (chain.doppler_bins, chain.range_bins)
        for c, cpi in enumerate(cpis):
            out = {"threshold": torch.full(shape, -1.0, device="cuda"),
                   "detections": torch.full(shape, 7, dtype=torch.uint8, device="cuda")}
            if c % 2 == 0:
                out["power"] = torch.full(shape, -1.0, device="cuda")
            items.append((chain, torch.as_tensor(cpi.x).cuda(), out))
    return items, chains


def check_alone(items):
    for i, (chain, x, out) in enumerate(items):
        ref = chain.run(x)
        torch.cuda.synchronize()
        assert torch.equal(out["threshold"], ref["threshold"]), i
        assert torch.equal(out["detections"], ref["detections"]), i
        if "power" in out:
            assert torch.equal(out["power"], ref["power"]), i


COVERED = [(64, 1024, 3, {}), (128, 4096, 2, {}), (256, 2048, 2, {}), (64, 4096, 2, {}),
           (64, 8192, 1, {}), (512, 512, 1, {}), (128, 256, 2, {}), (1024, 1024, 1, {}),
           (100, 2048, 3, {"doppler_nfft": 128})]   # Doppler zero padding: 100 pulses -> 128 bins


def test_worklist_equals_each_cpi_alone(z):
    items, _ = make_items(z, COVERED, 1)
    wl = z.WorkList(items)
    info = wl.info()
    # every stage of every plan on the work-list kernels: compression and Doppler one
    # launch per resource class (up to 16 and 32 values per thread), CFAR one launch, plus
    # the copies of the power planes asked for
    powers = sum("power" in o for _, _, o in items)
    assert info["groups"] == len(COVERED)
    assert info["launches"] == 5 + powers
    wl.launch()
    torch.cuda.synchronize()
    check_alone(items)
    from zkx_dev_b200 import _lib
    assert _lib.kernel_status(clear=True) == 0


def test_worklist_stages_on_the_plans_own_kernels(z):
    """Plans whose stages the work-list kernels do not take, mixed with ones they do."""
    specs = [
        (64, 1024, 2, {}),
        (1024, 16384, 1, {}),                       # four-step compression by default
        (64, 16384, 2, {}),                         # 16384 points: the plan's own compression
        (64, 32768, 2, {}),                         # cluster compression
        (100, 1000, 2, {}),                         # chirp-z range and Doppler lengths
        (2048, 1024, 1, {}),                        # Doppler length 2048
        (128, 4096, 2, {"cfar_mode": "compat"}),
        (128, 4096, 2, {"tuning": (3, 0, 2)}),      # four-step compression, half-tile CFAR
        (256, 2048, 2, {"guard": (1, 1), "train": (4, 4)}),   # another window geometry
        (96, 2048, 1, {}),                          # Doppler length 96: chirp-z
    ]
    items, _ = make_items(z, specs, 2)
    wl = z.WorkList(items)
    assert wl.info()["groups"] == len(specs)
    wl.launch()
    torch.cuda.synchronize()
    check_alone(items)
    from zkx_dev_b200 import _lib
    assert _lib.kernel_status(clear=True) == 0


def test_worklist_graph_replay_and_many_groups(z):
    """More plans than one launch's 24 groups (several launches per stage), captured in a
    CUDA graph and replayed on new inputs copied into the same buffers."""
    from zkx_dev_b200.synth import make_cpi
    specs = [(64, 1024, 1, {}) for _ in range(20)] + [(64, 2048, 1, {}) for _ in range(10)]
    items, _ = make_items(z, specs, 3)
    wl = z.WorkList(items)
    info = wl.info()
    assert info["groups"] == 30 and info["launches"] == 6 + sum("power" in o for _, _, o in items)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        wl.launch()
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        wl.launch()
    for i, (chain, x, _) in enumerate(items):
        P, N = x.shape
        x.copy_(torch.as_tensor(make_cpi(P, N, 9, max(16, N // 16), seed=7000 + i).x).cuda())
    graph.replay()
    torch.cuda.synchronize()
    check_alone(items)
    del graph


def test_worklist_rejects_bad_items(z):
    from zkx_dev_b200.synth import make_cpi
    cpi = make_cpi(64, 4096, 5, 256, seed=5)
    tc = z.RangeDopplerChain(z.ChainConfig(64, 4096, 256, precision="tc_f16"), torch.as_tensor(cpi.replica).cuda())
    out = {"threshold": torch.empty((64, 4096), device="cuda"),
           "detections": torch.empty((64, 4096), dtype=torch.uint8, device="cuda")}
    with pytest.raises(z.ZkxError) as e:
        z.WorkList([(tc, torch.as_tensor(cpi.x).cuda(), out)])
    assert e.value.code == 1004
    fp = z.RangeDopplerChain(z.ChainConfig(64, 4096, 256), torch.as_tensor(cpi.replica).cuda())
    with pytest.raises(ValueError):
        z.WorkList([(fp, torch.as_tensor(cpi.x).cuda(), {"threshold": out["threshold"]})])
    with pytest.raises(ValueError):
        z.WorkList([(fp, torch.as_tensor(cpi.x[:32]).cuda(), out)])
