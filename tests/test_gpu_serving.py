"""The continuous-batching serving loop (zkx_rd_submit / zkx_rd_poll): a mixed-shape
stream of CPIs submitted while others run gives, for every CPI, exactly the result of
the same CPI processed alone; admission keeps the workspaces within the HBM budget."""
from __future__ import annotations

import random
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SHAPES = [(64, 1024), (128, 4096), (32, 2048), (64, 32768), (256, 1024), (32, 16384)]


@pytest.fixture(scope="module")
def z():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import zkx_dev_b200
    return zkx_dev_b200


def make_stream(count, seed):
    from zkx_dev_b200.synth import make_cpi
    rng = random.Random(seed)
    reqs = []
    for i in range(count):
        P, N = rng.choice(SHAPES)
        cpi = make_cpi(P, N, rng.randint(5, 20), N // 16, seed=seed * 1000 + i)
        reqs.append((P, N, cpi))
    return reqs


def alone(z, cpi, P, N, cfar_mode="accurate"):
    chain = z.RangeDopplerChain(z.ChainConfig(P, N, N // 16, cfar_mode=cfar_mode),
                                torch.as_tensor(cpi.replica).cuda())
    out = chain.run(torch.as_tensor(cpi.x).cuda())
    torch.cuda.synchronize()
    return {k: v.cpu() for k, v in out.items() if v is not None}


def submit_all(z, server, reqs, on_host=True, arrival_gaps=True):
    replicas = {}
    tickets = []
    rng = random.Random(5)
    for P, N, cpi in reqs:
        key = (P, N)
        if key not in replicas:
            replicas[key] = torch.as_tensor(cpi.replica).cuda()
        if on_host:
            x = torch.as_tensor(cpi.x).pin_memory()
            outs = {"detections": torch.empty((P, N), dtype=torch.uint8).pin_memory(),
                    "threshold": torch.empty((P, N), dtype=torch.float32).pin_memory(),
                    "power": torch.empty((P, N), dtype=torch.float32).pin_memory(),
                    "rd": torch.empty((P, N), dtype=torch.complex64).pin_memory()}
        else:
            x = torch.as_tensor(cpi.x).cuda()
            outs = {"detections": torch.empty((P, N), dtype=torch.uint8, device="cuda"),
                    "threshold": torch.empty((P, N), dtype=torch.float32, device="cuda"),
                    "power": torch.empty((P, N), dtype=torch.float32, device="cuda"),
                    "rd": None}
        # the same chirp for every CPI of a shape: one waveform id per shape
        t = server.submit(x, replicas[key], waveform_id=P * 100000 + N, **outs)
        tickets.append((t, outs))
        if arrival_gaps and rng.random() < 0.3:
            time.sleep(rng.uniform(0, 0.002))  # requests keep arriving while others run
    return tickets


def test_mixed_stream_equals_each_cpi_alone(z):
    reqs = make_stream(24, 1)
    # the synthetic model draws one chirp per (shape, length), so replicas agree per shape
    with z.RdServer(z.ServerConfig(streams=3, max_batch=4)) as server:
        tickets = submit_all(z, server, reqs)
        for t, _ in tickets:
            server.wait(t)
        st = server.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["p50_us"] <= st["p99_us"] <= st["max_us"]
    assert st["plans"] == len({(P, N) for P, N, _ in reqs})
    for (P, N, cpi), (_, outs) in zip(reqs, tickets):
        ref = alone(z, cpi, P, N)
        assert torch.equal(outs["detections"], ref["detections"]), (P, N)
        assert torch.equal(outs["threshold"], ref["threshold"]), (P, N)
        assert torch.equal(outs["power"], ref["power"]), (P, N)
        assert torch.equal(outs["rd"], ref["rd"]), (P, N)


def test_device_buffers_and_batching(z):
    reqs = make_stream(12, 2)
    with z.RdServer(z.ServerConfig(streams=2, max_batch=8)) as server:
        tickets = submit_all(z, server, reqs, on_host=False, arrival_gaps=False)
        for t, _ in tickets:
            server.wait(t)
        st = server.stats()
    assert st["completed"] == len(reqs)
    for (P, N, cpi), (_, outs) in zip(reqs, tickets):
        ref = alone(z, cpi, P, N)
        assert torch.equal(outs["detections"].cpu(), ref["detections"])
        assert torch.equal(outs["threshold"].cpu(), ref["threshold"])


def test_host_and_device_inputs_in_one_batch(z):
    """CPIs of one shape alternate between page-locked host and device memory: a batch
    stages the host ones and reads the device ones in place, with the same results."""
    from zkx_dev_b200.synth import make_cpi
    P, N = 64, 2048
    cpis = [make_cpi(P, N, 8, 128, seed=500 + i) for i in range(8)]
    rep = torch.as_tensor(cpis[0].replica).cuda()
    # every buffer exists before the first submit, so the requests arrive back to back
    # and queue behind the first batch instead of trickling in one per completion
    bufs = []
    for i, c in enumerate(cpis):
        x = torch.as_tensor(c.x).pin_memory() if i % 2 else torch.as_tensor(c.x).cuda()
        det = torch.empty((P, N), dtype=torch.uint8).pin_memory()
        thr = torch.empty((P, N), dtype=torch.float32, device="cuda")
        bufs.append((x, det, thr))
    torch.cuda.synchronize()
    with z.RdServer(z.ServerConfig(max_batch=8)) as server:
        tickets = []
        for x, det, thr in bufs:
            tickets.append((server.submit(x, rep, 3, det, threshold=thr), det, thr))
        for t, _, _ in tickets:
            server.wait(t)
        assert server.stats()["mean_batch"] > 1
    for c, (_, det, thr) in zip(cpis, tickets):
        ref = alone(z, c, P, N)
        assert torch.equal(det, ref["detections"]) and torch.equal(thr.cpu(), ref["threshold"])


def test_admission_within_budget(z):
    """A budget that holds one 128 x 4096 workspace (plus the plan) at a time: every
    request still completes, one per batch, and the peak stays within the budget."""
    from zkx_dev_b200.synth import make_cpi
    P, N = 128, 4096
    one = 2 * P * N * 8 + 2 * P * N * 4 + P * N + 8 * 256
    budget = int(1.5 * one)
    cpis = [make_cpi(P, N, 10, 256, seed=300 + i) for i in range(6)]
    reqs = [(P, N, c) for c in cpis]
    with z.RdServer(z.ServerConfig(budget_bytes=budget, max_batch=8)) as server:
        tickets = []
        rep = torch.as_tensor(cpis[0].replica).cuda()
        for _, _, c in reqs:
            det = torch.empty((P, N), dtype=torch.uint8).pin_memory()
            tickets.append((server.submit(torch.as_tensor(c.x).pin_memory(), rep, 7, det), det))
        for t, _ in tickets:
            server.wait(t)
        st = server.stats()
    assert st["completed"] == 6
    assert st["peak_bytes"] + st["plan_bytes"] <= budget
    assert st["mean_batch"] == 1.0
    for (_, _, c), (_, det) in zip(reqs, tickets):
        assert torch.equal(det, alone(z, c, P, N)["detections"])


def test_admission_tight_budget_counts_every_block(z):
    """A budget only 5 % above one 128 x 4096 workspace: the block's size class (14 MB)
    would not fit, so the server allocates the exact size; smaller CPIs of another shape
    reuse that block.  Every block the server holds plus its plans stays within the budget
    (peak_bytes counts idle blocks too), and every result equals the CPI processed alone."""
    from zkx_dev_b200.synth import make_cpi
    one = 2 * 128 * 4096 * 8 + 2 * 128 * 4096 * 4 + 128 * 4096 + 8 * 256
    budget = int(1.05 * one)
    reqs = [(128, 4096, make_cpi(128, 4096, 10, 256, seed=700 + i)) for i in range(4)]
    reqs += [(64, 4096, make_cpi(64, 4096, 6, 256, seed=710 + i)) for i in range(4)]
    with z.RdServer(z.ServerConfig(budget_bytes=budget, max_batch=8)) as server:
        tickets = []
        for P, N, c in reqs:
            rep = torch.as_tensor(c.replica).cuda()
            det = torch.empty((P, N), dtype=torch.uint8).pin_memory()
            tickets.append((server.submit(torch.as_tensor(c.x).pin_memory(), rep, 11, det), det))
        for t, _ in tickets:
            server.wait(t)
        st = server.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["peak_bytes"] + st["plan_bytes"] <= budget
    for (P, N, c), (_, det) in zip(reqs, tickets):
        assert torch.equal(det, alone(z, c, P, N)["detections"])


def test_max_pending_sheds_load(z):
    """With max_pending = 4, submits that arrive while four requests wait for admission
    are refused at once with 3002 (no ticket), counted in the statistics, and every
    accepted request still completes with the result it gets alone."""
    from zkx_dev_b200.synth import make_cpi
    P, N = 256, 8192
    cpi = make_cpi(P, N, 8, 512, seed=811)
    x = torch.as_tensor(cpi.x).cuda()
    rep = torch.as_tensor(cpi.replica).cuda()
    accepted, refused = [], 0
    with z.RdServer(z.ServerConfig(max_pending=4, max_batch=1, streams=1, max_inflight=1)) as server:
        for _ in range(64):
            det = torch.empty((P, N), dtype=torch.uint8, device="cuda")
            try:
                accepted.append((server.submit(x, rep, 5, det), det))
            except z.ZkxError as e:
                assert e.code == 3002
                refused += 1
        for t, _ in accepted:
            server.wait(t)
        st = server.stats()
    assert refused > 0 and st["refused"] == refused
    assert st["completed"] == len(accepted)
    ref = alone(z, cpi, P, N)["detections"]
    for _, det in accepted:
        assert torch.equal(det.cpu(), ref)


def test_oversized_request_is_refused(z):
    with z.RdServer(z.ServerConfig(budget_bytes=1 << 20)) as server:
        x = torch.zeros((64, 4096), dtype=torch.complex64)
        rep = torch.ones(16, dtype=torch.complex64, device="cuda")
        det = torch.empty((64, 4096), dtype=torch.uint8)
        with pytest.raises(z.ZkxError) as e:
            server.submit(x, rep, 1, det)
        assert e.value.code == 2003


def test_compat_mode_serving(z):
    reqs = [r for r in make_stream(8, 3) if r[1] <= 16384]
    with z.RdServer(z.ServerConfig(cfar_mode="compat", streams=2)) as server:
        tickets = submit_all(z, server, reqs)
        for t, _ in tickets:
            server.wait(t)
    for (P, N, cpi), (_, outs) in zip(reqs, tickets):
        ref = alone(z, cpi, P, N, cfar_mode="compat")
        assert torch.equal(outs["detections"], ref["detections"])
        assert torch.equal(outs["threshold"], ref["threshold"])


def test_invalid_request_fails_alone(z):
    """A CPI too short for the CFAR window (16 pulses < 2 * (2 + 8)) fails through its
    poll with the reference's INVALID_SHAPE code; requests around it complete."""
    from zkx_dev_b200.synth import make_cpi
    good = make_cpi(64, 1024, 5, 64, seed=11)
    bad = make_cpi(16, 1024, 5, 64, seed=12)
    with z.RdServer(z.ServerConfig()) as server:
        outs = []
        for cpi, P in ((good, 64), (bad, 16), (good, 64)):
            det = torch.empty((P, 1024), dtype=torch.uint8).pin_memory()
            rep = torch.as_tensor(cpi.replica).cuda()
            outs.append((server.submit(torch.as_tensor(cpi.x).pin_memory(), rep, P, det), det))
        server.wait(outs[0][0])
        with pytest.raises(z.ZkxValueError) as e:
            server.wait(outs[1][0])
        assert e.value.code == 1002
        server.wait(outs[2][0])
        assert server.stats()["failed"] == 1
    ref = alone(z, good, 64, 1024)["detections"]
    assert torch.equal(outs[0][1], ref) and torch.equal(outs[2][1], ref)
