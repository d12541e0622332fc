"""The autotuner (zkx_rd_plan_autotune): the kernel choices that share one transform
(compression variants 1 and 2, both Doppler tile widths) give the same chain results bit
for bit, variant 3 (its own four-step transform) agrees with the FP64 oracle and with them
to FP32 rounding, the chosen values are valid, and later plans of the same shape start
from them."""
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
    assert chosen["compression_variant"] in (1, 2, 3) and chosen["doppler_columns"] in (8, 16)
    assert chosen["cfar_tile"] in (1, 2, 3)
    assert chosen["compression_radix"] in (0, 16, 32) and chosen["compression_ctas_per_sm"] in (0, 1, 2)
    assert chosen["cfar_ctas_per_sm"] in (0, 1)
    assert chain.tuning == chosen
    again = z.RangeDopplerChain(z.ChainConfig(P, N, L), rep)
    assert again.tuning == chosen
    out = again(x)
    torch.cuda.synchronize()
    assert out["detections"].sum().item() > 0


@pytest.mark.parametrize("P,N,L,nfft", [(512, 8192, 512, -1), (1024, 4096, 256, -1), (128, 16384, 1024, -1),
                                        (96, 3000, 200, 4096), (40, 20000, 1024, 16384)])
def test_local_variant_matches_fp64(z, P, N, L, nfft):
    """Variant 3 (the persistent kernel with the four-step transform and the spectrum held
    in tensor memory) rounds differently from variants 1 and 2, so it is checked on its own:
    compressed pulses against the FP64 oracle (zero padding and truncation included), within
    FP32 rounding of variant 2, and a detection mask equal to the FP64 CFAR of its power."""
    import oracle as O
    from zkx_dev_b200.synth import make_cpi
    cpi = make_cpi(P, N, 8, L, seed=P + N)
    chain = z.RangeDopplerChain(z.ChainConfig(P, N, L, range_nfft=nfft), torch.as_tensor(cpi.replica).cuda())
    x = torch.as_tensor(cpi.x).cuda()
    set_tuning(chain, 2, 8)
    ref = {k: v.clone() for k, v in chain(x).items()}
    set_tuning(chain, 3, 8)
    got = chain(x)
    torch.cuda.synchronize()
    comp = got["compressed"].cpu().numpy().astype(np.complex128)
    comp2 = ref["compressed"].cpu().numpy().astype(np.complex128)
    assert np.linalg.norm(comp - comp2) / np.linalg.norm(comp2) <= 1e-6
    rows = [0, 1, P // 2, P - 1]
    c64 = O.pulse_compression_fft64(cpi.x[rows], cpi.replica, nfft, True, O.radar_window_f32("hamming", L))
    assert np.linalg.norm(comp[rows] - c64) / np.linalg.norm(c64) <= 1e-5
    _, m64 = O.ca_cfar_f64(got["power"].cpu().numpy(), (2, 2), (8, 8), 1e-6)
    np.testing.assert_array_equal(got["detections"].cpu().numpy(), m64)
    from zkx_dev_b200 import _lib
    assert _lib.kernel_status(clear=True) == 0


def test_local_variant_stacked_batch(z):
    """Variant 3 over a stack of CPIs (run_batch: one launch over all their pulses) gives
    every CPI the result it gets alone."""
    from zkx_dev_b200.synth import make_cpi
    cpis = [make_cpi(64, 8192, 6, 512, seed=90 + b) for b in range(3)]
    chain = z.RangeDopplerChain(z.ChainConfig(64, 8192, 512), torch.as_tensor(cpis[0].replica).cuda())
    set_tuning(chain, 3, 8)
    batch = chain.run_batch(torch.as_tensor(np.stack([c.x for c in cpis])).cuda())
    torch.cuda.synchronize()
    for b, c in enumerate(cpis):
        alone = chain(torch.as_tensor(c.x).cuda())
        torch.cuda.synchronize()
        assert torch.equal(batch["compressed"][b], alone["compressed"])
        assert torch.equal(batch["detections"][b], alone["detections"])


@pytest.mark.parametrize("P,N,batch", [(1024, 16384, 1), (100, 4000, 2), (256, 2048, 3), (64, 1024, 40)])
def test_cfar_tiles_give_the_fp64_mask(z, P, N, batch):
    """The tiled CA-CFAR kernels (row-sum planes of the whole tile, built in two 32-row
    halves, or whole-tile planes in persistent CTAs that walk the tiles of every map) give
    the FP64 CFAR's mask of the same power, on full and partial tiles and on stacked
    batches; their thresholds agree to FP32 rounding, and the persistent kernel's equal the
    whole-tile kernel's bit for bit."""
    import oracle as O
    from zkx_dev_b200.synth import make_cpi
    cpis = [make_cpi(P, N, 10, 64, seed=N + b) for b in range(batch)]
    chain = z.RangeDopplerChain(z.ChainConfig(P, N, 64), torch.as_tensor(cpis[0].replica).cuda())
    x = torch.as_tensor(np.stack([c.x for c in cpis])).cuda()
    outs = {}
    for tile in (1, 2, 3):
        set_tuning(chain, 0, 0, tile)
        o = chain.run_batch(x)
        torch.cuda.synchronize()
        outs[tile] = {k: v.cpu().numpy().copy() for k, v in o.items() if v is not None}
    for b in range(batch):
        _, m64 = O.ca_cfar_f64_bands(outs[2]["power"][b], (2, 2), (8, 8), 1e-6)
        np.testing.assert_array_equal(outs[2]["detections"][b], m64)
        np.testing.assert_array_equal(outs[1]["detections"][b], m64)
        np.testing.assert_array_equal(outs[3]["detections"][b], m64)
        np.testing.assert_array_equal(outs[3]["threshold"][b], outs[1]["threshold"][b])
        t1 = outs[1]["threshold"][b].astype(np.float64)
        t2 = outs[2]["threshold"][b].astype(np.float64)
        inside = t1 > 0
        assert np.array_equal(inside, t2 > 0)
        assert np.max(np.abs(t2[inside] - t1[inside]) / t1[inside]) <= 2e-6
    from zkx_dev_b200 import _lib
    assert _lib.kernel_status(clear=True) == 0


@pytest.mark.parametrize("P,N", [(600, 16384), (2400, 4096)])
def test_local_variant_output_alignment(z, P, N):
    """The four-step kernel stores pairs of outputs with 128-bit stores when the output is
    16-byte aligned and single values otherwise; both give the same bits (the C ABI with an
    output pointer 8 bytes past a 16-byte boundary)."""
    from zkx_dev_b200 import _lib as L
    from zkx_dev_b200.synth import draw_targets, device_cpi, lfm_chirp
    lib, sh = L.lib(), L.stream_handle()
    x = device_cpi(P, N, draw_targets(P, N, 8, 256, seed=3), 256, seed=4)
    rep = torch.as_tensor(lfm_chirp(256).astype(np.complex64)).cuda()
    spec = torch.empty(N, dtype=torch.complex64, device="cuda")
    L.check(lib.zkx_replica_spectrum_c64(rep.data_ptr(), 256, N, 1, L.WINDOW_HAMMING, None, spec.data_ptr(), sh))
    aligned = torch.empty((P, N), dtype=torch.complex64, device="cuda")
    buf = torch.empty(P * N + 1, dtype=torch.complex64, device="cuda")
    shifted = buf[1:].view(P, N)
    assert aligned.data_ptr() % 16 == 0 and shifted.data_ptr() % 16 == 8
    for y in (aligned, shifted):
        L.check(lib.zkx_pulse_compression_spectrum_c64(x.data_ptr(), P, N, N, spec.data_ptr(), y.data_ptr(), sh))
    torch.cuda.synchronize()
    assert torch.equal(aligned, shifted)
    assert L.kernel_status(clear=True) == 0


def set_full_tuning(chain, **kw):
    from zkx_dev_b200 import _lib as L
    t = L.RdTuning(**kw)
    L.check(L.lib().zkx_rd_plan_set_tuning(chain._plan, ctypes.byref(t)))


@pytest.mark.parametrize("P,N,L", [(256, 1024, 64), (128, 2048, 128), (96, 4096, 256), (64, 8192, 512)])
def test_radix_plan_matches_fp64(z, P, N, L):
    """The other radix plan of the Stockham compression kernels (16 <-> 32 values per
    thread) rounds differently: compressed pulses against the FP64 oracle and within FP32
    rounding of the table's plan, a mask equal to the FP64 CFAR of its power, and each CPI
    of a stacked batch equal to the CPI alone."""
    import oracle as O
    from zkx_dev_b200.synth import make_cpi
    cpis = [make_cpi(P, N, 8, L, seed=P * 7 + N + b) for b in range(2)]
    chain = z.RangeDopplerChain(z.ChainConfig(P, N, L), torch.as_tensor(cpis[0].replica).cuda())
    x = torch.as_tensor(cpis[0].x).cuda()
    for variant in (1, 2):
        set_full_tuning(chain, compression_variant=variant)
        ref = {k: v.clone() for k, v in chain(x).items()}
        alt = 16 if N in (1024, 8192) else 32
        set_full_tuning(chain, compression_variant=variant, compression_radix=alt)
        got = {k: v.clone() for k, v in chain(x).items()}
        torch.cuda.synchronize()
        comp = got["compressed"].cpu().numpy().astype(np.complex128)
        comp2 = ref["compressed"].cpu().numpy().astype(np.complex128)
        assert np.linalg.norm(comp - comp2) / np.linalg.norm(comp2) <= 1e-6
        rows = [0, P // 2, P - 1]
        c64 = O.pulse_compression_fft64(cpis[0].x[rows], cpis[0].replica, -1, True, O.radar_window_f32("hamming", L))
        assert np.linalg.norm(comp[rows] - c64) / np.linalg.norm(c64) <= 1e-5
        _, m64 = O.ca_cfar_f64(got["power"].cpu().numpy(), (2, 2), (8, 8), 1e-6)
        np.testing.assert_array_equal(got["detections"].cpu().numpy(), m64)
        batch = chain.run_batch(torch.as_tensor(np.stack([c.x for c in cpis])).cuda())
        torch.cuda.synchronize()
        assert torch.equal(batch["compressed"][0], got["compressed"])
        assert torch.equal(batch["detections"][0], got["detections"])
    from zkx_dev_b200 import _lib
    assert _lib.kernel_status(clear=True) == 0


@pytest.mark.parametrize("P,N,L,variant", [(512, 8192, 512, 2), (1024, 4096, 256, 3), (600, 16384, 1024, 3)])
def test_cta_caps_do_not_change_results(z, P, N, L, variant):
    """Capping the persistent compression and CA-CFAR kernels at 1 or 2 CTAs per SM only
    changes how the pulses and tiles are spread: the results are the same bits."""
    from zkx_dev_b200.synth import make_cpi
    cpi = make_cpi(P, N, 10, L, seed=N + variant)
    chain = z.RangeDopplerChain(z.ChainConfig(P, N, L), torch.as_tensor(cpi.replica).cuda())
    x = torch.as_tensor(cpi.x).cuda()
    set_full_tuning(chain, compression_variant=variant, cfar_tile=3)
    ref = {k: v.clone() for k, v in chain(x).items()}
    for k in (1, 2):
        set_full_tuning(chain, compression_variant=variant, cfar_tile=3, compression_ctas_per_sm=k,
                        cfar_ctas_per_sm=k)
        got = chain(x)
        torch.cuda.synchronize()
        for key in ("compressed", "power", "threshold", "detections"):
            assert torch.equal(got[key], ref[key]), (k, key)


def test_tuning_rejects_unknown_choices(z):
    from zkx_dev_b200 import _lib as L
    from zkx_dev_b200.synth import make_cpi
    cpi = make_cpi(64, 1024, 4, 64, seed=3)
    chain = z.RangeDopplerChain(z.ChainConfig(64, 1024, 64), torch.as_tensor(cpi.replica).cuda())
    for kw in ({"compression_radix": 8}, {"compression_ctas_per_sm": -1}, {"cfar_ctas_per_sm": 64},
               {"cfar_tile": 4}, {"compression_variant": 4}):
        t = L.RdTuning(**kw)
        assert L.lib().zkx_rd_plan_set_tuning(chain._plan, ctypes.byref(t)) == L.INVALID_ARGUMENT


@pytest.mark.parametrize("P,N", [(2048, 1024), (4096, 512), (1500, 640)])
def test_long_doppler_tiles_match(z, P, N):
    """Slow-time transforms of 2048 and 4096 bins on the bulk-copy tiles, on 16-byte-misaligned
    input (the per-thread-load kernel) and against the FP64 DFT: the same bits on both paths,
    within FP32 rounding of FP64; both tile widths of the chain give the same bits."""
    import oracle as O
    from zkx_dev_b200 import _lib as L
    rng = np.random.default_rng(P + N)
    xh = (rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))).astype(np.complex64)
    nfft = 1 << (P - 1).bit_length()
    buf = torch.empty(P * N + 1, dtype=torch.complex64, device="cuda")
    mis = buf[1:].view(P, N)
    mis.copy_(torch.as_tensor(xh).cuda())
    x = torch.as_tensor(xh).cuda()
    outs = []
    for src in (x, mis):
        rd = torch.empty((nfft, N), dtype=torch.complex64, device="cuda")
        pw = torch.empty((nfft, N), dtype=torch.float32, device="cuda")
        L.check(L.lib().zkx_pulse_doppler_c64(src.data_ptr(), P, N, nfft, L.WINDOW_HAMMING, None, rd.data_ptr(),
                                              pw.data_ptr(), L.stream_handle()))
        torch.cuda.synchronize()
        outs.append((rd.cpu(), pw.cpu()))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    cols = [0, N // 2, N - 1]
    rd64, _ = O.pulse_doppler_fft64(xh[:, cols], nfft, O.radar_window_f32("hamming", P))
    got = outs[0][0].numpy()[:, cols].astype(np.complex128)
    assert np.linalg.norm(got - rd64) / np.linalg.norm(rd64) <= 1e-5
    # the chain with each tile width
    from zkx_dev_b200.synth import make_cpi
    cpi = make_cpi(P, N, 5, 64, seed=P)
    chain = z.RangeDopplerChain(z.ChainConfig(P, N, 64, doppler_nfft=nfft), torch.as_tensor(cpi.replica).cuda())
    res = []
    for c in ((0, 8, 4) if nfft == 2048 else (0, 4, 2, 1)):   # 0: by shape; 1: per-thread loads
        set_full_tuning(chain, doppler_columns=c)
        o = chain(torch.as_tensor(cpi.x).cuda())
        torch.cuda.synchronize()
        res.append({k: o[k].clone() for k in ("rd", "power", "detections")})
    for r in res[1:]:
        for k in res[0]:
            assert torch.equal(res[0][k], r[k]), k
    assert L.kernel_status(clear=True) == 0


def test_cfar_tiles_on_task1_window(z):
    """Task1's CA-CFAR window (guard 1 x 2, reference 2 x 6) runs the tiled kernels: every tile
    choice gives the FP64 CFAR's mask, the full and persistent tiles the same thresholds."""
    import oracle as O
    from zkx_dev_b200.synth import make_cpi
    P, N = 128, 4096
    cpi = make_cpi(P, N, 12, 256, seed=77)
    chain = z.RangeDopplerChain(z.ChainConfig(P, N, 256, guard_cells=(1, 2), reference_cells=(2, 6), pfa=1e-4),
                                torch.as_tensor(cpi.replica).cuda())
    x = torch.as_tensor(cpi.x).cuda()
    outs = {}
    for tile in (1, 2, 3):
        set_tuning(chain, 0, 0, tile)
        o = chain(x)
        torch.cuda.synchronize()
        outs[tile] = {k: o[k].cpu().numpy().copy() for k in ("power", "threshold", "detections")}
    _, m64 = O.ca_cfar_f64(outs[1]["power"], (1, 2), (2, 6), 1e-4)
    for tile in (1, 2, 3):
        np.testing.assert_array_equal(outs[tile]["detections"], m64)
    np.testing.assert_array_equal(outs[3]["threshold"], outs[1]["threshold"])
