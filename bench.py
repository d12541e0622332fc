"""Benchmark: the radar front end + range-Doppler chain at scale on B200.

Workload (one step = one CPI):
  front end  16 channels x 2^20 float32 -> 127-tap Kaiser(8) lowpass firfilter ->
             resample_poly 3/2 (default Kaiser(5), 61 taps) -> 16 x 1572864 float32
  chain      1024 pulses x 16384 range complex64 CPI (64 targets, 1024-sample LFM
             chirp) -> pulse_compression (Hamming replica, normalised) ->
             pulse_doppler (Hamming over pulses) + |.|^2 -> 2-D CA-CFAR
             (guard 2x2, train 8x8, Pfa 1e-6)
Inputs are seeded synthetic data; each timed step reads a different input set (three
rotating sets, every set larger than the 126 MB L2), so no step starts with its inputs
cached.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun, one rank per GPU) runs independent replicas: CPIs are independent,
there is no data exchange; the barrier and the max-over-ranks time are the only
collectives.  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "CPIs/sec + HBM GB/s, range-Doppler+CFAR; p99 latency; rel err vs FP64"
UNIT = "CPIs/s"
WORKLOAD = "front end 16x2^20 fir127+resample_poly 3/2 + range-Doppler-CFAR 1024x16384"

P, NR, L = 1024, 16384, 1024
CH, NS = 16, 1 << 20
FIR_TAPS, FIR_BETA, FIR_CUTOFF = 127, 8.0, 0.3
UP, DOWN = 3, 2
N_TARGETS = 64
CELLS = P * NR

# algorithmic bytes per launch (compulsory reads + writes)
ALG_BYTES = {
    "fir": CH * NS * 8,
    "resample_poly": CH * NS * 4 + CH * (NS * UP // DOWN) * 4,
    "pulse_compression": CELLS * 16,
    "pulse_doppler": CELLS * 20,
    "ca_cfar": CELLS * 9,
}


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic():
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh)
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------- our arm

def run_ours(args, rank: int, world: int, dist) -> dict:
    import torch
    import zkx_dev_b200 as z
    from zkx_dev_b200 import synth

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()

    # inputs: three rotating sets (host pinned + device copies)
    n_sets = 1 if args.profile else 3
    host_fe, host_cube = [], []
    for i in range(n_sets):
        seed = synth.seed_for(2, rank * 100 + i)
        host_fe.append(torch.from_numpy(synth.make_front_end(CH, NS, seed)).pin_memory())
        cpi = synth.make_cpi(P, NR, N_TARGETS, L, seed)
        host_cube.append(torch.from_numpy(cpi.x).pin_memory())
        replica = cpi.replica
    dev_fe = [h.to(dev) for h in host_fe]
    dev_cube = [h.to(dev) for h in host_cube]

    taps_fir = torch.as_tensor(synth.firwin_kaiser(FIR_TAPS, FIR_CUTOFF, FIR_BETA).astype(np.float32), device=dev)
    taps_rs = torch.as_tensor(z.resample_poly_taps(NS, UP, DOWN, 5.0).astype(np.float32), device=dev)
    chain = z.RangeDopplerChain(z.ChainConfig(P, NR, L, pfa=1e-6), torch.as_tensor(replica, device=dev))
    # set-up: per-shape kernel choices, outside the timed region; the profiling pass keeps the
    # by-shape defaults, since timings taken under a profiler would choose arbitrarily
    tuning = chain.tuning if args.profile else chain.autotune(dev_cube[0])
    out = chain.allocate_outputs()
    fir_out = torch.empty((CH, NS), dtype=torch.float32, device=dev)
    from zkx_dev_b200 import _lib as LB
    import ctypes
    lay = z.filtering.resample_layout(NS, UP, DOWN)
    rs_out = torch.empty((CH, lay.output_samples), dtype=torch.float32, device=dev)
    lib = LB.lib()
    sh = LB.stream_handle()

    def front_end(x, on=None):
        h = sh if on is None else on
        LB.check(lib.zkx_fir_f32(taps_fir.data_ptr(), FIR_TAPS, x.data_ptr(), CH, NS, None,
                                 fir_out.data_ptr(), None, h))
        LB.check(lib.zkx_resample_poly_f32(fir_out.data_ptr(), CH, NS, ctypes.byref(lay),
                                           taps_rs.data_ptr(), rs_out.data_ptr(), h))

    # A step: the front end (FIR, resample_poly) and the range-Doppler chain of one CPI; the
    # two are independent, so the front end runs on its own stream beside the chain (each
    # fills the other's partial waves).  With --lanes L, L steps are in flight: step i runs on
    # lane i % L (a front-end stream, a chain stream and its own output buffers); step i+L
    # reuses step i's lane, whose stream order protects its buffers.
    fe_stream = torch.cuda.Stream(device=dev)
    fe_sh = fe_stream.cuda_stream
    fe_events = [torch.cuda.Event() for _ in range(4)]
    lanes = max(1, args.lanes)
    # the chain's streams get the device's highest scheduling priority and the front end's the
    # lowest (unless --equal-priority), so pending chain CTAs are placed first and the front
    # end fills what the chain leaves
    lo, hi = torch.cuda.Stream.priority_range()
    prio = not args.equal_priority
    lane_chain = [torch.cuda.Stream(device=dev, priority=hi if prio else 0) for _ in range(lanes)]
    lane_fe = [torch.cuda.Stream(device=dev, priority=lo if prio else 0) for _ in range(lanes)]
    lane_out = [out] + [chain.allocate_outputs() for _ in range(lanes - 1)]
    lane_fir = [fir_out] + [torch.empty_like(fir_out) for _ in range(lanes - 1)]
    lane_rs = [rs_out] + [torch.empty_like(rs_out) for _ in range(lanes - 1)]

    def step(i):
        k, ln = i % n_sets, i % lanes
        h = lane_fe[ln].cuda_stream
        LB.check(lib.zkx_fir_f32(taps_fir.data_ptr(), FIR_TAPS, dev_fe[k].data_ptr(), CH, NS, None,
                                 lane_fir[ln].data_ptr(), None, h))
        LB.check(lib.zkx_resample_poly_f32(lane_fir[ln].data_ptr(), CH, NS, ctypes.byref(lay),
                                           taps_rs.data_ptr(), lane_rs[ln].data_ptr(), h))
        with torch.cuda.stream(lane_chain[ln]):
            chain(dev_cube[k], lane_out[ln])

    def lanes_begin():
        ev = torch.cuda.Event()
        ev.record(stream)
        for s_ in lane_chain + lane_fe:
            s_.wait_event(ev)

    def lanes_end():
        for s_ in lane_chain + lane_fe:
            ev = torch.cuda.Event()
            ev.record(s_)
            stream.wait_event(ev)

    # warm-up
    lanes_begin()
    for i in range(args.warmup):
        step(i)
    lanes_end()
    torch.cuda.synchronize()
    if args.profile:
        lanes_begin()
        step(0)
        lanes_end()
        torch.cuda.synchronize()
        chain.close()
        return None

    # per-stage timing (separate pass, kernels bracketed by events)
    stage_ms = {k: [] for k in ("fir", "resample_poly", "pulse_compression", "pulse_doppler", "ca_cfar")}
    step_ms = []
    for i in range(max(3, args.steps)):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        k = i % n_sets
        ev[0].record(stream)
        LB.check(lib.zkx_fir_f32(taps_fir.data_ptr(), FIR_TAPS, dev_fe[k].data_ptr(), CH, NS, None,
                                 fir_out.data_ptr(), None, sh))
        ev[1].record(stream)
        LB.check(lib.zkx_resample_poly_f32(fir_out.data_ptr(), CH, NS, ctypes.byref(lay),
                                           taps_rs.data_ptr(), rs_out.data_ptr(), sh))
        ev[2].record(stream)
        LB.check(lib.zkx_pulse_compression_spectrum_c64(dev_cube[k].data_ptr(), P, NR, NR,
                                                        chain_spectrum(chain), out["compressed"].data_ptr(), sh))
        ev[3].record(stream)
        LB.check(lib.zkx_pulse_doppler_c64(out["compressed"].data_ptr(), P, NR, P, LB.WINDOW_HAMMING, None,
                                           out["rd"].data_ptr(), out["power"].data_ptr(), sh))
        ev[4].record(stream)
        LB.check(lib.zkx_ca_cfar_f32(out["power"].data_ptr(), 2, P, NR, 2, 2, 8, 8, 1e-6, LB.CFAR_ACCURATE,
                                     out["threshold"].data_ptr(), out["detections"].data_ptr(), sh))
        ev[5].record(stream)
        torch.cuda.synchronize()
        for j, name in enumerate(stage_ms):
            stage_ms[name].append(ev[j].elapsed_time(ev[j + 1]))
        step_ms.append(ev[0].elapsed_time(ev[5]))

    # timed region: K steps, device time, max over ranks
    clocks = ClockSampler(dev.index)
    clocks.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    lanes_begin()
    for i in range(args.steps):
        step(i)
    lanes_end()
    t1.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    elapsed_ms = t0.elapsed_time(t1)

    # end to end through the public API with host buffers: H2D of every step's inputs from
    # page-locked memory, the computation, D2H of its detection mask.  Copies run on their
    # own streams and are double-buffered, so step i+1's inputs cross PCIe while step i
    # computes and step i-1's mask comes back.
    h2d = CH * NS * 4 + CELLS * 8
    d2h = CELLS
    copy_s = torch.cuda.Stream(device=dev)
    back_s = torch.cuda.Stream(device=dev)
    ins = [(torch.empty((CH, NS), dtype=torch.float32, device=dev),
            torch.empty((P, NR), dtype=torch.complex64, device=dev)) for _ in range(2)]
    outs = [out, chain.allocate_outputs()]
    host_det = [torch.empty((P, NR), dtype=torch.uint8).pin_memory() for _ in range(2)]
    copied = [torch.cuda.Event() for _ in range(2)]
    computed = [torch.cuda.Event() for _ in range(2)]
    drained = [torch.cuda.Event() for _ in range(2)]
    for ev in copied + computed + drained:
        ev.record(stream)

    def e2e_step(i):
        b = i % 2
        with torch.cuda.stream(copy_s):
            copy_s.wait_event(computed[b])           # the step that last read ins[b] is done
            ins[b][0].copy_(host_fe[i % n_sets], non_blocking=True)
            ins[b][1].copy_(host_cube[i % n_sets], non_blocking=True)
            copied[b].record(copy_s)
        stream.wait_event(copied[b])
        stream.wait_event(drained[b])                # outs[b]'s mask has been read back
        start, done = fe_events[2 * b], fe_events[2 * b + 1]
        start.record(stream)
        fe_stream.wait_event(start)
        front_end(ins[b][0], fe_sh)                  # beside the chain, as in the timed steps
        done.record(fe_stream)
        chain(ins[b][1], outs[b])
        stream.wait_event(done)
        computed[b].record(stream)
        with torch.cuda.stream(back_s):
            back_s.wait_event(computed[b])
            host_det[b].copy_(outs[b]["detections"], non_blocking=True)
            drained[b].record(back_s)

    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for i in range(2):
        e2e_step(i)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0.record(stream)
    for i in range(args.steps):
        e2e_step(i)
    stream.wait_event(drained[0])
    stream.wait_event(drained[1])
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    clk = clocks.stop()

    # per-step end-to-end latency (host buffers in, mask out, one step at a time), a
    # separate bounded pass
    e2e_step_ms = []
    for i in range(min(args.steps, 50)):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ins[0][0].copy_(host_fe[i % n_sets], non_blocking=True)
        ins[0][1].copy_(host_cube[i % n_sets], non_blocking=True)
        front_end(ins[0][0])
        chain(ins[0][1], out)
        host_det[0].copy_(out["detections"], non_blocking=True)
        b.record(stream)
        b.synchronize()
        e2e_step_ms.append(a.elapsed_time(b))

    # accuracy of this run's outputs against an FP64 recomputation (sampled)
    chain(dev_cube[0], out)
    torch.cuda.synchronize()
    errors = fp64_errors(host_cube[0].numpy(), replica, out)

    if dist is not None:
        from zkx_dev_b200.replicas import max_over_ranks
        elapsed_ms, e2e_ms = max_over_ranks([elapsed_ms, e2e_ms], dist, dev)

    chain.close()
    per_stage = {k: statistics.median(v) for k, v in stage_ms.items()}
    dominant = max(per_stage, key=per_stage.get)
    peak, peak_kind = _peaks()
    achieved = ALG_BYTES[dominant] / (per_stage[dominant] * 1e-3) / 1e9
    traffic = _traffic().get(dominant)
    stage_gbs = {k: round(ALG_BYTES[k] / (v * 1e-3) / 1e9, 1) for k, v in per_stage.items()}
    return {
        "value": world * args.steps / (elapsed_ms * 1e-3),
        "ms_per_step": elapsed_ms / args.steps,
        "e2e": {"value": world * args.steps / (e2e_ms * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1),
                     "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic},
        "stages_ms": {k: round(v, 4) for k, v in per_stage.items()},
        "stages_gbs": stage_gbs,
        "chain_gbs": round(sum(ALG_BYTES.values()) / (elapsed_ms / args.steps * 1e-3) / 1e9, 1),
        # per step: FIR tap spectrum + FIR, resample_poly, compression, Doppler, CFAR
        "gpu_launches": 6 * args.steps,
        "clocks": clk,
        "latency_ms": {"step_p50": round(percentile(step_ms, 50), 4),
                       "step_p99": round(percentile(step_ms, 99), 4),
                       "e2e_p50": round(percentile(e2e_step_ms, 50), 4),
                       "e2e_p99": round(percentile(e2e_step_ms, 99), 4)},
        "rel_err_vs_fp64": errors,
        "tuning": tuning,
    }


def percentile(values, q: float) -> float:
    v = sorted(values)
    return v[min(len(v) - 1, max(0, int(np.ceil(q / 100.0 * len(v))) - 1))]


def hamming_f32(n: int) -> np.ndarray:
    """The symmetric Hamming window as the kernels apply it: FP64 formula rounded to FP32."""
    k = np.arange(n, dtype=np.float64)
    return (0.54 - 0.46 * np.cos(2.0 * np.pi * k / (n - 1))).astype(np.float32).astype(np.float64)


def cfar_fp64_plane(power: np.ndarray, guard=(2, 2), train=(8, 8), pfa: float = 1e-6) -> np.ndarray:
    """FP64 CA-CFAR thresholds of a whole power plane: per row the full-width and the two
    side-band training sums, then along columns the full-width sums of the training rows
    plus the side-band sums of the guard rows.  Each is a direct FP64 sum of the plane's
    own cells (sliding windows, no running-sum differences), so a target's power cannot
    cancel against its neighbours'.  Border cells (incomplete window) get threshold 0."""
    from numpy.lib.stride_tricks import sliding_window_view as swv
    gr, gc = guard
    tr, tc = train
    rm, cm = gr + tr, gc + tc
    p = np.asarray(power, dtype=np.float64)
    R, C = p.shape
    nc = C - 2 * cm
    side = swv(p, tc, axis=1)[:, 0:nc].sum(axis=-1)
    side += swv(p, tc, axis=1)[:, cm + gc + 1:cm + gc + 1 + nc].sum(axis=-1)
    full = swv(p, 2 * cm + 1, axis=1)[:, 0:nc].sum(axis=-1)
    nr = R - 2 * rm
    ring = swv(full, tr, axis=0)[0:nr].sum(axis=-1)
    ring += swv(full, tr, axis=0)[rm + gr + 1:rm + gr + 1 + nr].sum(axis=-1)
    ring += swv(side, 2 * gr + 1, axis=0)[rm - gr:rm - gr + nr].sum(axis=-1)
    nref = (2 * rm + 1) * (2 * cm + 1) - (2 * gr + 1) * (2 * gc + 1)
    alpha = nref * (pfa ** (-1.0 / nref) - 1.0)
    t64 = np.zeros((R, C), dtype=np.float64)
    t64[rm:R - rm, cm:C - cm] = alpha / nref * ring
    return t64


def fp64_errors(x: np.ndarray, replica: np.ndarray, out) -> dict:
    """Errors of the chain's outputs against numpy FP64: relative L2 on 16 pulses of the
    compressed cube and on 64 range columns of the range-Doppler map and power (computed
    from the GPU's compressed cube, so each stage is measured on its own input); the CFAR
    on the WHOLE plane: every cell's decision against an FP64 CFAR of the GPU's power
    (mask mismatches), the largest relative threshold error over all interior cells, and
    the number of cells within 1e-5 relative of their FP64 threshold."""
    import torch
    rng = np.random.default_rng(7)
    pulses, nr = x.shape
    rows = np.sort(rng.choice(pulses, 16, replace=False))
    h = replica.astype(np.complex128) * hamming_f32(replica.size)
    h /= np.linalg.norm(h)
    spec = np.conj(np.fft.fft(h, nr))
    comp64 = np.fft.ifft(np.fft.fft(x[rows].astype(np.complex128), axis=1) * spec, axis=1)
    comp = out["compressed"].cpu().numpy()
    cols = np.sort(rng.choice(nr, 64, replace=False))
    rd64 = np.fft.fft(comp[:, cols].astype(np.complex128) * hamming_f32(pulses)[:, None], axis=0)
    rd = out["rd"][:, torch.as_tensor(cols)].cpu().numpy()
    power = out["power"].cpu().numpy()
    pow64 = np.abs(rd64) ** 2
    thr = out["threshold"].cpu().numpy()
    det = out["detections"].cpu().numpy()
    t64 = cfar_fp64_plane(power)
    interior = t64 > 0
    p64 = power.astype(np.float64)

    def rel(a, b):
        return float(np.linalg.norm((np.asarray(a) - b).ravel()) / np.linalg.norm(b.ravel()))

    return {"compressed": rel(comp[rows], comp64), "rd": rel(rd, rd64),
            "power": rel(p64[:, cols], pow64),
            "threshold_max": float(np.max(np.abs(thr[interior] - t64[interior]) / t64[interior])),
            "mask_mismatches": int(np.count_nonzero(det != (p64 > t64))),
            "near_threshold_cells": int(np.count_nonzero(np.abs(p64 - t64) <= 1e-5 * t64)),
            "detections": int(np.count_nonzero(det)),
            "sample": f"16 pulses; 64 range columns; CFAR over all {pulses * nr} cells"}


def mixed_requests(n_requests: int = 256, pool: int = 24):
    """The mixed-size stream's seeded pool of CPIs (pulses 2^U{6..10}, range 2^U{10..15}, 5-50
    targets, chirp range/16) and the pool indices of `n_requests` requests drawn from it."""
    from zkx_dev_b200 import synth
    rng = np.random.default_rng(synth.seed_for(4, 0))
    cpis = []
    for i in range(pool):
        P_, N_ = int(2 ** rng.integers(6, 11)), int(2 ** rng.integers(10, 16))
        cpis.append(synth.make_cpi(P_, N_, int(rng.integers(5, 51)), N_ // 16, synth.seed_for(4, i + 1)))
    order = [int(rng.integers(0, pool)) for _ in range(n_requests)]
    return cpis, order


def profile_mixed() -> None:
    """The mixed-size batch (256 requests) once as per-shape stacked batches and once as one
    work list, after one untimed pass of each, inside a profiler range (the command profiled
    for the work-list launch list: ncu --profile-from-start off)."""
    import torch
    import zkx_dev_b200 as z
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cpis, order = mixed_requests()
    dev_x = [torch.as_tensor(c.x, device=dev) for c in cpis]
    chains = {}
    for c in cpis:
        if c.x.shape not in chains:
            P_, N_ = c.x.shape
            chains[c.x.shape] = z.RangeDopplerChain(z.ChainConfig(P_, N_, N_ // 16), torch.as_tensor(c.replica, device=dev))
    groups = {}
    for k in order:
        groups.setdefault(cpis[k].x.shape, []).append(k)
    stacked = []
    for shp, ks in groups.items():
        ch = chains[shp]
        stacked.append((ch, torch.stack([dev_x[k] for k in ks]),
                        ch.allocate_outputs(keep_compressed=False, keep_rd=False, batch=len(ks))))
    items = []
    for k in order:
        ch = chains[cpis[k].x.shape]
        shp = (ch.doppler_bins, ch.range_bins)
        items.append((ch, dev_x[k], {"threshold": torch.empty(shp, device=dev),
                                     "detections": torch.empty(shp, dtype=torch.uint8, device=dev)}))
    wl = z.WorkList(items)

    def per_shape():
        for ch, xb, ob in stacked:
            ch.run_batch(xb, ob)
    for f in (per_shape, wl.launch):
        f()
        torch.cuda.synchronize()
    torch.cuda.profiler.start()
    per_shape()
    torch.cuda.synchronize()
    wl.launch()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    wl.close()
    for ch in chains.values():
        ch.close()


def run_serving(dev, n_requests: int = 256, pool: int = 24, seconds: float = 2.0) -> dict:
    """The mixed-size stream: pulses 2^U{6..10}, range 2^U{10..15}, 5-50 targets, chirp
    length range/16, Hamming windows, CFAR guard 2x2 train 8x8 Pfa 1e-6.  A pool of `pool`
    seeded CPIs is drawn from that distribution and `n_requests` requests are drawn from
    the pool.  Measures (1) the plain path, one CPI per launch sequence on one stream,
    (1b) the same requests grouped by shape into stacked batches captured as one CUDA graph,
    (2) the serving loop on device-resident buffers and (3) with page-locked host
    buffers (copies included), all submitted at once, then (4) the serving loop under
    Poisson arrivals at 70 % of (3)'s rate for `seconds`, for its latency."""
    import random
    import torch
    import zkx_dev_b200 as z
    from zkx_dev_b200 import synth

    cpis, order = mixed_requests(n_requests, pool)
    dev_x = [torch.as_tensor(c.x, device=dev) for c in cpis]
    host_x = [torch.as_tensor(c.x).pin_memory() for c in cpis]
    replicas = {}
    for c in cpis:
        replicas.setdefault(c.x.shape, torch.as_tensor(c.replica, device=dev))
    cells = sum(cpis[k].x.size for k in order)

    # (1) plain: one RangeDopplerChain per shape, one CPI after another on one stream
    chains = {}
    for c in cpis:
        P_, N_ = c.x.shape
        if c.x.shape not in chains:
            ch = z.RangeDopplerChain(z.ChainConfig(P_, N_, N_ // 16), replicas[c.x.shape])
            chains[c.x.shape] = (ch, ch.allocate_outputs(keep_compressed=False, keep_rd=False))
    for k in range(pool):
        ch, o = chains[cpis[k].x.shape]
        ch.run(dev_x[k], o)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for k in order:
        ch, o = chains[cpis[k].x.shape]
        ch.run(dev_x[k], o)
    b.record()
    b.synchronize()
    plain = n_requests / (a.elapsed_time(b) * 1e-3)

    # (1b) the uneven batch as one CUDA graph: the requests grouped by shape, each group one
    # stacked batch (one launch per stage), every group captured into a single graph
    groups = {}
    for k in order:
        groups.setdefault(cpis[k].x.shape, []).append(k)
    stacked = []
    for shp, ks in groups.items():
        ch, _ = chains[shp]
        xb = torch.stack([dev_x[k] for k in ks])
        ob = ch.allocate_outputs(keep_compressed=False, keep_rd=False, batch=len(ks))
        ch.run_batch(xb, ob)                         # plan-owned buffers sized before capture
        stacked.append((ch, xb, ob))
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for ch, xb, ob in stacked:
            ch.run_batch(xb, ob)
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    a.record()
    reps = 5
    for _ in range(reps):
        graph.replay()
    b.record()
    b.synchronize()
    uneven_graph = reps * n_requests / (a.elapsed_time(b) * 1e-3)
    del graph, stacked

    # (1c) the same requests as one work list: one launch per stage over every (CPI, tile)
    # entry of every shape (stages the work-list kernels do not take run on their plan's
    # kernels), captured as one CUDA graph
    items = []
    for k in order:
        ch, _ = chains[cpis[k].x.shape]
        shp = (ch.doppler_bins, ch.range_bins)
        items.append((ch, dev_x[k], {"threshold": torch.empty(shp, device=dev),
                                     "detections": torch.empty(shp, dtype=torch.uint8, device=dev)}))
    wl = z.WorkList(items)
    wl_info = wl.info()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        wl.launch()
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        wl.launch()
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    a.record()
    for _ in range(reps):
        graph.replay()
    b.record()
    b.synchronize()
    worklist_graph = reps * n_requests / (a.elapsed_time(b) * 1e-3)
    # each shape's first request against its CPI alone
    wl_identical = True
    seen = set()
    for (ch, x, o) in items:
        if ch in seen:
            continue
        seen.add(ch)
        ref = ch.run(x)
        wl_identical &= bool(torch.equal(ref["detections"], o["detections"]) and
                             torch.equal(ref["threshold"], o["threshold"]))
    del graph, items
    wl.close()
    for ch, _ in chains.values():
        ch.close()

    def burst(server, xs, outs):
        tickets = [server.submit(xs[k], replicas[cpis[k].x.shape], cpis[k].x.shape[0] * 100000 + cpis[k].x.shape[1],
                                 outs[k]) for k in order]
        for t in tickets:
            server.wait(t)

    dev_det = [torch.empty(c.x.shape, dtype=torch.uint8, device=dev) for c in cpis]
    host_det = [torch.empty(c.x.shape, dtype=torch.uint8).pin_memory() for c in cpis]
    res = {}
    with z.RdServer(z.ServerConfig()) as server:
        burst(server, dev_x, dev_det)            # builds the plans, warms the pool
        server.reset_stats()
        burst(server, dev_x, dev_det)
        st_dev = server.stats()
        server.reset_stats()
        burst(server, host_x, host_det)
        st_host = server.stats()
        # Poisson arrivals at 70 % of the host-buffer burst rate
        rate = 0.7 * st_host["cpis_per_s"]
        server.reset_stats()
        prng = random.Random(11)
        tickets = []
        t_next = time.perf_counter()
        t_end = t_next + seconds
        i = 0
        while t_next < t_end:
            while time.perf_counter() < t_next:
                pass
            k = order[i % n_requests]
            tickets.append(server.submit(host_x[k], replicas[cpis[k].x.shape],
                                         cpis[k].x.shape[0] * 100000 + cpis[k].x.shape[1], host_det[k]))
            i += 1
            t_next += prng.expovariate(rate)
        for t in tickets:
            server.wait(t)
        st_poisson = server.stats()
    res = {
        "workload": (f"mixed stream: {n_requests} CPIs drawn from {pool} seeded CPIs with pulses "
                     "2^U{6..10}, range 2^U{10..15}, chirp range/16, 5-50 targets"),
        "cells": cells,
        "plain_device_cpis_per_s": round(plain, 1),
        "uneven_graph_cpis_per_s": round(uneven_graph, 1),
        "uneven_graph_shapes": len(groups),
        "worklist_graph_cpis_per_s": round(worklist_graph, 1),
        "worklist_launches": wl_info["launches"],
        "worklist_identical_to_alone": wl_identical,
        "served_device_cpis_per_s": round(st_dev["cpis_per_s"], 1),
        "served_vs_plain_device": round(st_dev["cpis_per_s"] / plain, 3),
        "served_device_gbs": round(st_dev["cpis_per_s"] * cells / n_requests * 45 / 1e9, 1),
        "served_host_cpis_per_s": round(st_host["cpis_per_s"], 1),
        "mean_batch": round(st_dev["mean_batch"], 2),
        "poisson_rate_cpis_per_s": round(rate, 1),
        "poisson_requests": int(st_poisson["completed"]),
        "poisson_p50_ms": round(st_poisson["p50_us"] / 1e3, 3),
        "poisson_p99_ms": round(st_poisson["p99_us"] / 1e3, 3),
        "poisson_cpis_per_s": round(st_poisson["cpis_per_s"], 1),
        "buffers": "device: inputs and masks in HBM; host: page-locked inputs in, masks out",
    }
    return res


def run_precision(dev) -> dict:
    """The precision comparison: one 512 x 8192 CPI (40 targets, chirp 512, 5 % of the targets
    at 0-3 dB SNR near the threshold), the chain with range compression in plain FP32 and as
    tensor-core DFT GEMMs with split hi+lo FP16 / BF16 operands, against a full FP64 chain
    (numpy): relative L2 and max |error| / max |reference| of the compressed cube and of the
    power map, and detection-mask cells that differ from the FP64 chain's CA-CFAR."""
    import torch
    import zkx_dev_b200 as z
    from zkx_dev_b200 import synth
    P_, N_, L_ = 512, 8192, 512
    cpi = synth.make_cpi(P_, N_, 40, L_, synth.seed_for(3, 0), low_snr_fraction=0.05, low_snr_db=(0.0, 3.0))
    h = cpi.replica.astype(np.complex128) * hamming_f32(L_)
    h /= np.linalg.norm(h)
    comp64 = np.fft.ifft(np.fft.fft(cpi.x.astype(np.complex128), axis=1) * np.conj(np.fft.fft(h, N_)), axis=1)
    pow64 = np.abs(np.fft.fft(comp64 * hamming_f32(P_)[:, None], axis=0)) ** 2
    gr, gc, tr, tc = 2, 2, 8, 8
    nref = (2 * (gr + tr) + 1) * (2 * (gc + tc) + 1) - (2 * gr + 1) * (2 * gc + 1)
    alpha = nref * (1e-6 ** (-1.0 / nref) - 1.0)
    cum = np.zeros((P_ + 1, N_ + 1))
    cum[1:, 1:] = np.cumsum(np.cumsum(pow64, axis=0), axis=1)

    def box(r0, r1, c0, c1):  # sums of pow64[r0:r1, c0:c1] for arrays of corners
        return cum[r1, c1] - cum[r0, c1] - cum[r1, c0] + cum[r0, c0]

    rr, cc = np.meshgrid(np.arange(gr + tr, P_ - gr - tr), np.arange(gc + tc, N_ - gc - tc), indexing="ij")
    outer = box(rr - gr - tr, rr + gr + tr + 1, cc - gc - tc, cc + gc + tc + 1)
    inner = box(rr - gr, rr + gr + 1, cc - gc, cc + gc + 1)
    mask64 = pow64[rr, cc] > alpha / nref * (outer - inner)

    def rel(a, b):
        return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))

    res = {"workload": "512x8192 CPI, 40 targets (5% at 0-3 dB), chirp 512, Hamming, CFAR 2x2/8x8 1e-6",
           "reference": "FP64 chain (numpy)"}
    x = torch.as_tensor(cpi.x, device=dev)
    for prec in ("fp32", "tc_f16", "tc_bf16"):
        chain = z.RangeDopplerChain(z.ChainConfig(P_, N_, L_, pfa=1e-6, precision=prec),
                                    torch.as_tensor(cpi.replica, device=dev))
        out = chain.run(x)
        torch.cuda.synchronize()
        comp = out["compressed"].cpu().numpy().astype(np.complex128)
        power = out["power"].cpu().numpy().astype(np.float64)
        det = out["detections"].cpu().numpy()[rr, cc].astype(bool)
        res[prec] = {"compressed_rel_l2": rel(comp, comp64),
                     "compressed_max_rel": float(np.max(np.abs(comp - comp64)) / np.max(np.abs(comp64))),
                     "power_rel_l2": rel(power, pow64),
                     "power_max_rel": float(np.max(np.abs(power - pow64)) / np.max(pow64)),
                     "mask_cells_differing_from_fp64": int(np.sum(det != mask64)),
                     "detections": int(det.sum()), "detections_fp64": int(mask64.sum())}
        chain.close()
    return res


def run_serving_sweep(dev, rates=(1000, 2000, 5000, 10000, 20000, 50000), seconds: float = 10.0,
                      pool: int = 24, max_pending: int = 256) -> dict:
    """Poisson arrivals of device-resident CPIs at the offered rates of the serving
    configuration (1 k to 50 k CPIs/s; 10 s per rate instead of 60 s, to keep the whole
    bench within a few minutes): the mixed-size stream (pulses 2^U{6..10}, range
    2^U{10..15}, chirp range/16) with 10 % large 2048 x 65536 CPIs, all generated on the
    device.  The server bounds its admission queue (max_pending): arrivals beyond it are
    refused at once and counted as shed, so an overloaded server shows its plateau instead
    of an unbounded backlog.  Per rate: the offered rate actually generated, accepted and
    shed requests, completed CPIs/s and latency p50/p99/max of the accepted ones (submit ->
    mask in the caller's device buffer)."""
    import random
    import torch
    import zkx_dev_b200 as z
    from zkx_dev_b200 import synth

    rng = np.random.default_rng(synth.seed_for(5, 0))
    shapes = [(int(2 ** rng.integers(6, 11)), int(2 ** rng.integers(10, 16))) for _ in range(pool)]
    shapes += [(2048, 65536)] * 2
    cpis, replicas = [], {}
    for i, (P_, N_) in enumerate(shapes):
        L_ = N_ // 16
        targets = synth.draw_targets(P_, N_, int(rng.integers(5, 51)), L_, synth.seed_for(5, i + 1))
        cpis.append(synth.device_cpi(P_, N_, targets, L_, synth.seed_for(5, i + 101)))
        if (P_, N_) not in replicas:
            replicas[(P_, N_)] = torch.as_tensor(synth.lfm_chirp(L_).astype(np.complex64), device=dev)
    dets = [torch.empty(c.shape, dtype=torch.uint8, device=dev) for c in cpis]
    small, large = list(range(pool)), [pool, pool + 1]
    prng = random.Random(13)

    def pick():
        return prng.choice(large) if prng.random() < 0.1 else prng.choice(small)

    res = {"workload": ("Poisson arrivals, device-resident CPIs: pulses 2^U{6..10} x range 2^U{10..15} "
                        "plus 10% 2048x65536, chirp range/16, 5-50 targets"), "seconds_per_rate": seconds,
           "max_pending": max_pending, "rates": []}
    with z.RdServer(z.ServerConfig(max_pending=max_pending)) as server:
        def submit(k):
            P_, N_ = cpis[k].shape
            return server.submit(cpis[k], replicas[(P_, N_)], P_ * 100000 + N_, dets[k])

        def submit_or_shed(k):
            try:
                return submit(k)
            except z.ZkxError as e:
                if e.code != 3002:
                    raise
                return None
        for _ in range(2):   # plans and the workspaces of the batch sizes bursts form
            for t in [submit_or_shed(pick()) for _ in range(4 * len(cpis))]:
                if t is not None:
                    server.wait(t)
        for rate in rates:
            server.reset_stats()
            tickets, shed, offered = [], 0, 0
            t0 = t_next = time.perf_counter()
            t_end = t_next + seconds
            while t_next < t_end:
                while time.perf_counter() < t_next:
                    pass
                t = submit_or_shed(pick())
                offered += 1
                if t is None:
                    shed += 1
                else:
                    tickets.append(t)
                t_next += prng.expovariate(rate)
            window = time.perf_counter() - t0
            for t in tickets:
                server.wait(t)
            st = server.stats()
            res["rates"].append({"offered_cpis_per_s": rate, "generated_cpis_per_s": round(offered / window, 1),
                                 "accepted": len(tickets), "shed": shed, "completed": int(st["completed"]),
                                 "cpis_per_s": round(st["cpis_per_s"], 1),
                                 "p50_ms": round(st["p50_us"] / 1e3, 3), "p99_ms": round(st["p99_us"] / 1e3, 3),
                                 "max_ms": round(st["max_us"] / 1e3, 3)})
    return res


def chain_spectrum(chain) -> int:
    """Device pointer of a plan's resident replica spectrum, via a fresh spectrum call
    with the plan's settings (kept alive on the chain object)."""
    import zkx_dev_b200 as z
    if not hasattr(chain, "_bench_spectrum"):
        chain._bench_spectrum = z.replica_spectrum(chain._keep[0], chain.range_bins, normalize=True,
                                                   window="hamming")
    return chain._bench_spectrum.data_ptr()


# ---------------------------------------------------------------- reference arm

class CpuChain:
    """The reference's CPU implementation of one bench step (oracle/_ref: the reference's
    own *_typed_cpu<float> functions; the repository's C restatement only where that
    library was not built), over the WHOLE workload, computed as a chain:

      firfilter (127 taps) on all 16 x 2^20 channels -> resample_poly 3/2 of its output;
      pulse_compression of all 1024 pulses -> pulse_doppler of all 16384 range columns of
      the compressed cube -> |.|^2 -> ca_cfar of the whole 1024 x 16384 power plane.

    Work is split across host threads the way the operators allow it without changing
    their results: one channel per task for the front end, slices of pulses for
    compression, slices of range columns for Doppler; the CFAR (17 ms) runs as one call.
    The reference itself is single-threaded (ZKX/test_all/operators/shared/radartools/
    radartools_operator_probe.cu:49-60 times each call on one thread)."""

    def __init__(self, threads: int, pulses: int = P, samples: int = NR, chirp: int = L,
                 targets: int = N_TARGETS, channels: int = CH, channel_samples: int = NS,
                 seed: int = 0):
        import oracle as O
        from zkx_dev_b200 import synth
        self.O = O
        self.kind = "port" if O.reference() is None else "reference"
        self.threads = threads
        self.cpi = synth.make_cpi(pulses, samples, targets, chirp, seed)
        self.fe = synth.make_front_end(channels, channel_samples, seed) if channels else None
        self.fir_taps = synth.firwin_kaiser(FIR_TAPS, FIR_CUTOFF, FIR_BETA).astype(np.float32)

    def _slices(self, n: int):
        k = max(1, min(n, 4 * self.threads))
        bounds = [n * i // k for i in range(k + 1)]
        return [(bounds[i], bounds[i + 1]) for i in range(k) if bounds[i + 1] > bounds[i]]

    def run(self, ex, fraction: float = 1.0) -> dict:
        """One pass; `fraction` < 1 processes that leading fraction of every stage (the
        warm-up pass).  Returns seconds per stage."""
        O, ref = self.O, self.kind == "reference"
        x, replica = self.cpi.x, self.cpi.replica
        pulses, samples = x.shape
        secs = {}
        if self.fe is not None:
            ch = max(1, int(round(self.fe.shape[0] * fraction)))
            t0 = time.perf_counter()
            fir = list(ex.map(lambda c: (O.ref_firfilter if ref else O.firfilter)(
                self.fir_taps, self.fe[c:c + 1])[0], range(ch)))
            secs["fir"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            list(ex.map(lambda y: (O.ref_resample_poly(y, UP, DOWN)[0] if ref
                                   else O.resample_poly(y, UP, DOWN)), fir))
            secs["resample_poly"] = time.perf_counter() - t0
        npul = max(1, int(round(pulses * fraction)))
        ncol = max(32, int(round(samples * fraction)))
        comp = np.zeros((pulses, samples), dtype=np.complex64)

        def compress(s):
            p0, p1 = s
            y = (O.ref_pulse_compression(x[p0:p1], replica, -1, True, "hamming")[0] if ref
                 else O.pulse_compression_direct(x[p0:p1], replica, -1, True, "hamming"))
            comp[p0:p1] = y
        t0 = time.perf_counter()
        list(ex.map(compress, self._slices(npul)))
        secs["pulse_compression"] = time.perf_counter() - t0
        power = np.empty((pulses, ncol), dtype=np.float32)

        def doppler(s):
            c0, c1 = s
            rd = (O.ref_pulse_doppler(comp[:, c0:c1], -1, "hamming")[0] if ref
                  else O.pulse_doppler_direct(comp[:, c0:c1], -1, "hamming"))
            power[:, c0:c1] = (rd.real ** 2 + rd.imag ** 2).astype(np.float32)
        t0 = time.perf_counter()
        list(ex.map(doppler, self._slices(ncol)))
        secs["pulse_doppler"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        _, det = (O.ref_ca_cfar if ref else O.ca_cfar_compat)(power, (2, 2), (8, 8), 1e-6)
        secs["ca_cfar"] = time.perf_counter() - t0
        self.detections = int(det.sum())
        return secs


def reference_cpu_baseline(steps: int, warmup: int, budget_s: float = 90.0,
                           one_core_c1: bool = True) -> dict:
    """Time the reference's CPU path on the whole bench workload (CpuChain), all host
    threads.  One warm-up pass over 1/64 of every stage when `warmup` > 0, then full steps:
    at least one, at most `steps`, and no new step once `budget_s` seconds of timed steps
    have passed -- the steps actually run are reported.  Also times one 128 x 4096 CPI
    (20 targets, 256-sample chirp, no front end) on ONE thread."""
    import concurrent.futures as cf
    from zkx_dev_b200 import synth

    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    chain = CpuChain(cores, seed=synth.seed_for(2, 999))
    step_s, stages = [], {}
    with cf.ThreadPoolExecutor(max_workers=cores) as ex:
        warm = 0
        if warmup > 0:
            chain.run(ex, fraction=1.0 / 64)
            warm = 1
        while len(step_s) < max(1, steps):
            t0 = time.perf_counter()
            secs = chain.run(ex)
            step_s.append(time.perf_counter() - t0)
            for k, v in secs.items():
                stages.setdefault(k, []).append(v)
            if sum(step_s) >= budget_s:
                break
    total = sum(step_s)
    res = {"value": len(step_s) / total, "unit": UNIT, "cores": cores, "kind": chain.kind,
           "steps_run": len(step_s), "warmup_run": warm, "seconds_per_step": total / len(step_s),
           "stage_seconds": {k: round(statistics.median(v), 4) for k, v in stages.items()},
           "detections": chain.detections,
           "sample": (f"whole workload every step, {cores} threads: firfilter + resample_poly on "
                      f"all {CH}x{NS} samples, pulse_compression of all {P} pulses, pulse_doppler "
                      f"of all {NR} columns, ca_cfar of the whole {P}x{NR} plane; "
                      f"{len(step_s)} timed step(s)" + (", 1 warm-up pass on 1/64 of each stage"
                                                        if warm else ""))}
    if one_core_c1:
        c1 = CpuChain(1, pulses=128, samples=4096, chirp=256, targets=20, channels=0,
                      seed=synth.seed_for(1))
        with cf.ThreadPoolExecutor(max_workers=1) as ex1:
            t0 = time.perf_counter()
            secs = c1.run(ex1)
            t = time.perf_counter() - t0
        res["c1_one_core"] = {"workload": "128x4096 CPI, 20 targets, chirp 256 (no front end)",
                              "cores": 1, "seconds_per_cpi": round(t, 4),
                              "cpis_per_s": round(1.0 / t, 4),
                              "stage_seconds": {k: round(v, 4) for k, v in secs.items()}}
    return res


def profile_shape(shape: str, precision: str = "fp32") -> None:
    """One warm-up and one run of the chain with the by-shape kernel defaults on a P x N CPI
    generated on the device (the profiling target for transform lengths the bench workload
    does not use)."""
    import torch
    import zkx_dev_b200 as z
    from zkx_dev_b200 import synth
    P_, N_ = (int(v) for v in shape.lower().split("x"))
    L_ = max(1, N_ // 16)
    torch.cuda.set_device(0)
    x = synth.device_cpi(P_, N_, synth.draw_targets(P_, N_, 64, L_, synth.seed_for(5, 7)), L_, synth.seed_for(5, 8))
    chain = z.RangeDopplerChain(z.ChainConfig(P_, N_, L_, precision=precision),
                                torch.as_tensor(synth.lfm_chirp(L_).astype(np.complex64), device="cuda"))
    out = chain.allocate_outputs(keep_rd=False)
    for _ in range(2):
        chain(x, out)
    torch.cuda.synchronize()
    chain.close()


# ------------------------------------------------------------------------ main

def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--lanes", type=int, default=1,
                    help="steps in flight, each on its own front-end and chain streams and buffers "
                         "(2 measured slower over 1000 steps: 0.331 against 0.314 ms per step, the "
                         "other step's traffic evicting the compressed cube Doppler reads from L2)")
    ap.add_argument("--equal-priority", action="store_true",
                    help="run the chain's and the front end's streams at the same scheduling priority "
                         "(default: the chain's highest, the front end's lowest; 0.3134 against 0.3146 ms "
                         "per step over 1000 steps)")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the mixed-stream serving measurement")
    ap.add_argument("--serving-only", action="store_true",
                    help="print only the serving measurements as JSON (run in a fresh process by "
                         "the default invocation)")
    ap.add_argument("--profile", action="store_true",
                    help="one input set, one warm-up and one step of every stage, no timing "
                         "(the command profiled under ncu)")
    ap.add_argument("--shape", default=None,
                    help="with --profile: PxN runs the chain (compression, Doppler, CFAR) on one device-"
                         "generated P x N CPI (chirp N/16, 64 targets) instead of the bench workload, "
                         "one warm-up and one run (the command profiled for other transform lengths)")
    ap.add_argument("--mixed", action="store_true",
                    help="with --profile: the mixed-size batch (256 requests) as per-shape stacked batches "
                         "and as one work list, inside a profiler range (ncu --profile-from-start off)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "tc_f16", "tc_bf16"],
                    help="with --profile --shape: the range-compression arithmetic of the profiled chain")
    args = ap.parse_args()
    args.warmup = 1 if args.profile else max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.profile and args.shape:
        profile_shape(args.shape, args.precision)
        print("profile pass done")
        return
    if args.profile and args.mixed:
        profile_mixed()
        print("profile pass done")
        return
    if args.serving_only:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        serving = run_serving(dev)
        serving["sweep"] = run_serving_sweep(dev)
        print(json.dumps(serving))
        return
    config = {"workload": WORKLOAD, "pulses": P, "range": NR, "chirp": L, "targets": N_TARGETS,
              "front_end": f"{CH}x{NS} fir{FIR_TAPS} resample {UP}/{DOWN}",
              "cfar": "guard 2x2 train 8x8 pfa 1e-6", "parallelism": f"replicas{world}",
              "l2": "inputs larger than L2, three rotating input sets"}

    if args.impl == "reference":
        if rank != 0:
            return
        base = reference_cpu_baseline(args.steps, args.warmup)
        line = {"metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": base["steps_run"], "warmup": base["warmup_run"],
                "steps_requested": args.steps, "warmup_requested": args.warmup,
                "ms_per_step": 1e3 * base["seconds_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded CN(0,1) + LFM targets)", "config": config,
                "impl": "reference",
                "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "stage_seconds": base["stage_seconds"], "detections": base["detections"],
                "c1_one_core": base["c1_one_core"]}
        print(json.dumps(line))
        return

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    res = run_ours(args, rank, world, dist)
    if res is None:
        print("profile pass done")
        return
    if rank == 0:
        line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded CN(0,1) + LFM targets)", "config": config,
                "e2e": res["e2e"], "roofline": res["roofline"], "gpu_launches": res["gpu_launches"],
                "clocks": res["clocks"], "stages_ms": res["stages_ms"], "stages_gbs": res["stages_gbs"],
                "chain_gbs": res["chain_gbs"], "latency_ms": res["latency_ms"],
                "rel_err_vs_fp64": res["rel_err_vs_fp64"], "tuning": res["tuning"]}
        if world == 1 and not args.no_serving:
            import torch
            # the serving loop in a process of its own: its host threads and allocations start
            # from a clean process rather than after the step benchmark's
            r = subprocess.run([sys.executable, os.path.abspath(__file__), "--serving-only"],
                               capture_output=True, text=True, timeout=900)
            try:
                line["serving"] = json.loads(r.stdout.strip().splitlines()[-1])
            except (IndexError, ValueError):
                line["serving"] = {"error": (r.stderr or "no output").strip().splitlines()[-1][:300]}
            line["precision"] = run_precision(torch.device("cuda", 0))
        if world == 1 and not args.no_cpu_baseline:
            base = reference_cpu_baseline(1, 0)
            line["cpu_baseline"] = {k: base[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                         "stage_seconds", "c1_one_core")}
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
