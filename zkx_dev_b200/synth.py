"""Seeded synthetic radar inputs (host, numpy).

A coherent processing interval (CPI) is [pulses, range] complex64: i.i.d. CN(0, 1)
noise plus point targets, each a delayed LFM chirp with a Doppler phase ramp across
pulses.  Generated in FP64 and rounded once to complex64, so the GPU path, the
reference's CPU functions and the FP64 oracle all read the same buffer.  The chirp
is the normalised form of the reference's Task1 waveform
(ZKX/Task1/pipeline/src/steps/step1/step1.cu:27-37): s[n] = exp(i pi (B/L) (n - L/2)^2).

Seeds follow 20261203 + 1000 * config + cpi_index.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

BASE_SEED = 20261203


def seed_for(config: int, cpi_index: int = 0) -> int:
    return BASE_SEED + 1000 * config + cpi_index


def lfm_chirp(length: int, bandwidth: float = 0.5) -> np.ndarray:
    n = np.arange(length, dtype=np.float64)
    return np.exp(1j * np.pi * (bandwidth / length) * (n - length / 2.0) ** 2)


@dataclass
class Target:
    delay: int
    doppler_bin: int
    snr_db: float
    phase: float


@dataclass
class Cpi:
    x: np.ndarray              # [pulses, range] complex64
    replica: np.ndarray        # [L] complex64 (unwindowed chirp)
    targets: List[Target] = field(default_factory=list)


def make_cpi(pulses: int, samples: int, n_targets: int, chirp_length: int, seed: int,
             snr_db: Tuple[float, float] = (10.0, 30.0), low_snr_fraction: float = 0.0,
             low_snr_db: Tuple[float, float] = (0.0, 3.0), bandwidth: float = 0.5) -> Cpi:
    rng = np.random.default_rng(seed)
    s = lfm_chirp(chirp_length, bandwidth)
    x = (rng.standard_normal((pulses, samples)) + 1j * rng.standard_normal((pulses, samples)))
    x *= np.sqrt(0.5)
    p = np.arange(pulses, dtype=np.float64)
    targets = []
    n_low = int(round(low_snr_fraction * n_targets))
    for k in range(n_targets):
        delay = int(rng.integers(0, max(1, samples - chirp_length + 1)))
        dop = int(rng.integers(0, pulses))
        lo, hi = low_snr_db if k < n_low else snr_db
        snr = float(rng.uniform(lo, hi))
        phase = float(rng.uniform(0.0, 2.0 * np.pi))
        amp = 10.0 ** (snr / 20.0)
        ramp = np.exp(1j * (2.0 * np.pi * dop * p / pulses + phase))
        seg = min(chirp_length, samples - delay)
        x[:, delay:delay + seg] += amp * np.outer(ramp, s[:seg])
        targets.append(Target(delay, dop, snr, phase))
    return Cpi(x.astype(np.complex64), s.astype(np.complex64), targets)


def make_front_end(channels: int, samples: int, seed: int, tones: int = 4) -> np.ndarray:
    """[channels, samples] float32: unit-variance noise plus a few seeded tones."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((channels, samples))
    n = np.arange(samples, dtype=np.float64)
    for c in range(channels):
        for _ in range(tones):
            f = rng.uniform(0.01, 0.45)
            a = rng.uniform(0.5, 3.0)
            x[c] += a * np.cos(2.0 * np.pi * f * n + rng.uniform(0, 2 * np.pi))
    return x.astype(np.float32)


def firwin_kaiser(numtaps: int, cutoff: float, beta: float) -> np.ndarray:
    """Windowed-sinc lowpass (fs = 2 convention, unity DC gain) with a Kaiser(beta)
    window: the front end's 127-tap Kaiser(8) filter.  FP64."""
    from numpy import i0
    alpha = 0.5 * (numtaps - 1)
    m = np.arange(numtaps, dtype=np.float64) - alpha
    h = cutoff * np.sinc(cutoff * m)
    w = i0(beta * np.sqrt(np.clip(1.0 - (m / alpha) ** 2, 0.0, None))) / i0(beta)
    h = h * w
    return h / h.sum()


# ------------------------------------------------------------ device generation

def draw_targets(pulses: int, samples: int, n_targets: int, chirp_length: int, seed: int,
                 snr_db: Tuple[float, float] = (10.0, 30.0)) -> List[Target]:
    """Seeded targets of the CPI model (delay, Doppler bin, SNR, phase) for device_cpi."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_targets):
        delay = int(rng.integers(0, max(1, samples - chirp_length + 1)))
        dop = int(rng.integers(0, pulses))
        snr = float(rng.uniform(*snr_db))
        out.append(Target(delay, dop, snr, float(rng.uniform(0.0, 2.0 * np.pi))))
    return out


def device_cpi(pulses: int, samples: int, targets: List[Target], chirp_length: int, seed: int,
               noise_power: float = 1.0, bandwidth: float = 0.5, out=None, stream=None):
    """The CPI model generated on the current CUDA device (zkx_synth_cpi_c64): CN(0,
    noise_power) noise that is a pure function of (seed, element) plus the targets, each
    amplitude 10^(snr/20) times the chirp of lfm_chirp(chirp_length, bandwidth).  Returns a
    complex64 CUDA tensor [pulses, samples]; nothing crosses PCIe but the target table."""
    import torch
    from . import _lib as L
    if len(targets) > 64:
        raise ValueError("at most 64 targets")
    table = (L.SynthTarget * max(1, len(targets)))()
    for i, t in enumerate(targets):
        table[i] = L.SynthTarget(t.delay, t.doppler_bin, 10.0 ** (t.snr_db / 20.0), t.phase)
    if out is None:
        out = torch.empty((pulses, samples), dtype=torch.complex64, device="cuda")
    L.check(L.lib().zkx_synth_cpi_c64(pulses, samples, chirp_length, bandwidth, table, len(targets),
                                      seed & 0xFFFFFFFFFFFFFFFF, noise_power, out.data_ptr(),
                                      L.stream_handle(stream)))
    return out


def device_lfm(length: int, sample_rate: float, bandwidth: float):
    """Task1 LFM waveform on the device (zkx_lfm_waveform_c64), complex64 [length]."""
    import torch
    from . import _lib as L
    out = torch.empty(length, dtype=torch.complex64, device="cuda")
    L.check(L.lib().zkx_lfm_waveform_c64(length, sample_rate, bandwidth, out.data_ptr(), L.stream_handle()))
    return out


def device_task1_echo(waveform, pulses: int, samples: int, delay: int, doppler_hz: float, seed: int,
                      prf: float, sample_rate: float, amplitude: float, noise_std: float):
    """Task1 step-1 echo on the device (zkx_task1_echo_c64): (noiseless, noise, echo),
    complex64 CUDA tensors [pulses, samples]."""
    import torch
    from . import _lib as L
    outs = [torch.empty((pulses, samples), dtype=torch.complex64, device="cuda") for _ in range(3)]
    L.check(L.lib().zkx_task1_echo_c64(waveform.data_ptr(), waveform.numel(), pulses, samples, delay,
                                       doppler_hz, seed & 0xFFFFFFFF, prf, sample_rate, amplitude, noise_std,
                                       outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(),
                                       L.stream_handle()))
    return tuple(outs)
