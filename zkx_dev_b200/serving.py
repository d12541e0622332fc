"""Python mirror of the serving loop (zkx_rd_server_*, zkx_rd_submit, zkx_rd_poll in
include/zkx_rd.h): CPIs of mixed shapes are submitted as they arrive and complete
asynchronously; results land in caller-owned buffers (page-locked host or device
tensors)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Dict, Optional, Sequence

import torch

from . import _lib as L

_WINDOWS = {"none": L.WINDOW_NONE, None: L.WINDOW_NONE, "hann": L.WINDOW_HANN,
            "hamming": L.WINDOW_HAMMING}


@dataclass
class ServerConfig:
    normalize: bool = True
    range_window: Optional[str] = "hamming"
    doppler_window: Optional[str] = "hamming"
    guard_cells: Sequence[int] = (2, 2)
    reference_cells: Sequence[int] = (8, 8)
    pfa: float = 1e-6
    cfar_mode: str = "accurate"
    streams: int = 2
    max_inflight: int = 0      # 0: 2 * streams
    max_batch: int = 32
    hbm_fraction: float = 0.8
    budget_bytes: int = 0      # 0: no cap below hbm_fraction of free HBM
    max_pending: int = 0       # 0: unbounded queue; else submits beyond it raise ZkxError 3002


def _check_buffer(t: Optional[torch.Tensor], shape, dtype, name: str, required: bool = False):
    if t is None:
        if required:
            raise ValueError(f"{name} is required")
        return None
    if tuple(t.shape) != tuple(shape) or t.dtype != dtype or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous {dtype} tensor of shape {tuple(shape)}")
    return t


class RdServer:
    """A continuous-batching range-Doppler server on the current CUDA device."""

    def __init__(self, cfg: ServerConfig = ServerConfig()):
        d = L.ServerDesc()
        d.normalize = int(cfg.normalize)
        d.range_window = _WINDOWS[cfg.range_window]
        d.doppler_window = _WINDOWS[cfg.doppler_window]
        d.guard_cells[0], d.guard_cells[1] = cfg.guard_cells
        d.reference_cells[0], d.reference_cells[1] = cfg.reference_cells
        d.pfa = cfg.pfa
        d.cfar_mode = {"accurate": L.CFAR_ACCURATE, "compat": L.CFAR_COMPAT}[cfg.cfar_mode]
        d.streams = cfg.streams
        d.max_inflight = cfg.max_inflight
        d.max_batch = cfg.max_batch
        d.hbm_fraction = cfg.hbm_fraction
        d.budget_bytes = cfg.budget_bytes
        d.max_pending = cfg.max_pending
        h = ctypes.c_void_p()
        L.check(L.lib().zkx_rd_server_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        self._live: Dict[int, tuple] = {}

    def submit(self, x: torch.Tensor, replica: torch.Tensor, waveform_id: int,
               detections: torch.Tensor, threshold: Optional[torch.Tensor] = None,
               power: Optional[torch.Tensor] = None, rd: Optional[torch.Tensor] = None) -> int:
        """Queue one CPI x [P, N] complex64 (host, ideally pinned, or CUDA).  Outputs are
        [P, N]: detections uint8 (required), threshold/power float32, rd complex64."""
        if x.dtype != torch.complex64 or x.ndim != 2 or not x.is_contiguous():
            raise ValueError("x must be a contiguous complex64 [P, N] tensor")
        if not replica.is_cuda or replica.dtype != torch.complex64 or not replica.is_contiguous():
            raise ValueError("replica must be a contiguous complex64 CUDA tensor")
        P, N = x.shape
        _check_buffer(detections, (P, N), torch.uint8, "detections", required=True)
        _check_buffer(threshold, (P, N), torch.float32, "threshold")
        _check_buffer(power, (P, N), torch.float32, "power")
        _check_buffer(rd, (P, N), torch.complex64, "rd")
        r = L.Request()
        r.num_pulses, r.samples_per_pulse = P, N
        r.waveform_id = int(waveform_id)
        r.replica = replica.data_ptr()
        r.replica_length = replica.numel()
        r.x = x.data_ptr()
        r.detections = detections.data_ptr()
        r.threshold = L.ptr(threshold)
        r.power = L.ptr(power)
        r.rd = L.ptr(rd)
        t = ctypes.c_uint64()
        L.check(L.lib().zkx_rd_submit(self._h, ctypes.byref(r), ctypes.byref(t)))
        # keep every buffer alive until the request completes
        self._live[t.value] = (x, replica, detections, threshold, power, rd)
        return t.value

    def poll(self, ticket: int, timeout_ms: int = 0) -> bool:
        """True once the request has completed (its outputs are then in place)."""
        done = ctypes.c_int()
        rc = L.lib().zkx_rd_poll(self._h, ctypes.c_uint64(ticket), int(timeout_ms), ctypes.byref(done))
        if done.value:
            self._live.pop(ticket, None)
        L.check(rc)
        return bool(done.value)

    def wait(self, ticket: int) -> None:
        self.poll(ticket, -1)

    def stats(self) -> Dict[str, float]:
        s = L.ServerStats()
        L.check(L.lib().zkx_rd_server_stats_get(self._h, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in L.ServerStats._fields_}

    def reset_stats(self) -> None:
        L.check(L.lib().zkx_rd_server_stats_reset(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().zkx_rd_server_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
