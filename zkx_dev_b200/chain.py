"""The range-Doppler chain as one plan: pulse_compression -> pulse_doppler (+|.|^2)
-> 2-D CA-CFAR, the path of the reference's Task1 steps 2-4
(ZKX/Task1/pipeline/src/steps/step{2,3,4}/step*.cu).

A plan keeps the replica spectrum and the Doppler window resident on the device;
executing it launches three kernels on the current stream.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Dict, Optional, Sequence

import torch

from . import _lib as L
from .radartools import _window, _complex_input


@dataclass
class ChainConfig:
    num_pulses: int
    samples_per_pulse: int
    replica_length: int
    range_nfft: int = -1
    doppler_nfft: int = -1
    normalize: bool = True
    range_window: object = "hamming"
    doppler_window: object = "hamming"
    guard_cells: Sequence[int] = (2, 2)
    reference_cells: Sequence[int] = (8, 8)
    pfa: float = 1e-6
    cfar_mode: str = "accurate"
    precision: str = "fp32"   # range compression: "fp32", "tc_f16" or "tc_bf16"


class RangeDopplerChain:
    """Owns a zkx_rd_plan for one CPI shape and waveform."""

    def __init__(self, cfg: ChainConfig, replica: torch.Tensor):
        replica = _complex_input(replica, 1, "replica")
        if replica.numel() != cfg.replica_length:
            raise ValueError("replica length mismatch")
        self.cfg = cfg
        dev = replica.device
        rk, rw = _window(cfg.range_window, cfg.replica_length, dev)
        dk, dw = _window(cfg.doppler_window, cfg.num_pulses, dev)
        d = L.RdDesc()
        d.num_pulses = cfg.num_pulses
        d.samples_per_pulse = cfg.samples_per_pulse
        d.range_nfft = cfg.range_nfft
        d.doppler_nfft = cfg.doppler_nfft
        d.replica_length = cfg.replica_length
        d.normalize = int(cfg.normalize)
        d.range_window = rk
        d.doppler_window = dk
        d.guard_cells[0], d.guard_cells[1] = cfg.guard_cells
        d.reference_cells[0], d.reference_cells[1] = cfg.reference_cells
        d.pfa = cfg.pfa
        d.cfar_mode = {"accurate": L.CFAR_ACCURATE, "compat": L.CFAR_COMPAT}[cfg.cfar_mode]
        d.precision = {"fp32": L.PRECISION_FP32, "tc_f16": L.PRECISION_TC_F16,
                       "tc_bf16": L.PRECISION_TC_BF16}[cfg.precision]
        self._keep = (replica, rw, dw)
        h = ctypes.c_void_p()
        L.check(L.lib().zkx_rd_plan_create(ctypes.byref(d), replica.data_ptr(), L.ptr(rw),
                                           L.ptr(dw), L.stream_handle(), ctypes.byref(h)))
        self._plan = h
        nr, nd = ctypes.c_int(), ctypes.c_int()
        L.check(L.lib().zkx_rd_plan_shape(h, ctypes.byref(nr), ctypes.byref(nd)))
        self.range_bins, self.doppler_bins = nr.value, nd.value
        self.device = dev

    def allocate_outputs(self, keep_compressed: bool = True, keep_rd: bool = True,
                         batch: Optional[int] = None) -> Dict[str, Optional[torch.Tensor]]:
        P, nr, nd = self.cfg.num_pulses, self.range_bins, self.doppler_bins
        dev = self.device
        lead = () if batch is None else (batch,)
        return {
            "compressed": torch.empty(lead + (P, nr), dtype=torch.complex64, device=dev) if keep_compressed else None,
            "rd": torch.empty(lead + (nd, nr), dtype=torch.complex64, device=dev) if keep_rd else None,
            "power": torch.empty(lead + (nd, nr), dtype=torch.float32, device=dev),
            "threshold": torch.empty(lead + (nd, nr), dtype=torch.float32, device=dev),
            "detections": torch.empty(lead + (nd, nr), dtype=torch.uint8, device=dev),
        }

    def run(self, x: torch.Tensor, out: Optional[Dict[str, Optional[torch.Tensor]]] = None):
        x = _complex_input(x, 2, "x")
        if tuple(x.shape) != (self.cfg.num_pulses, self.cfg.samples_per_pulse):
            raise ValueError("CPI shape does not match the plan")
        if out is None:
            out = self.allocate_outputs()
        L.check(L.lib().zkx_rd_execute(self._plan, x.data_ptr(), L.ptr(out["compressed"]),
                                       L.ptr(out["rd"]), L.ptr(out["power"]),
                                       out["threshold"].data_ptr(), out["detections"].data_ptr(),
                                       L.stream_handle()))
        return out

    __call__ = run

    def run_batch(self, x: torch.Tensor, out: Optional[Dict[str, Optional[torch.Tensor]]] = None):
        """The chain on a stack of CPIs x [B, P, N] with one launch per stage."""
        if not isinstance(x, torch.Tensor) or not x.is_cuda or x.dtype != torch.complex64 or x.ndim != 3:
            raise TypeError("x must be a complex64 CUDA tensor [B, P, N]")
        x = x.contiguous()
        if tuple(x.shape[1:]) != (self.cfg.num_pulses, self.cfg.samples_per_pulse):
            raise ValueError("CPI shape does not match the plan")
        B = x.shape[0]
        if out is None:
            out = self.allocate_outputs(batch=B)
        L.check(L.lib().zkx_rd_execute_batch(self._plan, x.data_ptr(), B, L.ptr(out["compressed"]),
                                             L.ptr(out["rd"]), L.ptr(out["power"]),
                                             out["threshold"].data_ptr(), out["detections"].data_ptr(),
                                             L.stream_handle()))
        return out

    def capture(self, x: torch.Tensor, out: Dict[str, Optional[torch.Tensor]]) -> "ChainGraph":
        """A CUDA graph replaying run_batch(x, out) (fixed tensors) with one launch."""
        x = x.contiguous()
        B = x.shape[0] if x.ndim == 3 else 1
        g = ctypes.c_void_p()
        L.check(L.lib().zkx_rd_graph_create(self._plan, x.data_ptr(), B, L.ptr(out["compressed"]),
                                            L.ptr(out["rd"]), L.ptr(out["power"]),
                                            out["threshold"].data_ptr(), out["detections"].data_ptr(),
                                            ctypes.byref(g)))
        return ChainGraph(g, (x, out, self))

    def autotune(self, x: torch.Tensor) -> Dict[str, int]:
        """Time the kernel candidates of each stage on x ([P, N] or [B, P, N]) and keep the
        fastest for this plan and for later plans of the same shape (zkx_rd_plan_autotune)."""
        x = x.contiguous()
        batch = x.shape[0] if x.ndim == 3 else 1
        t = L.RdTuning()
        L.check(L.lib().zkx_rd_plan_autotune(self._plan, x.data_ptr(), batch, L.stream_handle(),
                                             ctypes.byref(t)))
        return {name: getattr(t, name) for name, _ in L.RdTuning._fields_}

    @property
    def tuning(self) -> Dict[str, int]:
        t = L.RdTuning()
        L.check(L.lib().zkx_rd_plan_get_tuning(self._plan, ctypes.byref(t)))
        return {name: getattr(t, name) for name, _ in L.RdTuning._fields_}

    def close(self) -> None:
        if getattr(self, "_plan", None) is not None and self._plan.value:
            L.lib().zkx_rd_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ChainGraph:
    """An instantiated CUDA graph of the chain; replay with launch()."""

    def __init__(self, handle: ctypes.c_void_p, keep):
        self._g = handle
        self._keep = keep

    def launch(self) -> None:
        L.check(L.lib().zkx_rd_graph_launch(self._g, L.stream_handle()))

    def close(self) -> None:
        if self._g is not None and self._g.value:
            L.lib().zkx_rd_graph_destroy(self._g)
            self._g = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class WorkList:
    """The chain over CPIs of mixed shapes, one launch per stage and resource class
    (zkx_rd_worklist_*; plans whose stages the work-list kernels do not cover run those
    stages on their own kernels).

    ``items`` is a sequence of ``(chain, x, outputs)``: a RangeDopplerChain (its plan gives
    the CPI's shape and parameters), the device input CPI and a dict with device
    ``threshold`` and ``detections`` planes and optionally ``power``.  Each CPI's outputs
    equal ``chain.run(x)``'s bit for bit.  The tensors must stay alive while the list is
    used; ``launch`` runs on the current stream and may be captured in a CUDA graph."""

    def __init__(self, items):
        arr = (L.WorkItem * len(items))()
        keep = []
        for i, (chain, x, out) in enumerate(items):
            P, N = chain.cfg.num_pulses, chain.cfg.samples_per_pulse
            shape = (chain.doppler_bins, chain.range_bins)
            x = _complex_input(x, 2, "x")
            if tuple(x.shape) != (P, N):
                raise ValueError(f"work item {i}: x must be {P} x {N}")
            for key, dtype in (("threshold", torch.float32), ("detections", torch.uint8), ("power", torch.float32)):
                t = out.get(key)
                if t is None:
                    if key != "power":
                        raise ValueError(f"work item {i}: {key} is required")
                    continue
                if tuple(t.shape) != shape or t.dtype != dtype or not t.is_contiguous() or not t.is_cuda:
                    raise ValueError(f"work item {i}: {key} must be a contiguous device {dtype} {shape}")
            arr[i].plan = chain._plan.value
            arr[i].x = x.data_ptr()
            arr[i].threshold = out["threshold"].data_ptr()
            arr[i].detections = out["detections"].data_ptr()
            arr[i].power = out["power"].data_ptr() if out.get("power") is not None else None
            keep.append((chain, x, out))
        h = ctypes.c_void_p()
        L.check(L.lib().zkx_rd_worklist_create(arr, len(items), ctypes.byref(h)))
        self._h = h
        self._keep = keep

    def launch(self) -> None:
        L.check(L.lib().zkx_rd_worklist_launch(self._h, L.stream_handle()))

    def info(self) -> Dict[str, int]:
        launches, groups, scratch = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        L.check(L.lib().zkx_rd_worklist_info(self._h, ctypes.byref(launches), ctypes.byref(groups),
                                             ctypes.byref(scratch)))
        return {"launches": launches.value, "groups": groups.value, "scratch_bytes": scratch.value}

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().zkx_rd_worklist_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
