"""Front-end filters on the B200: firfilter, upfirdn, resample_poly, firfilter2, hilbert.

Mirrors the reference's operator interface (cuSignal 23.08 ``filtering/filtering.py:109``
``firfilter(b, x, axis=-1, zi=None)``, ``filtering/resample.py:304,448`` ``resample_poly``
and ``upfirdn``, as re-implemented in ``ZKX/cusignal_cpp/include/cusignal/operators/
filtering/filtering_typed.h:552-770``).  Inputs are float32 CUDA tensors; the kernels
filter along the last axis, other axes are moved there (a device copy) and back.
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional

import numpy as np
import torch

from . import _lib as L


def _real_input(x: torch.Tensor, name: str) -> torch.Tensor:
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if x.dtype != torch.float32:
        raise TypeError(f"{name} must be float32 (got {x.dtype})")
    return x


def _to_last(x: torch.Tensor, axis: int):
    nd = x.ndim
    if nd == 0:
        raise ValueError("input must have at least one dimension")
    ax = axis + nd if axis < 0 else axis
    if ax < 0 or ax >= nd:
        raise ValueError("axis out of range")
    moved = x.movedim(ax, -1).contiguous() if ax != nd - 1 else x.contiguous()
    return moved, ax


def _from_last(y: torch.Tensor, ax: int, nd: int) -> torch.Tensor:
    return y.movedim(-1, ax).contiguous() if ax != nd - 1 else y


_FIR_METHODS = {"auto": L.FIR_AUTO, "direct": L.FIR_DIRECT, "fft": L.FIR_FFT}


def firfilter(b: torch.Tensor, x: torch.Tensor, axis: int = -1,
              zi: Optional[torch.Tensor] = None, method: str = "auto"):
    """Causal FIR y = b * x along ``axis`` with the output length of x; with ``zi``
    returns (y, zf).  ``method``: "direct" sums, "fft" overlap-save convolution (two lines
    per complex transform, up to 4096 taps), or "auto" (by tap count)."""
    if method not in _FIR_METHODS:
        raise ValueError("firfilter method")
    b = _real_input(b, "b").contiguous()
    x = _real_input(x, "x")
    if b.ndim != 1 or b.numel() < 1:
        raise ValueError("firfilter coefficients")
    xm, ax = _to_last(x, axis)
    n = xm.shape[-1]
    lines = xm.numel() // n if n else 0
    y = torch.empty_like(xm)
    zf = None
    zim = None
    if zi is not None:
        zi = _real_input(zi, "zi")
        zim, _ = _to_last(zi, axis)
        if zim.shape[-1] != b.numel() - 1 or zim.numel() != lines * (b.numel() - 1):
            raise ValueError("firfilter zi broadcast shape")
        zf = torch.empty_like(zim)
    L.check(L.lib().zkx_fir_ex_f32(b.data_ptr(), b.numel(), xm.data_ptr(), lines, n, L.ptr(zim),
                                   y.data_ptr(), L.ptr(zf), _FIR_METHODS[method], L.stream_handle()))
    y = _from_last(y, ax, x.ndim)
    if zi is None:
        return y
    return y, _from_last(zf, ax, x.ndim)


def upfirdn_length(n: int, nh: int, up: int, down: int) -> int:
    return int(L.lib().zkx_upfirdn_length(n, nh, up, down))


def upfirdn(h: torch.Tensor, x: torch.Tensor, up: int = 1, down: int = 1, axis: int = -1):
    """Upsample by ``up``, FIR filter with ``h``, downsample by ``down`` (causal, zero
    extended); output length floor(((n-1)*up + len(h) - 1) / down) + 1."""
    h = _real_input(h, "h").contiguous()
    x = _real_input(x, "x")
    if h.ndim != 1 or h.numel() < 1:
        raise ValueError("upfirdn coefficients")
    if x.ndim > 2:
        raise ValueError("upfirdn rank")
    if int(up) < 1 or int(down) < 1:
        raise ValueError("upfirdn factors")
    xm, ax = _to_last(x, axis)
    n = xm.shape[-1]
    lines = xm.numel() // n if n else (xm.shape[0] if xm.ndim == 2 else 1)
    nout = upfirdn_length(n, h.numel(), up, down)
    y = torch.empty(xm.shape[:-1] + (max(nout, 0),), dtype=torch.float32, device=x.device)
    L.check(L.lib().zkx_upfirdn_f32(h.data_ptr(), h.numel(), xm.data_ptr(), lines, n, int(up),
                                    int(down), y.data_ptr(), L.stream_handle()))
    return _from_last(y, ax, x.ndim)


def resample_layout(n: int, up: int, down: int, ncoeffs: Optional[int] = None) -> L.ResampleLayout:
    lay = L.ResampleLayout()
    L.check(L.lib().zkx_resample_poly_layout(n, int(up), int(down), int(ncoeffs is not None),
                                             ncoeffs or 0, ctypes.byref(lay)))
    return lay


def resample_poly_taps(n: int, up: int, down: int, beta: float = 5.0) -> np.ndarray:
    """The default Kaiser(beta) design in FP64 (taps sum to the reduced ``up``)."""
    lay = resample_layout(n, up, down)
    if lay.identity:
        return np.ones(1)
    taps = np.zeros(lay.coefficient_count, dtype=np.float64)
    L.check(L.lib().zkx_resample_poly_design(ctypes.byref(lay), float(beta),
                                             taps.ctypes.data))
    return taps


def resample_poly(x: torch.Tensor, up: int, down: int, axis: int = 0, window=("kaiser", 5.0),
                  taps: Optional[torch.Tensor] = None):
    """Rational resampling by up/down with a zero-phase polyphase FIR.

    ``window=("kaiser", beta)`` designs the reference's default filter (in FP64 on the
    host, rounded to FP32 taps); an array ``window`` is taken as custom filter
    coefficients (scaled by ``up`` as the reference does).  ``taps`` may pass already
    designed FP32 device taps to skip the design and upload.  The output is float32;
    the reference stores the default design's result as FP64 after computing it in
    FP32, which ``.double()`` reproduces.
    """
    x = _real_input(x, "x")
    if x.ndim > 2:
        raise ValueError("resample_poly nonidentity rank")
    custom = None
    if taps is None and not (isinstance(window, tuple) and len(window) == 2 and window[0] == "kaiser"):
        custom = torch.as_tensor(window, dtype=torch.float32, device=x.device).reshape(-1)
    xm, ax = _to_last(x, axis)
    n = xm.shape[-1]
    lines = xm.numel() // n if n else 1
    lay = resample_layout(n, up, down, None if custom is None and taps is None
                          else (custom.numel() if custom is not None else taps.numel()))
    if lay.identity:
        return x.clone()
    if taps is None:
        if custom is None:
            design = resample_poly_taps(n, up, down, float(window[1]))
            taps = torch.as_tensor(design.astype(np.float32), device=x.device)
        else:
            g = math.gcd(int(up), int(down))
            taps = (custom * float(up // g)).contiguous()
    y = torch.empty(xm.shape[:-1] + (lay.output_samples,), dtype=torch.float32, device=x.device)
    L.check(L.lib().zkx_resample_poly_f32(xm.data_ptr(), lines, n, ctypes.byref(lay),
                                          taps.data_ptr(), y.data_ptr(), L.stream_handle()))
    return _from_last(y, ax, x.ndim)


_PADTYPES = {"odd": L.PAD_ODD, "even": L.PAD_EVEN, "constant": L.PAD_CONSTANT, None: L.PAD_NONE,
             "none": L.PAD_NONE}


def firfilter2(b: torch.Tensor, x: torch.Tensor, axis: int = -1, padtype: Optional[str] = "odd",
               padlen: Optional[int] = None, method: str = "pad", irlen: Optional[int] = None,
               pad_rounding: int = 0, evaluation: str = "auto") -> torch.Tensor:
    """Zero-phase FIR along ``axis`` (cuSignal ``firfilter2(b, x, axis=-1, padtype='odd',
    padlen=None, method='pad', irlen=None)``; filtering_typed.cpp:1226-1302, 1631-1730):
    reflection padding by ``padlen`` samples (default 3 * len(b)), forward and backward FIR
    with steady-state initial conditions, crop.  ``irlen`` is ignored by the pad method, as
    in the reference; ``method='gust'`` is not supported there either.  ``pad_rounding``
    (``L.PAD_ROUND_*``) rounds odd-reflected pad values as a half / integer input would.
    ``evaluation``: "direct" (forward and backward passes), "fft" (one overlap-save
    convolution with the taps' autocorrelation; needs padlen >= len(b)) or "auto"."""
    if evaluation not in _FIR_METHODS:
        raise ValueError("firfilter2 evaluation")
    if method == "gust":
        raise ValueError("firfilter2 gust is not supported by cuSignal 23.08.00")
    if method != "pad":
        raise ValueError("firfilter2 method")
    if padtype not in _PADTYPES:
        raise ValueError("firfilter2 padtype")
    b = _real_input(b, "b").contiguous()
    x = _real_input(x, "x")
    if b.ndim != 1 or b.numel() < 1:
        raise ValueError("firfilter2 coefficients")
    xm, ax = _to_last(x, axis)
    n = xm.shape[-1]
    lines = xm.numel() // n if n else 0
    y = torch.empty_like(xm)
    L.check(L.lib().zkx_firfilter2_ex_f32(b.data_ptr(), b.numel(), xm.data_ptr(), lines, n, _PADTYPES[padtype],
                                          int(padlen is not None), int(padlen or 0), int(pad_rounding),
                                          y.data_ptr(), _FIR_METHODS[evaluation], L.stream_handle()))
    return _from_last(y, ax, x.ndim)


def hilbert(x: torch.Tensor, N: Optional[int] = None, axis: int = -1) -> torch.Tensor:
    """Analytic signal along ``axis`` (cuSignal ``hilbert(x, N=None, axis=-1)``;
    filtering_typed.cpp:500-562, 1819-1872): x zero-padded or truncated to N, DFT, bins
    1..ceil(N/2)-1 doubled, the upper half zeroed, inverse DFT.  complex64 result with N
    samples along ``axis``."""
    x = _real_input(x, "x")
    xm, ax = _to_last(x, axis)
    n = xm.shape[-1]
    nfft = n if N is None else int(N)
    if nfft <= 0:
        raise ValueError("hilbert N must be positive")
    lines = int(np.prod(xm.shape[:-1])) if xm.ndim > 1 else 1
    y = torch.empty(xm.shape[:-1] + (nfft,), dtype=torch.complex64, device=x.device)
    L.check(L.lib().zkx_hilbert_f32(xm.data_ptr(), lines, n, nfft, y.data_ptr(), L.stream_handle()))
    return _from_last(y, ax, x.ndim)
