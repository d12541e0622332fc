"""Radar tools on the B200: pulse_compression, pulse_doppler, cfar_alpha, ca_cfar.

Names, argument meanings and error behaviour follow the reference's operator
interface (cuSignal 23.08 ``cusignal/radartools/radartools.py:21-124,243-470`` as
re-implemented by ``ZKX/cusignal_cpp/include/cusignal/operators/radartools/
radartools_typed.h``): inputs are CUDA tensors (complex64 for signals, float32 for
power), invalid shapes or parameters raise ``ValueError`` before any work is queued,
and every computation runs in libzkx_rd.so on torch's current stream.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence, Tuple, Union

import torch

from . import _lib as L

WindowArg = Union[None, str, Sequence[float], torch.Tensor]


def _window(window: WindowArg, length: int, device) -> Tuple[int, Optional[torch.Tensor]]:
    """Map a window argument to (RadarWindowKind, explicit FP32 device values or None)."""
    if window is None:
        return L.WINDOW_NONE, None
    if isinstance(window, str):
        name = window.lower()
        if name == "hann" or name == "hanning":
            return L.WINDOW_HANN, None
        if name == "hamming":
            return L.WINDOW_HAMMING, None
        raise ValueError(f"unsupported window name {window!r} (use hann, hamming or values)")
    w = torch.as_tensor(window, dtype=torch.float32, device=device).contiguous()
    if w.ndim != 1 or w.numel() != length:
        raise ValueError("explicit radar window size mismatch")
    return L.WINDOW_EXPLICIT_FP32, w


def _complex_input(x: torch.Tensor, ndim: int, name: str) -> torch.Tensor:
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if x.dtype != torch.complex64:
        raise TypeError(f"{name} must be complex64 (got {x.dtype})")
    if x.ndim != ndim:
        raise ValueError(f"{name} must be {ndim}-D")
    return x.contiguous()


def replica_spectrum(template: torch.Tensor, nfft: int, normalize: bool = False,
                     window: WindowArg = None) -> torch.Tensor:
    """conj(FFT(w * template / ||w * template||, nfft)) / nfft, the factor the fused
    range-compression kernel applies per bin (kept resident per waveform).  For nfft
    above 16384 the bins are stored in the library's cluster order (bin k1 + R*k2 at
    k1*16384 + k2, R = nfft / 16384): pass the tensor back unchanged."""
    t = _complex_input(template, 1, "template")
    kind, w = _window(window, t.numel(), t.device)
    out = torch.empty(nfft, dtype=torch.complex64, device=t.device)
    L.check(L.lib().zkx_replica_spectrum_c64(t.data_ptr(), t.numel(), nfft, int(normalize), kind,
                                             L.ptr(w), out.data_ptr(), L.stream_handle()))
    return out


def pulse_compression(x: torch.Tensor, template: torch.Tensor, normalize: bool = False,
                      window: WindowArg = None, nfft: Optional[int] = None,
                      spectrum: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Matched filter per pulse: IFFT(FFT(x, nfft) * conj(FFT(w*template/||.||, nfft))).

    x: complex64 [num_pulses, samples_per_pulse]; template: complex64 [L].  Returns
    complex64 [num_pulses, nfft].  A precomputed ``spectrum`` (from
    :func:`replica_spectrum`) skips the per-call replica transform.
    """
    x = _complex_input(x, 2, "x")
    P, N = x.shape
    nf = N if nfft is None else int(nfft)
    y = torch.empty((P, nf), dtype=torch.complex64, device=x.device)
    if spectrum is not None:
        L.check(L.lib().zkx_pulse_compression_spectrum_c64(
            x.data_ptr(), P, N, nf, spectrum.data_ptr(), y.data_ptr(), L.stream_handle()))
        return y
    t = _complex_input(template, 1, "template")
    kind, w = _window(window, t.numel(), x.device)
    L.check(L.lib().zkx_pulse_compression_c64(
        x.data_ptr(), P, N, t.data_ptr(), t.numel(), nf, int(normalize), kind, L.ptr(w),
        y.data_ptr(), L.stream_handle()))
    return y


def fft(x: torch.Tensor, inverse: bool = False, out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Batched C2C transform of the rows of x (complex64 [rows, n]; n a power of two up to
    65536, or any length up to 32768 by the chirp-z identity, as the reference's FFT
    backend does for such lengths): forward unnormalised, inverse scaled by 1/n
    (FFTInterface::fft_batch_device / ifft_batch_device).  ``out`` may be x itself."""
    x = _complex_input(x, 2, "x")
    rows, n = x.shape
    y = torch.empty_like(x) if out is None else out
    L.check(L.lib().zkx_fft_c2c_c64(x.data_ptr(), rows, n, int(bool(inverse)), y.data_ptr(),
                                    L.stream_handle()))
    return y


_AMBGFUN_CUTS = {"2d": 0, "delay": 1, "doppler": 2}


def ambgfun(x: torch.Tensor, fs: float, prf: float, y: Optional[torch.Tensor] = None,
            cut: str = "2d", cutValue: float = 0.0) -> torch.Tensor:
    """Normalised ambiguity function (cuSignal ``ambgfun(x, fs, prf, y=None, cut='2d',
    cutValue=0)``, radartools.py).  x, y: complex64 CUDA tensors of any shape whose first
    extent is the signal length (the norm runs over the whole tensor).  Returns float32:
    [nx+ny-1, nfreq] for '2d', [nfreq] for 'delay', [nx+ny-1] for 'doppler'.  ``prf`` does
    not enter the result, as in the reference."""
    if cut not in _AMBGFUN_CUTS:
        raise ValueError("cut must be '2d', 'delay' or 'doppler'")
    if not isinstance(x, torch.Tensor) or not x.is_cuda or x.dtype != torch.complex64:
        raise TypeError("x must be a complex64 CUDA tensor")
    x = x.contiguous()
    nx = x.shape[0] if x.ndim else 1
    if y is not None:
        if not y.is_cuda or y.dtype != torch.complex64:
            raise TypeError("y must be a complex64 CUDA tensor")
        y = y.contiguous()
    ny = (y.shape[0] if y.ndim else 1) if y is not None else nx
    if cut != "2d" and (x.ndim > 1 or (y is not None and y.ndim > 1)):
        raise ValueError("ambgfun high-rank input is only defined for cut='2d'")
    count, rows, nfreq = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int()
    code = _AMBGFUN_CUTS[cut]
    L.check(L.lib().zkx_ambgfun_shape(nx, ny, code, ctypes.byref(count), ctypes.byref(rows),
                                      ctypes.byref(nfreq)))
    shape = {0: (rows.value, nfreq.value), 1: (nfreq.value,), 2: (rows.value,)}[code]
    out = torch.empty(shape, dtype=torch.float32, device=x.device)
    L.check(L.lib().zkx_ambgfun_c64(x.data_ptr(), x.numel(), nx, L.ptr(y),
                                    0 if y is None else y.numel(), ny, code, float(fs),
                                    float(cutValue), out.data_ptr(), L.stream_handle()))
    return out


def pulse_doppler(x: torch.Tensor, window: WindowArg = None, nfft: Optional[int] = None,
                  return_power: bool = False):
    """FFT along pulses (axis 0) of window[p] * x[p, n]; returns complex64 [nfft, N]
    (and the float32 power |.|^2 of the same shape when ``return_power``)."""
    x = _complex_input(x, 2, "x")
    P, N = x.shape
    nf = P if nfft is None else int(nfft)
    kind, w = _window(window, P, x.device)
    out = torch.empty((nf, N), dtype=torch.complex64, device=x.device)
    power = torch.empty((nf, N), dtype=torch.float32, device=x.device) if return_power else None
    L.check(L.lib().zkx_pulse_doppler_c64(x.data_ptr(), P, N, nf, kind, L.ptr(w), out.data_ptr(),
                                          L.ptr(power), L.stream_handle()))
    return (out, power) if return_power else out


def cfar_alpha(pfa: float, N: int) -> float:
    """alpha = N * (pfa ** (-1/N) - 1) (radartools.py:243-261)."""
    a = ctypes.c_double()
    L.check(L.lib().zkx_cfar_alpha(float(pfa), int(N), ctypes.byref(a)))
    return a.value


def ca_cfar(array: torch.Tensor, guard_cells, reference_cells, pfa: float = 1e-3,
            mode: str = "accurate") -> Tuple[torch.Tensor, torch.Tensor]:
    """Cell-averaging CFAR on a 1-D or 2-D float32 CUDA tensor.

    Returns (threshold float32, detections bool).  ``mode="accurate"`` sums the
    training ring in FP32 without cancellation and re-decides near-threshold cells in
    FP64; ``mode="compat"`` reproduces the reference's FP32 integral image exactly.
    """
    if not isinstance(array, torch.Tensor) or not array.is_cuda:
        raise TypeError("array must be a CUDA tensor")
    if array.dtype != torch.float32:
        raise TypeError("array must be float32")
    if array.ndim not in (1, 2):
        raise TypeError("Only 1D and 2D arrays are currently supported.")
    x = array.contiguous()
    g = [int(v) for v in (guard_cells if isinstance(guard_cells, (list, tuple)) else [guard_cells])]
    r = [int(v) for v in (reference_cells if isinstance(reference_cells, (list, tuple)) else [reference_cells])]
    if len(g) != x.ndim or len(r) != x.ndim:
        raise ValueError("ca_cfar cell parameter rank mismatch")
    g += [0] * (2 - len(g))
    r += [0] * (2 - len(r))
    rows = x.shape[0]
    cols = x.shape[1] if x.ndim == 2 else 1
    m = {"accurate": L.CFAR_ACCURATE, "compat": L.CFAR_COMPAT}.get(mode)
    if m is None:
        raise ValueError(f"unknown ca_cfar mode {mode!r}")
    thr = torch.empty_like(x)
    det = torch.empty(x.shape, dtype=torch.uint8, device=x.device)
    L.check(L.lib().zkx_ca_cfar_f32(x.data_ptr(), x.ndim, rows, cols, g[0], g[1], r[0], r[1],
                                    float(pfa), m, thr.data_ptr(), det.data_ptr(),
                                    L.stream_handle()))
    return thr, det.view(torch.bool)
