"""The oracle: test infrastructure, never part of the product path.

Two CPU implementations of the radar range-Doppler chain, loaded through ctypes:

* ``restatement`` -- ``oracle/liboracle.so``, this repository's plain-C restatement of
  the reference's CPU algorithms plus FP64 truth variants (``rd_oracle.c``).
* ``reference`` -- ``oracle/_ref/libzkx_ref.so``, the reference library's own
  ``*_typed_cpu`` functions (ZKX/cusignal_cpp) compiled from the reference checkout by
  ``oracle/Makefile``; absent when it was never built.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import this package.  Arrays are numpy; complex arrays are ``complex64`` in and
``complex128`` out.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_PATH = os.path.join(_HERE, "liboracle.so")
REFERENCE_PATH = os.path.join(_HERE, "_ref", "libzkx_ref.so")

WINDOW = {"none": 0, "hann": 1, "hamming": 2, "explicit_fp32": 3, "explicit_fp64": 4}

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_F = ctypes.c_float


def build_restatement() -> None:
    """Compile ``liboracle.so`` with gcc (the reference is not needed for this)."""
    subprocess.run(["make", "-s", "-C", _HERE, "restatement"], check=True)


def reference_root() -> str:
    """The ZKX_dev checkout the reference builds read: $ZKX_REFERENCE_ROOT when set, else a
    checkout named "reference" beside this repository."""
    env = os.environ.get("ZKX_REFERENCE_ROOT")
    if env:
        return env
    return os.path.normpath(os.path.join(_HERE, "..", "..", "reference"))


def build_reference(ref_root: Optional[str] = None) -> bool:
    """Compile the reference CPU library when the reference checkout is present."""
    ref_root = ref_root or reference_root()
    if not os.path.isdir(os.path.join(ref_root, "ZKX", "cusignal_cpp")):
        return False
    subprocess.run(["make", "-s", "-j8", "-C", _HERE, "ref", f"REF_ROOT={ref_root}"],
                   check=True)
    return True


def build_probes(ref_root: Optional[str] = None) -> bool:
    """Compile the reference's own operator probes against include/ and libzkx_rd.so
    (test infrastructure for the drop-in check) when the reference checkout is present."""
    ref_root = ref_root or reference_root()
    if not os.path.isdir(os.path.join(ref_root, "ZKX", "test_all")):
        return False
    subprocess.run(["make", "-s", "-j8", "-C", _HERE, "probes", f"REF_ROOT={ref_root}"], check=True)
    return True


def build_task1(ref_root: Optional[str] = None) -> bool:
    """Compile the reference's Task1 pipeline and its pipeline benchmark, unchanged, against
    include/ and libzkx_rd.so (the drop-in check for Task1) when the checkout is present."""
    ref_root = ref_root or reference_root()
    if not os.path.isdir(os.path.join(ref_root, "ZKX", "Task1", "pipeline")):
        return False
    subprocess.run(["make", "-s", "-j8", "-C", _HERE, "task1", f"REF_ROOT={ref_root}"], check=True)
    return True


_lib_cache: dict = {}


def restatement() -> ctypes.CDLL:
    if "r" not in _lib_cache:
        if not os.path.exists(RESTATEMENT_PATH):
            build_restatement()
        lib = ctypes.CDLL(RESTATEMENT_PATH)
        lib.or_radar_window_f32.restype = _F
        lib.or_radar_window_f32.argtypes = [_I, _I, _I, _P]
        lib.or_pulse_compression_direct.argtypes = [_P, _I, _I, _P, _I, _I, _I, _I, _P, _P]
        lib.or_pulse_compression_fft64.argtypes = [_P, _I, _I, _P, _I, _I, _I, _P, _P]
        lib.or_pulse_doppler_direct.argtypes = [_P, _I, _I, _I, _I, _P, _P]
        lib.or_pulse_doppler_fft64.argtypes = [_P, _I, _I, _I, _P, _P, _P]
        lib.or_cfar_alpha.argtypes = [_D, _I, _P]
        lib.or_cfar_reference_count_2d.argtypes = [_I, _I, _I, _I]
        lib.or_ca_cfar_compat_f32.argtypes = [_P, _I, _I, _I, _I, _I, _I, _I, _D, _P, _P]
        lib.or_ca_cfar_f64.argtypes = [_P, _I, _I, _I, _I, _I, _I, _D, _P, _P]
        lib.or_ca_cfar_f64_rows.argtypes = [_P, _I, _I, _I, _I, _I, _I, _D, _I, _I, _P, _P]
        lib.or_firfilter.argtypes = [_P, _I, _P, _I, _I, _P, _P, _P]
        lib.or_upfirdn_length.restype = ctypes.c_int64
        lib.or_upfirdn_length.argtypes = [_I, _I, _I, _I]
        lib.or_upfirdn_f32.argtypes = [_P, _I, _P, _I, _I, _I, _I, _P]
        lib.or_resample_poly_layout.argtypes = [_I, _I, _I, _I, _I, _P]
        lib.or_resample_poly_design.argtypes = [_P, _D, _P]
        lib.or_resample_poly_f64.argtypes = [_P, _P, _P, _I, _I, _P]
        lib.or_resample_poly_f32.argtypes = [_P, _P, _P, _I, _I, _P]
        lib.or_ambgfun.argtypes = [_P, _I, _I, _P, _I, _I, _I, _D, _D, _P]
        lib.or_task1_echo.argtypes = [_P, _I, _I, _I, _I, _D, ctypes.c_uint32, _D, _D, _D,
                                      ctypes.c_float, _P, _P]
        lib.or_firfilter2.argtypes = [_P, _I, _P, _I, _I, _I, _I, _I, _I, _P]
        lib.or_hilbert.argtypes = [_P, _I, _I, _I, _P]
        _lib_cache["r"] = lib
    return _lib_cache["r"]


def reference() -> Optional[ctypes.CDLL]:
    """The compiled reference CPU library, or None when it is not built."""
    if "ref" not in _lib_cache:
        if not os.path.exists(REFERENCE_PATH):
            return None
        lib = ctypes.CDLL(REFERENCE_PATH)
        lib.zkx_ref_last_error.restype = ctypes.c_char_p
        lib.zkx_ref_pulse_compression_f32.argtypes = [_P, _I, _I, _P, _I, _I, _I, _I, _P, _P, _P]
        lib.zkx_ref_pulse_doppler_f32.argtypes = [_P, _I, _I, _I, _I, _P, _P, _P]
        lib.zkx_ref_ca_cfar_f32.argtypes = [_P, _I, _I, _I, _I, _I, _I, _I, _D, _P, _P]
        lib.zkx_ref_cfar_alpha_f32.argtypes = [_F, _I, _P]
        lib.zkx_ref_firfilter_f32.argtypes = [_P, _I, _P, _I, _I, _P, _P, _P]
        lib.zkx_ref_upfirdn_f32.argtypes = [_P, _I, _P, _I, _I, _I, _I, _P, _P]
        lib.zkx_ref_resample_poly_f32.argtypes = [_P, _I, _I, _I, _I, _D, _P, _I, _P, _P, _P]
        lib.zkx_ref_firwin_kaiser.argtypes = [_I, _D, _D, _P]
        lib.zkx_ref_ambgfun_f32.argtypes = [_P, _I, _I, _P, _I, _I, _I, _D, _D, _P, _P]
        lib.zkx_ref_firfilter2.argtypes = [_I, _P, _I, _P, _P, _I, _I, _I, _I, _I, _P, _P]
        lib.zkx_ref_hilbert.argtypes = [_I, _P, _P, _I, _I, _I, _I, _P, _P]
        _lib_cache["ref"] = lib
    return _lib_cache["ref"]


class OracleError(ValueError):
    pass


def _check(rc: int, lib=None) -> None:
    if rc != 0:
        msg = ""
        if lib is not None and hasattr(lib, "zkx_ref_last_error"):
            msg = lib.zkx_ref_last_error().decode(errors="replace")
        raise OracleError(f"oracle call failed with code {rc}: {msg}")


def _c64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex64)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


# ----------------------------------------------------------------- windows

def radar_window_f32(kind: str, length: int) -> np.ndarray:
    """FP32 window values as the reference evaluates them (rt.cpp:238-251)."""
    lib = restatement()
    k = WINDOW[kind]
    return np.array([lib.or_radar_window_f32(k, i, length, None) for i in range(length)],
                    dtype=np.float32)


# -------------------------------------------------------- pulse compression

def pulse_compression_direct(x, tmpl, nfft: int = -1, normalize: bool = True,
                             window: str = "none", explicit_window=None) -> np.ndarray:
    x, t = _c64(x), _c64(tmpl)
    P, N = x.shape
    nf = N if nfft == -1 else nfft
    out = np.zeros((P, nf), dtype=np.complex128)
    w = None if explicit_window is None else _f32(explicit_window)
    _check(restatement().or_pulse_compression_direct(
        x.ctypes.data, P, N, t.ctypes.data, t.size, nf, int(normalize), WINDOW[window],
        _ptr(w), out.ctypes.data))
    return out


def pulse_compression_fft64(x, tmpl, nfft: int = -1, normalize: bool = True,
                            window_f32=None) -> np.ndarray:
    x, t = _c64(x), _c64(tmpl)
    P, N = x.shape
    nf = N if nfft == -1 else nfft
    out = np.zeros((P, nf), dtype=np.complex128)
    w = None if window_f32 is None else _f32(window_f32)
    _check(restatement().or_pulse_compression_fft64(
        x.ctypes.data, P, N, t.ctypes.data, t.size, nf, int(normalize), _ptr(w),
        out.ctypes.data))
    return out


def ref_pulse_compression(x, tmpl, nfft: int = -1, normalize: bool = True,
                          window: str = "none", explicit_window=None):
    """The reference's own pulse_compression_typed_cpu<float>; returns (out, is_fp64)."""
    lib = reference()
    if lib is None:
        raise OracleError("reference library not built")
    x, t = _c64(x), _c64(tmpl)
    P, N = x.shape
    nf = N if nfft == -1 else nfft
    out = np.zeros((P, nf), dtype=np.complex128)
    is64 = ctypes.c_int(0)
    w = None if explicit_window is None else _f32(explicit_window)
    _check(lib.zkx_ref_pulse_compression_f32(
        x.ctypes.data, P, N, t.ctypes.data, t.size, nfft, int(normalize), WINDOW[window],
        _ptr(w), out.ctypes.data, ctypes.byref(is64)), lib)
    return out, bool(is64.value)


# ------------------------------------------------------------ pulse doppler

def pulse_doppler_direct(x, nfft: int = -1, window: str = "none",
                         explicit_window=None) -> np.ndarray:
    x = _c64(x)
    P, N = x.shape
    nf = P if nfft == -1 else nfft
    out = np.zeros((nf, N), dtype=np.complex128)
    w = None if explicit_window is None else _f32(explicit_window)
    _check(restatement().or_pulse_doppler_direct(
        x.ctypes.data, P, N, nf, WINDOW[window], _ptr(w), out.ctypes.data))
    return out


def pulse_doppler_fft64(x, nfft: int = -1, window_f32=None):
    """FP64 Doppler of a complex array (any precision in); returns (rd, power)."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    P, N = x.shape
    nf = P if nfft == -1 else nfft
    out = np.zeros((nf, N), dtype=np.complex128)
    power = np.zeros((nf, N), dtype=np.float64)
    w = None if window_f32 is None else _f32(window_f32)
    _check(restatement().or_pulse_doppler_fft64(
        x.ctypes.data, P, N, nf, _ptr(w), out.ctypes.data, power.ctypes.data))
    return out, power


def ref_pulse_doppler(x, nfft: int = -1, window: str = "none", explicit_window=None):
    lib = reference()
    if lib is None:
        raise OracleError("reference library not built")
    x = _c64(x)
    P, N = x.shape
    nf = P if nfft == -1 else nfft
    out = np.zeros((nf, N), dtype=np.complex128)
    is64 = ctypes.c_int(0)
    w = None if explicit_window is None else _f32(explicit_window)
    _check(lib.zkx_ref_pulse_doppler_f32(
        x.ctypes.data, P, N, nfft, WINDOW[window], _ptr(w), out.ctypes.data,
        ctypes.byref(is64)), lib)
    return out, bool(is64.value)


# --------------------------------------------------------------------- CFAR

def cfar_alpha(pfa: float, reference_count: int) -> float:
    a = ctypes.c_double()
    _check(restatement().or_cfar_alpha(pfa, reference_count, ctypes.byref(a)))
    return a.value


def ref_cfar_alpha(pfa: float, reference_count: int) -> float:
    lib = reference()
    a = ctypes.c_double()
    _check(lib.zkx_ref_cfar_alpha_f32(pfa, reference_count, ctypes.byref(a)), lib)
    return a.value


def reference_count_2d(guard, train) -> int:
    return restatement().or_cfar_reference_count_2d(guard[0], guard[1], train[0], train[1])


def ca_cfar_compat(x, guard, train, pfa: float):
    """Bit-exact restatement of the reference FP32 integral-image CA-CFAR."""
    x = _f32(x)
    rank = x.ndim
    rows = x.shape[0]
    cols = x.shape[1] if rank == 2 else 1
    g = list(guard) + [0] * (2 - len(guard))
    r = list(train) + [0] * (2 - len(train))
    thr = np.zeros(x.shape, dtype=np.float32)
    det = np.zeros(x.shape, dtype=np.uint8)
    _check(restatement().or_ca_cfar_compat_f32(
        x.ctypes.data, rank, rows, cols, g[0], g[1], r[0], r[1], pfa,
        thr.ctypes.data, det.ctypes.data))
    return thr, det


def ca_cfar_f64(x, guard, train, pfa: float):
    """FP64 truth CA-CFAR on the given (FP32) input; returns (threshold64, mask)."""
    x = _f32(x)
    rows, cols = x.shape
    thr = np.zeros(x.shape, dtype=np.float64)
    det = np.zeros(x.shape, dtype=np.uint8)
    _check(restatement().or_ca_cfar_f64(
        x.ctypes.data, rows, cols, guard[0], guard[1], train[0], train[1], pfa,
        thr.ctypes.data, det.ctypes.data))
    return thr, det


def ca_cfar_f64_bands(x, guard, train, pfa: float, threads: Optional[int] = None,
                      band_rows: int = 64):
    """The FP64 truth CA-CFAR of ``ca_cfar_f64`` computed separably in row bands on
    several threads (``or_ca_cfar_f64_rows``; ctypes releases the GIL during each call),
    for full planes of 10^7-10^8 cells.  Returns (threshold64, mask)."""
    import concurrent.futures as cf
    x = _f32(x)
    rows, cols = x.shape
    thr = np.zeros(x.shape, dtype=np.float64)
    det = np.zeros(x.shape, dtype=np.uint8)
    lib = restatement()
    if threads is None:
        threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)

    def band(r0: int) -> int:
        r1 = min(rows, r0 + band_rows)
        return lib.or_ca_cfar_f64_rows(x.ctypes.data, rows, cols, guard[0], guard[1], train[0],
                                       train[1], pfa, r0, r1,
                                       thr.ctypes.data + r0 * cols * 8,
                                       det.ctypes.data + r0 * cols)

    with cf.ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        for rc in ex.map(band, range(0, rows, band_rows)):
            _check(rc)
    return thr, det


def ref_ca_cfar(x, guard, train, pfa: float):
    lib = reference()
    x = _f32(x)
    rank = x.ndim
    rows = x.shape[0]
    cols = x.shape[1] if rank == 2 else 1
    g = list(guard) + [0] * (2 - len(guard))
    r = list(train) + [0] * (2 - len(train))
    thr = np.zeros(x.shape, dtype=np.float32)
    det = np.zeros(x.shape, dtype=np.uint8)
    _check(lib.zkx_ref_ca_cfar_f32(x.ctypes.data, rank, rows, cols, g[0], g[1], r[0], r[1],
                                   pfa, thr.ctypes.data, det.ctypes.data), lib)
    return thr, det


# ------------------------------------------------------------------ filters

def firfilter(b, x, zi=None):
    b, x = _f32(b), _f32(x)
    x2 = x.reshape(-1, x.shape[-1])
    rows, n = x2.shape
    y = np.zeros_like(x2)
    zf = None if zi is None else np.zeros((rows, b.size - 1), dtype=np.float32)
    zi2 = None if zi is None else _f32(zi).reshape(rows, b.size - 1)
    _check(restatement().or_firfilter(b.ctypes.data, b.size, x2.ctypes.data, rows, n,
                                      _ptr(zi2), y.ctypes.data, _ptr(zf)))
    y = y.reshape(x.shape)
    return y if zi is None else (y, zf)


def ref_firfilter(b, x, zi=None):
    lib = reference()
    b, x = _f32(b), _f32(x)
    x2 = x.reshape(-1, x.shape[-1])
    rows, n = x2.shape
    y = np.zeros_like(x2)
    zf = None if zi is None else np.zeros((rows, b.size - 1), dtype=np.float32)
    zi2 = None if zi is None else _f32(zi).reshape(rows, b.size - 1)
    _check(lib.zkx_ref_firfilter_f32(b.ctypes.data, b.size, x2.ctypes.data, rows, n,
                                     _ptr(zi2), y.ctypes.data, _ptr(zf)), lib)
    y = y.reshape(x.shape)
    return y if zi is None else (y, zf)


def upfirdn_length(n: int, nh: int, up: int, down: int) -> int:
    return int(restatement().or_upfirdn_length(n, nh, up, down))


def upfirdn(h, x, up: int, down: int) -> np.ndarray:
    h, x = _f32(h), _f32(x)
    x2 = x.reshape(-1, x.shape[-1])
    rows, n = x2.shape
    nout = upfirdn_length(n, h.size, up, down)
    out = np.zeros((rows, max(nout, 0)), dtype=np.float32)
    _check(restatement().or_upfirdn_f32(h.ctypes.data, h.size, x2.ctypes.data, rows, n, up,
                                        down, out.ctypes.data))
    return out.reshape(x.shape[:-1] + (out.shape[-1],))


def ref_upfirdn(h, x, up: int, down: int) -> np.ndarray:
    lib = reference()
    h, x = _f32(h), _f32(x)
    x2 = x.reshape(-1, x.shape[-1])
    rows, n = x2.shape
    nout = upfirdn_length(n, h.size, up, down)
    out = np.zeros((rows, max(nout, 0)), dtype=np.float32)
    ns = ctypes.c_int()
    _check(lib.zkx_ref_upfirdn_f32(h.ctypes.data, h.size, x2.ctypes.data, rows, n, up, down,
                                   out.ctypes.data, ctypes.byref(ns)), lib)
    return out.reshape(x.shape[:-1] + (out.shape[-1],))


class ResampleLayout(ctypes.Structure):
    _fields_ = [("up", _I), ("down", _I), ("identity", _I), ("output_samples", _I),
                ("coefficient_count", _I), ("half_length", _I), ("prefix_zeros", _I),
                ("output_start", _I)]


def resample_poly_layout(n: int, up: int, down: int, ncoeffs: Optional[int] = None):
    lay = ResampleLayout()
    _check(restatement().or_resample_poly_layout(
        n, up, down, int(ncoeffs is not None), ncoeffs or 0, ctypes.byref(lay)))
    return lay


def resample_poly_design(n: int, up: int, down: int, beta: float = 5.0) -> np.ndarray:
    lay = resample_poly_layout(n, up, down)
    taps = np.zeros(lay.coefficient_count, dtype=np.float64)
    _check(restatement().or_resample_poly_design(ctypes.byref(lay), beta, taps.ctypes.data))
    return taps


def resample_poly(x, up: int, down: int, beta: float = 5.0) -> np.ndarray:
    """Default Kaiser design, FP64 accumulation (the reference's default branch)."""
    x = _f32(x)
    x2 = x.reshape(-1, x.shape[-1])
    rows, n = x2.shape
    lay = resample_poly_layout(n, up, down)
    if lay.identity:
        return x.astype(np.float64)
    taps = resample_poly_design(n, up, down, beta)
    out = np.zeros((rows, lay.output_samples), dtype=np.float64)
    _check(restatement().or_resample_poly_f64(taps.ctypes.data, ctypes.byref(lay),
                                              x2.ctypes.data, rows, n, out.ctypes.data))
    return out.reshape(x.shape[:-1] + (lay.output_samples,))


def resample_poly_custom_f32(x, up: int, down: int, taps_f32) -> np.ndarray:
    """Custom taps (already scaled) with FP32 accumulation."""
    x, t = _f32(x), _f32(taps_f32)
    x2 = x.reshape(-1, x.shape[-1])
    rows, n = x2.shape
    lay = resample_poly_layout(n, up, down, t.size)
    out = np.zeros((rows, lay.output_samples), dtype=np.float32)
    _check(restatement().or_resample_poly_f32(t.ctypes.data, ctypes.byref(lay), x2.ctypes.data,
                                              rows, n, out.ctypes.data))
    return out.reshape(x.shape[:-1] + (lay.output_samples,))


def ref_resample_poly(x, up: int, down: int, beta: float = 5.0, coeffs=None):
    lib = reference()
    x = _f32(x)
    x2 = x.reshape(-1, x.shape[-1])
    rows, n = x2.shape
    lay = resample_poly_layout(n, up, down, None if coeffs is None else len(coeffs))
    out = np.zeros((rows, lay.output_samples), dtype=np.float64)
    ns, is64 = ctypes.c_int(), ctypes.c_int()
    c = None if coeffs is None else _f32(coeffs)
    _check(lib.zkx_ref_resample_poly_f32(x2.ctypes.data, rows, n, up, down, beta, _ptr(c),
                                         0 if c is None else c.size, out.ctypes.data,
                                         ctypes.byref(ns), ctypes.byref(is64)), lib)
    return out.reshape(x.shape[:-1] + (lay.output_samples,)), bool(is64.value)


def ref_firwin_kaiser(numtaps: int, cutoff: float, beta: float) -> np.ndarray:
    lib = reference()
    out = np.zeros(numtaps, dtype=np.float64)
    _check(lib.zkx_ref_firwin_kaiser(numtaps, cutoff, beta, out.ctypes.data), lib)
    return out


_CUTS = {"2d": 0, "delay": 1, "doppler": 2}


def ambgfun_shape(nx: int, ny: int, cut: str):
    rows = nx + ny - 1
    nfreq = 1
    while nfreq < rows:
        nfreq <<= 1
    return {"2d": (rows, nfreq), "delay": (nfreq,), "doppler": (rows,)}[cut]


def ambgfun(x, y=None, fs: float = 1.0, cut: str = "2d", cut_value: float = 0.0, nx=None, ny=None):
    """Restatement of ambgfun_typed_cpu (rt.cpp:330-463), values in FP64.  nx / ny: the
    first extents of high-rank inputs (default: the whole arrays)."""
    x = _c64(x).ravel()
    nx = x.size if nx is None else nx
    yy = None if y is None else _c64(y).ravel()
    ny = (nx if yy is None else yy.size) if ny is None else ny
    shape = ambgfun_shape(nx, ny, cut)
    out = np.empty(shape, dtype=np.float64)
    _check(restatement().or_ambgfun(_ptr(x), x.size, nx, _ptr(yy), 0 if yy is None else yy.size, ny,
                                    _CUTS[cut], fs, cut_value, _ptr(out)))
    return out


def ref_ambgfun(x, y=None, fs: float = 1.0, cut: str = "2d", cut_value: float = 0.0, nx=None, ny=None):
    """The reference's own ambgfun_typed_cpu<float>; returns (values as float64, is_fp64)."""
    x = _c64(x).ravel()
    nx = x.size if nx is None else nx
    yy = None if y is None else _c64(y).ravel()
    ny = (nx if yy is None else yy.size) if ny is None else ny
    out = np.empty(ambgfun_shape(nx, ny, cut), dtype=np.float64)
    is64 = ctypes.c_int()
    lib = reference()
    _check(lib.zkx_ref_ambgfun_f32(_ptr(x), x.size, nx, _ptr(yy), 0 if yy is None else yy.size, ny,
                                   _CUTS[cut], fs, cut_value, _ptr(out), ctypes.byref(is64)), lib)
    return out, bool(is64.value)


def task1_echo(waveform, pulses: int, samples: int, delay: int, doppler_hz: float, seed: int,
               prf: float, fs: float, amplitude: float, noise_std: float):
    """Task1 step-1 echo (step1.cu:11-71): (noiseless complex128 [P, N] with FP64 phases,
    noise complex64 [P, N] bit-exact to the reference's hash)."""
    w = _c64(waveform)
    noiseless = np.empty((pulses, samples), dtype=np.complex128)
    noise = np.empty((pulses, samples), dtype=np.complex64)
    _check(restatement().or_task1_echo(_ptr(w), w.size, pulses, samples, delay, doppler_hz, seed, prf, fs,
                                       amplitude, noise_std, _ptr(noiseless), _ptr(noise)))
    return noiseless, noise


# ------------------------------------------------------------ firfilter2 / hilbert

PADTYPE = {"odd": 0, "even": 1, "constant": 2, "none": 3}
# element types of the reference's instantiations, with the odd-pad rounding each implies
_REF_DTYPE = {np.dtype(np.float32): 0, np.dtype(np.float16): 1, np.dtype(np.int32): 2,
              np.dtype(np.int16): 3, np.dtype(np.int8): 4}
PAD_ROUNDING = {np.dtype(np.float32): 0, np.dtype(np.float16): 1, np.dtype(np.int8): 2,
                np.dtype(np.int16): 3, np.dtype(np.int32): 4}


def firfilter2(b, x, padtype: str = "odd", padlen: Optional[int] = None, rounding: int = 0) -> np.ndarray:
    """The C restatement along the last axis of x [lines, n] (float values); double result."""
    b, x = _f32(b), _f32(x)
    x2 = x.reshape(-1, x.shape[-1])
    out = np.zeros(x2.shape, dtype=np.float64)
    _check(restatement().or_firfilter2(b.ctypes.data, b.size, x2.ctypes.data, x2.shape[0], x2.shape[1],
                                       PADTYPE[padtype], int(padlen is not None), padlen or 0, rounding,
                                       out.ctypes.data))
    return out.reshape(x.shape)


def ref_firfilter2(b, x, axis: int = -1, padtype: str = "odd", padlen: Optional[int] = None):
    """The reference's firfilter2_typed_cpu<T> for T = x.dtype (b is cast to it); returns
    (result as double, is_fp64)."""
    lib = reference()
    if lib is None:
        raise OracleError("reference library not built")
    x = np.ascontiguousarray(x)
    b = np.ascontiguousarray(np.asarray(b).astype(x.dtype))
    shape = np.asarray(x.shape, dtype=np.int32)
    out = np.zeros(x.shape, dtype=np.float64)
    is64 = ctypes.c_int(0)
    _check(lib.zkx_ref_firfilter2(_REF_DTYPE[x.dtype], b.ctypes.data, b.size, x.ctypes.data, shape.ctypes.data,
                                  x.ndim, axis, PADTYPE[padtype], int(padlen is not None), padlen or 0,
                                  out.ctypes.data, ctypes.byref(is64)), lib)
    return out, bool(is64.value)


def hilbert(x, nfft: Optional[int] = None) -> np.ndarray:
    """The C restatement along the last axis of x [lines, n]; complex128 [lines, nfft]."""
    x = _f32(x)
    x2 = x.reshape(int(np.prod(x.shape[:-1])), x.shape[-1])
    nf = x2.shape[1] if nfft is None else nfft
    out = np.zeros((x2.shape[0], nf), dtype=np.complex128)
    _check(restatement().or_hilbert(x2.ctypes.data, x2.shape[0], x2.shape[1], nf, out.ctypes.data))
    return out.reshape(x.shape[:-1] + (nf,))


def ref_hilbert(x, nfft: Optional[int] = None, axis: int = -1):
    """The reference's hilbert_typed_cpu<T> for T = x.dtype; returns (complex128, is_fp64)."""
    lib = reference()
    if lib is None:
        raise OracleError("reference library not built")
    x = np.ascontiguousarray(x)
    shape = np.asarray(x.shape, dtype=np.int32)
    ax = axis % x.ndim
    out_shape = list(x.shape)
    out_shape[ax] = x.shape[ax] if nfft is None else nfft
    out = np.zeros(out_shape, dtype=np.complex128)
    is64 = ctypes.c_int(0)
    _check(lib.zkx_ref_hilbert(_REF_DTYPE[x.dtype], x.ctypes.data, shape.ctypes.data, x.ndim, axis,
                               int(nfft is not None), nfft or 0, out.ctypes.data, ctypes.byref(is64)), lib)
    return out, bool(is64.value)
