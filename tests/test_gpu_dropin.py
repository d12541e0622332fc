"""The cusignal:: C++ API (include/cusignal/...) end to end: tests/cpp/dropin_probe.cu is
compiled against the headers and libzkx_rd.so, run on the GPU with inputs written here,
and every result it writes is checked against the oracle."""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "cpp"))
import build_probe  # noqa: E402

REL_L2 = 1e-5
P, N, L, NF, NT = 32, 256, 40, 4096, 31


def rel(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def hilbert64(x, nfft):
    """Analytic signal along the last axis in FP64 (the same mask as the restatement)."""
    X = np.fft.fft(np.asarray(x, dtype=np.float64), n=nfft, axis=-1)
    w = np.zeros(nfft)
    w[0] = 1.0
    w[1:(nfft + 1) // 2] = 2.0
    if nfft % 2 == 0:
        w[nfft // 2] = 1.0
    return np.fft.ifft(X * w, axis=-1)


def test_dropin_headers_compile_and_link():
    """The headers compile as C++17 with nvcc and the probe links against the library
    (no GPU needed)."""
    with tempfile.TemporaryDirectory() as d:
        assert os.path.exists(build_probe.build(d))


def test_runtime_headers_host_side():
    """The runtime headers Task1 and the probes include (errors, FP64 storage boundaries,
    launch configuration) compile and behave on the host without a GPU."""
    with tempfile.TemporaryDirectory() as d:
        exe = build_probe.build(d, "runtime_probe")
        r = subprocess.run([exe, "host"], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "FAIL" not in r.stdout


@pytest.mark.gpu
def test_runtime_headers_on_device():
    """Device queries, the event timer, 1-D launches with argument conversion to the
    kernel's parameter types, device-side FP64 widening and the allocation tracker that
    DeviceArray routes through."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    with tempfile.TemporaryDirectory() as d:
        exe = build_probe.build(d, "runtime_probe")
        r = subprocess.run([exe, "device"], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "FAIL" not in r.stdout


@pytest.mark.gpu
def test_dropin_api_matches_oracle():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(42)
    x = (rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))).astype(np.complex64)
    t = (rng.standard_normal(L) + 1j * rng.standard_normal(L)).astype(np.complex64)
    xh = x.astype(np.complex64)
    xh16 = np.stack([xh.real, xh.imag], -1).astype(np.float16)
    th16 = np.stack([t.real, t.imag], -1).astype(np.float16)
    ipow = rng.integers(0, 50, size=(P, N)).astype(np.int16)
    b = rng.standard_normal(NT).astype(np.float32)
    s = rng.standard_normal(NF).astype(np.float32)
    h = rng.standard_normal(7).astype(np.float32)
    si = rng.integers(-100, 100, size=NF).astype(np.int16)
    hi = rng.integers(-5, 6, size=5).astype(np.int16)
    with tempfile.TemporaryDirectory() as d:
        exe = build_probe.build(d)
        for name, arr in [("dims", np.array([P, N, L, NF, NT], dtype=np.int32)), ("x", x), ("t", t),
                          ("xh", xh16), ("th", th16), ("ipow", ipow), ("b", b), ("s", s), ("h", h),
                          ("si", si), ("hi", hi)]:
            arr.tofile(os.path.join(d, name + ".bin"))
        r = subprocess.run([exe, d], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr

        def out(name, dtype):
            return np.fromfile(os.path.join(d, "out_" + name + ".bin"), dtype=dtype)

        pc = out("pc", np.float64).view(np.complex128).reshape(P, N)
        assert rel(pc, O.pulse_compression_direct(x, t, -1, True, "hamming")) <= REL_L2
        pc32 = out("pc32", np.float32).view(np.complex64).reshape(P, N)
        ref32 = O.pulse_compression_direct(x, t, -1, True)
        assert rel(pc32, ref32) <= REL_L2
        rd = out("rd", np.float32).view(np.complex64).reshape(P, N)
        rd64, _ = O.pulse_doppler_fft64(pc32, -1, O.radar_window_f32("hamming", P))
        assert rel(rd, rd64) <= REL_L2
        power = out("power", np.float32).reshape(P, N)
        thr_ref, det_ref = O.ca_cfar_compat(power, (2, 2), (4, 4), 1e-3)
        np.testing.assert_array_equal(out("thr", np.float32).reshape(P, N), thr_ref)
        np.testing.assert_array_equal(out("det", np.uint8).reshape(P, N), det_ref)
        # opted into the FP64-decided evaluation: the mask of an FP64 CFAR of the same power
        _, det64 = O.ca_cfar_f64(power, (2, 2), (4, 4), 1e-3)
        np.testing.assert_array_equal(out("det64", np.uint8).reshape(P, N), det64)
        # the probe passes pfa as float (1e-3f): alpha follows that FP32 probability in FP64
        assert out("alpha", np.float64)[0] == pytest.approx(
            O.cfar_alpha(float(np.float32(1e-3)), 2 * 4 * 13 + 2 * 5 * 4), rel=1e-15)
        # int16 CFAR: same thresholds as on the float-converted input, floor-rule mask
        ithr = out("ithr", np.float32).reshape(P, N)
        ithr_ref, _ = O.ca_cfar_compat(ipow.astype(np.float32), (2, 2), (4, 4), 1e-3)
        np.testing.assert_array_equal(ithr, ithr_ref)
        idet_ref = (ipow.astype(np.int64) > np.floor(ithr_ref).astype(np.int64)).astype(np.uint8)
        np.testing.assert_array_equal(out("idet", np.uint8).reshape(P, N), idet_ref)
        # half input: converted exactly to FP32, then the same compression
        xh32 = xh16.astype(np.float32).view(np.complex64).reshape(P, N)
        th32 = th16.astype(np.float32).view(np.complex64).reshape(L)
        assert rel(out("pch", np.float32).view(np.complex64).reshape(P, N),
                   O.pulse_compression_direct(xh32, th32, -1, True)) <= REL_L2
        # front end
        assert rel(out("fir", np.float32), O.firfilter(b, s)) <= REL_L2
        assert rel(out("fir_resident", np.float32), O.firfilter(b, s)) <= REL_L2
        fir0 = out("fir_axis0", np.float32).reshape(NF // 4, 4)
        assert rel(fir0, O.firfilter(b, s.reshape(NF // 4, 4).T.copy()).T) <= REL_L2
        assert rel(out("upfirdn", np.float32), O.upfirdn(h, s, 3, 2)) <= REL_L2
        assert rel(out("resample", np.float64), O.resample_poly(s, 3, 2)) <= REL_L2
        assert rel(out("upfirdn_i16", np.float32),
                   O.upfirdn(hi.astype(np.float32), si.astype(np.float32), 2, 3)) <= REL_L2
        a2d = out("amb2d", np.float32)
        ref2d = O.ambgfun(t, fs=2.0, cut="2d").ravel()
        assert np.linalg.norm(a2d - ref2d) / np.linalg.norm(ref2d) <= REL_L2
        for name, cut, cv in (("ambdoppler", "doppler", 0.1), ("ambdelay", "delay", 3.0)):
            got = out(name, np.float64)
            ref = O.ambgfun(t, fs=2.0, cut=cut, cut_value=cv)
            assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= REL_L2, name
        assert rel(out("fir2", np.float32), O.firfilter2(b, s)) <= REL_L2
        fir2i = out("fir2_i16_axis0", np.float32).reshape(NF // 8, 8)
        ref2i = O.firfilter2(np.array([1, 2, 1], np.float32), si.astype(np.float32).reshape(NF // 8, 8).T.copy(),
                             "even", 20, O.PAD_ROUNDING[np.dtype(np.int16)]).T
        assert rel(fir2i, ref2i) <= REL_L2
        hil = out("hilbert", np.float32).view(np.complex64)
        assert hil.size == 5000
        assert rel(hil, hilbert64(s, 5000)) <= REL_L2
        hili = out("hilbert_i16_axis0", np.float64).view(np.complex128).reshape(NF // 8, 8)
        assert rel(hili, hilbert64(si.astype(np.float32).reshape(NF // 8, 8).T, NF // 8).T) <= REL_L2
        spec = out("fft", np.float32).view(np.complex64).reshape(P, N)
        assert rel(spec, np.fft.fft(x.astype(np.complex128), axis=1)) <= REL_L2
        assert rel(out("ifft", np.float32).view(np.complex64).reshape(P, N), x) <= 1e-6
