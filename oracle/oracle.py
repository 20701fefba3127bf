"""Python access to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle is the checker of the CUDA search path: only tests/, the smoke entry
point and bench.py's cpu_baseline / reference legs use it.  It wraps

* ``liboracle.so`` -- the C restatement in brp_oracle.c of the reference's CPU
  code (src/science.cpp, src/workload.cpp) and of shaders/harmonic.comp, and
* ``_ref/libbrp_ref.so`` (optional) -- the reference's own src/science.cpp and
  src/workload.cpp compiled from their sources by ``make ref``.

The FP64 spectrum oracle is numpy's float64 real FFT (pocketfft), which
tests also pin against the C FP64 DFT of brp_oracle.c.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class Params(ctypes.Structure):
    """brp::Params, 108 bytes (include/brp/science.hpp:8-17)."""
    _fields_ = [("n", ctypes.c_uint32), ("unpadded", ctypes.c_uint32), ("steps", ctypes.c_uint32),
                ("logn", ctypes.c_uint32), ("tau", ctypes.c_float), ("omega", ctypes.c_float),
                ("psi", ctypes.c_float), ("dt", ctypes.c_float), ("step_inv", ctypes.c_float),
                ("s0", ctypes.c_float), ("fundamental", ctypes.c_uint32), ("harmonic", ctypes.c_uint32),
                ("window", ctypes.c_uint32), ("stage", ctypes.c_uint32), ("threshold", ctypes.c_float * 5),
                ("capacity", ctypes.c_uint32), ("fft_n", ctypes.c_uint32), ("fft_base", ctypes.c_uint32),
                ("fft_radix", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("twiddle3", ctypes.c_uint32),
                ("twiddle_real", ctypes.c_uint32), ("result_slot", ctypes.c_uint32)]


assert ctypes.sizeof(Params) == 108

CANDIDATE = np.dtype([("bin", "<u4"), ("level", "<u4"), ("power", "<f4"), ("reserved", "<u4")])
BANK_CANDIDATE = np.dtype([("power", "<f8"), ("period", "<f8"), ("tau", "<f8"), ("psi", "<f8"),
                           ("significance", "<f8"), ("harmonics", "<u4"), ("bin", "<u4")])


class OracleError(RuntimeError):
    pass


def _as_params(p):
    """Accepts any 108-byte brp::Params-layout ctypes structure."""
    if isinstance(p, Params):
        return p
    return Params.from_buffer_copy(bytes(p))


def _fp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _load(path, make_target):
    if not os.path.exists(path):
        subprocess.run(["make", "-s", "-C", HERE, make_target], check=True)
    return ctypes.CDLL(path)


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = _load(os.path.join(HERE, "liboracle.so"), "oracle")
        P = ctypes.POINTER(Params)
        L.oracle_lut_sin.restype = ctypes.c_float
        L.oracle_lut_sin.argtypes = [ctypes.c_float]
        L.oracle_fused_sin.restype = ctypes.c_float
        L.oracle_fused_sin.argtypes = [ctypes.c_float]
        L.oracle_sample_offset.restype = ctypes.c_float
        L.oracle_sample_offset.argtypes = [ctypes.c_uint32, P]
        L.oracle_resampling_steps.argtypes = [P]
        L.oracle_parameters.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_float,
                                        ctypes.c_float, ctypes.c_float, P]
        L.oracle_resample.argtypes = [ctypes.c_void_p, ctypes.c_size_t, P, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_exact_mean.restype = ctypes.c_float
        L.oracle_exact_mean.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        L.oracle_power_from_fft.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]
        L.oracle_harmonic.argtypes = [ctypes.c_void_p, ctypes.c_size_t, P, ctypes.c_void_p]
        L.oracle_select.restype = ctypes.c_size_t
        L.oracle_select.argtypes = [ctypes.c_void_p, P, ctypes.c_void_p, ctypes.c_size_t]
        L.oracle_chisq_Q.restype = ctypes.c_double
        L.oracle_chisq_Q.argtypes = [ctypes.c_double, ctypes.c_double]
        L.oracle_chisq_Qinv.restype = ctypes.c_double
        L.oracle_chisq_Qinv.argtypes = [ctypes.c_double, ctypes.c_double]
        L.oracle_search_parameters.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_uint32, P]
        L.oracle_toplist_init.argtypes = [ctypes.c_void_p]
        L.oracle_toplist_thresholds.argtypes = [ctypes.c_void_p, P]
        L.oracle_toplist_retain.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, P]
        L.oracle_toplist_final.restype = ctypes.c_size_t
        L.oracle_toplist_final.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_rfft64.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_rngmed.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]
        L.oracle_taus2_seed.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        L.oracle_taus2_get.restype = ctypes.c_uint32
        L.oracle_taus2_get.argtypes = [ctypes.c_void_p]
        L.oracle_gaussian_ziggurat.restype = ctypes.c_double
        L.oracle_gaussian_ziggurat.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.oracle_dd_sample.restype = ctypes.c_float
        L.oracle_dd_sample.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_double]
        L.oracle_preprocess.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_uint32, ctypes.c_void_p]
        L.oracle_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _check(status):
    if status:
        raise OracleError(lib().oracle_last_error().decode())


def lut_sin(x):
    return np.float32(lib().oracle_lut_sin(float(x)))


def fused_sin(x):
    return np.float32(lib().oracle_fused_sin(float(x)))


def sample_offset(i, p):
    return np.float32(lib().oracle_sample_offset(int(i), ctypes.byref(_as_params(p))))


def parameters(n, unpadded, tau, period, psi, dt):
    """science.cpp:46-65 (bench-mode template constants)."""
    p = Params()
    _check(lib().oracle_parameters(n, unpadded, float(np.float32(tau)), float(np.float32(period)),
                                   float(np.float32(psi)), float(np.float32(dt)), ctypes.byref(_as_params(p))))
    return p


def production(p):
    """src/main.cpp:41: production FMA arithmetic with the float-sine S0."""
    q = Params.from_buffer_copy(bytes(p))
    q.flags = 2 | 4
    q.s0 = np.float32(np.float32(q.tau) * np.float32(np.sin(np.float32(q.psi)))) * np.float32(q.step_inv)
    _check(lib().oracle_resampling_steps(ctypes.byref(q)))
    return q


def resampling_steps(p):
    q = Params.from_buffer_copy(bytes(p))
    _check(lib().oracle_resampling_steps(ctypes.byref(q)))
    return q


def search_parameters(n, samples, sample_us, period, tau, psi, f0=400.0, false_alarm=0.08, window=1000):
    """workload.cpp:108-125."""
    p = Params()
    _check(lib().oracle_search_parameters(n, samples, sample_us, period, tau, psi, f0, false_alarm, window,
                                          ctypes.byref(_as_params(p))))
    return p


def resample(x, p, with_index=False):
    """science.cpp:75-85: (padded series of length n, resample indices j(i) for i<steps)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(p.n, np.float32)
    idx = np.empty(max(p.steps, 1), np.int32)
    _check(lib().oracle_resample(_fp(x), x.size, ctypes.byref(_as_params(p)), _fp(out), _fp(idx)))
    return (out, idx[:p.steps]) if with_index else out


def exact_mean(resampled, steps):
    r = np.ascontiguousarray(resampled, dtype=np.float32)
    return np.float32(lib().oracle_exact_mean(_fp(r), steps))


def rfft64(x):
    """FP64 real DFT (numpy pocketfft) of a float32 series: n/2+1 complex128 bins."""
    return np.fft.rfft(np.asarray(x, dtype=np.float64))


def rfft64_c(x):
    """FP64 real DFT by the C oracle (independent of numpy)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    re = np.empty(x.size // 2 + 1)
    im = np.empty(x.size // 2 + 1)
    _check(lib().oracle_rfft64(_fp(x), x.size, _fp(re), _fp(im)))
    return re + 1j * im


def power_from_fft(X, n):
    """science.cpp:114-118 applied to an FP64 spectrum."""
    re = np.ascontiguousarray(X.real, dtype=np.float64)
    im = np.ascontiguousarray(X.imag, dtype=np.float64)
    out = np.empty(n // 2, np.float32)
    lib().oracle_power_from_fft(_fp(re), _fp(im), n, _fp(out))
    return out


def power64(X, n):
    """Power spectrum in FP64 (the power parity reference): |X_k|^2 / n, P[0] = 0."""
    P = (X.real[: n // 2] ** 2 + X.imag[: n // 2] ** 2) / n
    P[0] = 0
    return P


def harmonic(power, p):
    """shaders/harmonic.comp: summed[5*fundamental]."""
    P = np.ascontiguousarray(power, dtype=np.float32)
    out = np.empty(5 * p.fundamental, np.float32)
    _check(lib().oracle_harmonic(_fp(P), P.size, ctypes.byref(_as_params(p)), _fp(out)))
    return out


def select(summed, p, cap=1 << 22):
    s = np.ascontiguousarray(summed, dtype=np.float32)
    out = np.empty(cap, CANDIDATE)
    n = lib().oracle_select(_fp(s), ctypes.byref(_as_params(p)), _fp(out), cap)
    if n > cap:
        raise OracleError("candidate buffer too small")
    return out[:n].copy()


def chisq_Q(x, nu):
    return lib().oracle_chisq_Q(x, nu)


def chisq_Qinv(q, nu):
    return lib().oracle_chisq_Qinv(q, nu)


def pipeline(x, p):
    """The reference's CPU pipeline (science.cpp:113-120) with the FP64 FFT:
    returns dict(resampled, index, fft, power, summed, candidates)."""
    r, idx = resample(x, p, with_index=True)
    X = rfft64(r)
    P = power_from_fft(X, p.n)
    S = harmonic(P, p)
    return dict(resampled=r, index=idx, fft=X, power=P, summed=S, candidates=select(S, p))


class Toplist:
    """workload.cpp:126-159 (5 levels x 100 rows)."""

    def __init__(self):
        self._buf = np.zeros(500, BANK_CANDIDATE)
        lib().oracle_toplist_init(_fp(self._buf))

    def thresholds(self, p):
        q = Params.from_buffer_copy(bytes(p))
        lib().oracle_toplist_thresholds(_fp(self._buf), ctypes.byref(q))
        return q

    def retain(self, cands, period, tau, psi, p):
        c = np.ascontiguousarray(cands, dtype=CANDIDATE)
        _check(lib().oracle_toplist_retain(_fp(self._buf), _fp(c), c.size, period, tau, psi, ctypes.byref(_as_params(p))))

    def final(self):
        out = np.zeros(100, BANK_CANDIDATE)
        n = lib().oracle_toplist_final(_fp(self._buf), _fp(out))
        return out[:n].copy()


# ---- the reference's own CPU code, compiled from its sources (optional) ----
_ref = None


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libbrp_ref.so"))


def ref():
    """ctypes handle on _ref/libbrp_ref.so (built only where the reference sources exist)."""
    global _ref
    if _ref is None:
        R = ctypes.CDLL(os.path.join(HERE, "_ref", "libbrp_ref.so"))
        P = ctypes.POINTER(Params)
        R.ref_last_error.restype = ctypes.c_char_p
        R.ref_lut_sin.restype = ctypes.c_float
        R.ref_lut_sin.argtypes = [ctypes.c_float]
        R.ref_sample_offset.restype = ctypes.c_float
        R.ref_sample_offset.argtypes = [ctypes.c_uint32, P]
        R.ref_parameters.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_float,
                                     ctypes.c_float, ctypes.c_float, P]
        R.ref_resampling_steps.argtypes = [P]
        R.ref_resample.argtypes = [ctypes.c_void_p, ctypes.c_uint32, P, ctypes.c_void_p]
        R.ref_reference.argtypes = [ctypes.c_void_p, ctypes.c_uint32, P] + [ctypes.c_void_p] * 5 + \
            [ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]
        R.ref_harmonic.argtypes = [ctypes.c_void_p, ctypes.c_uint32, P, ctypes.c_void_p]
        R.ref_search_parameters.argtypes = [ctypes.c_uint32, ctypes.c_uint32] + [ctypes.c_double] * 6 + \
            [ctypes.c_uint32, P]
        R.ref_toplist_new.restype = ctypes.c_void_p
        R.ref_toplist_free.argtypes = [ctypes.c_void_p]
        R.ref_toplist_thresholds.argtypes = [ctypes.c_void_p, P]
        R.ref_toplist_retain.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, P]
        R.ref_toplist_final.restype = ctypes.c_uint32
        R.ref_toplist_final.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        R.ref_load_observation.argtypes = [ctypes.c_char_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_uint32]
        R.ref_preprocess.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_void_p]
        _ref = R
    return _ref


def _rcheck(status):
    if status:
        raise OracleError(ref().ref_last_error().decode())


def ref_parameters(n, unpadded, tau, period, psi, dt):
    p = Params()
    _rcheck(ref().ref_parameters(n, unpadded, float(np.float32(tau)), float(np.float32(period)),
                                 float(np.float32(psi)), float(np.float32(dt)), ctypes.byref(_as_params(p))))
    return p


def ref_resampling_steps(p):
    q = Params.from_buffer_copy(bytes(p))
    _rcheck(ref().ref_resampling_steps(ctypes.byref(q)))
    return q


def ref_search_parameters(n, samples, sample_us, period, tau, psi, f0=400.0, false_alarm=0.08, window=1000):
    p = Params()
    _rcheck(ref().ref_search_parameters(n, samples, sample_us, period, tau, psi, f0, false_alarm, window,
                                        ctypes.byref(_as_params(p))))
    return p


def ref_resample(x, p):
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(p.n, np.float32)
    _rcheck(ref().ref_resample(_fp(x), x.size, ctypes.byref(_as_params(p)), _fp(out)))
    return out


def ref_reference(x, p, cap=1 << 20):
    """src/science.cpp:113-120 run from the reference's own compiled code."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    r = np.empty(p.n, np.float32)
    f = np.empty(2 * (p.n // 2 + 1), np.float32)
    P = np.empty(p.n // 2, np.float32)
    S = np.empty(5 * p.fundamental, np.float32)
    c = np.empty(cap, CANDIDATE)
    count = ctypes.c_uint32()
    _rcheck(ref().ref_reference(_fp(x), x.size, ctypes.byref(_as_params(p)), _fp(r), _fp(f), _fp(P), _fp(S), _fp(c), cap,
                                ctypes.byref(count)))
    return dict(resampled=r, fft=f.view(np.complex64), power=P, summed=S, candidates=c[:count.value].copy())


def ref_harmonic(power, p):
    P = np.ascontiguousarray(power, dtype=np.float32)
    S = np.empty(5 * p.fundamental, np.float32)
    _rcheck(ref().ref_harmonic(_fp(P), P.size, ctypes.byref(_as_params(p)), _fp(S)))
    return S


class RefToplist:
    """brp::Toplist from the reference's compiled src/workload.cpp."""

    def __init__(self):
        self._t = ref().ref_toplist_new()

    def __del__(self):
        if getattr(self, "_t", None):
            ref().ref_toplist_free(self._t)

    def thresholds(self, p):
        q = Params.from_buffer_copy(bytes(p))
        ref().ref_toplist_thresholds(self._t, ctypes.byref(q))
        return q

    def retain(self, cands, period, tau, psi, p):
        c = np.ascontiguousarray(cands, dtype=CANDIDATE)
        _rcheck(ref().ref_toplist_retain(self._t, _fp(c), c.size, period, tau, psi, ctypes.byref(_as_params(p))))

    def final(self):
        out = np.zeros(100, BANK_CANDIDATE)
        n = ref().ref_toplist_final(self._t, _fp(out))
        return out[:n].copy()


# ---- whitening (src/workload.cpp:58-95) and DD decoding (:48-56) ----
class Taus2(ctypes.Structure):
    _fields_ = [("s1", ctypes.c_uint32), ("s2", ctypes.c_uint32), ("s3", ctypes.c_uint32)]


def rngmed(data, window):
    data = np.ascontiguousarray(data, np.float32)
    out = np.empty(len(data) - window + 1, np.float32)
    _check(lib().oracle_rngmed(_fp(data), len(data), window, _fp(out)))
    return out


def zap_noise(seed, count, sigma):
    """`count` (real, imaginary) Gaussian pairs of the restated taus2/ziggurat stream."""
    r = Taus2()
    lib().oracle_taus2_seed(ctypes.byref(r), seed)
    out = np.empty(2 * count, np.float32)
    for k in range(2 * count):
        out[k] = lib().oracle_gaussian_ziggurat(ctypes.byref(r), sigma)
    return out


def dd_decode(raw, samples, packed, scale):
    raw = np.ascontiguousarray(raw, np.uint8)
    return np.array([lib().oracle_dd_sample(_fp(raw), i, int(packed), scale) for i in range(samples)], np.float32)


def preprocess(decoded, n, sample_us, padding, window, zap_lower=(), zap_upper=()):
    decoded = np.ascontiguousarray(decoded, np.float32)
    lo = np.ascontiguousarray(zap_lower, np.float64)
    hi = np.ascontiguousarray(zap_upper, np.float64)
    out = np.empty(len(decoded), np.float32)
    _check(lib().oracle_preprocess(_fp(decoded), len(decoded), n, sample_us, padding, window, _fp(lo), _fp(hi),
                                   len(lo), _fp(out)))
    return out


def ref_preprocess(decoded, n, sample_us, padding, zap_path, window):
    decoded = np.ascontiguousarray(decoded, np.float32)
    out = np.empty(len(decoded), np.float32)
    _rcheck(ref().ref_preprocess(_fp(decoded), len(decoded), n, sample_us, padding, str(zap_path).encode(), window,
                                 _fp(out)))
    return out


def ref_load_observation(path, padding):
    """(sample_us, scale, samples, n), decoded samples, by the reference's loader."""
    meta = np.zeros(4, np.float64)
    _rcheck(ref().ref_load_observation(str(path).encode(), padding, _fp(meta), None, 0))
    out = np.empty(int(meta[2]), np.float32)
    _rcheck(ref().ref_load_observation(str(path).encode(), padding, _fp(meta), _fp(out), len(out)))
    return (float(meta[0]), float(meta[1]), int(meta[2]), int(meta[3])), out
