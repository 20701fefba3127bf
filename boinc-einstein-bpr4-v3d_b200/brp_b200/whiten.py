"""Whitening and RFI zapping of an observation on the GPU (brp::preprocess,
src/workload.cpp:58-95), optionally from the raw DD samples
(brp::load_observation's decoding, src/workload.cpp:48-56)."""
import ctypes

import numpy as np

from ._lib import BrpError, lib, ptr

_BOUND = False


def _bind():
    global _BOUND
    if _BOUND:
        return lib()
    L = lib()
    d, u32, i32, vp = ctypes.c_double, ctypes.c_uint32, ctypes.c_int32, ctypes.c_void_p
    L.brp_cuda_preprocess.argtypes = [vp, u32, u32, d, d, u32, vp, vp, u32, vp, i32]
    L.brp_cuda_preprocess_dd.argtypes = [vp, u32, i32, d, u32, d, d, u32, vp, vp, u32, vp, vp, i32]
    L.brp_cuda_preprocess_error.restype = ctypes.c_char_p
    L.brp_host_read_zap.argtypes = [ctypes.c_char_p, vp, vp, u32, ctypes.POINTER(u32)]
    L.brp_host_zap_noise.argtypes = [u32, u32, d, d, vp, vp, u32, vp, vp, u32, ctypes.POINTER(u32)]
    L.brp_host_error.restype = ctypes.c_char_p
    _BOUND = True
    return L


def read_zap(path):
    """(lower, upper) arrays of a zap-list file (src/workload.cpp:77-88 rules)."""
    L = _bind()
    n = ctypes.c_uint32()
    if L.brp_host_read_zap(str(path).encode(), None, None, 0, ctypes.byref(n)):
        raise BrpError(4, L.brp_host_error().decode())
    lo, hi = np.zeros(n.value, np.float64), np.zeros(n.value, np.float64)
    if n.value and L.brp_host_read_zap(str(path).encode(), ptr(lo), ptr(hi), n.value, ctypes.byref(n)):
        raise BrpError(4, L.brp_host_error().decode())
    return lo, hi


def zap_noise(seed, n, sample_us, padding, lower, upper):
    """(bins, values[count, 2]) of the zap noise, in the order the reference draws it."""
    L = _bind()
    lo, hi = np.ascontiguousarray(lower, np.float64), np.ascontiguousarray(upper, np.float64)
    c = ctypes.c_uint32()
    if L.brp_host_zap_noise(seed, n, sample_us, padding, ptr(lo), ptr(hi), len(lo), None, None, 0, ctypes.byref(c)):
        raise BrpError(4, L.brp_host_error().decode())
    bins, vals = np.zeros(c.value, np.uint32), np.zeros((c.value, 2), np.float32)
    if c.value and L.brp_host_zap_noise(seed, n, sample_us, padding, ptr(lo), ptr(hi), len(lo), ptr(bins), ptr(vals),
                                        c.value, ctypes.byref(c)):
        raise BrpError(4, L.brp_host_error().decode())
    return bins, vals


def preprocess(decoded, n, sample_us, padding, window=1000, zap=None, device=-1):
    """Whitened, zapped series (float32, len(decoded)) of a decoded series
    zero-padded to n; zap = (lower, upper) arrays or a zap-list path."""
    L = _bind()
    x = np.ascontiguousarray(decoded, np.float32)
    lo, hi = _zap_arrays(zap)
    out = np.empty(len(x), np.float32)
    st = L.brp_cuda_preprocess(ptr(x), len(x), n, sample_us, padding, window, ptr(lo), ptr(hi), len(lo), ptr(out),
                               device)
    if st:
        raise BrpError(st, L.brp_cuda_preprocess_error().decode())
    return out


def preprocess_dd(raw, samples, packed, scale, n, sample_us, padding, window=1000, zap=None, device=-1):
    """As preprocess() from raw DD sample bytes (int8, or two 4-bit samples per
    byte, high nibble first), decoded on the device; returns (decoded, preprocessed)."""
    L = _bind()
    b = np.ascontiguousarray(raw, np.uint8)
    lo, hi = _zap_arrays(zap)
    dec, out = np.empty(samples, np.float32), np.empty(samples, np.float32)
    st = L.brp_cuda_preprocess_dd(ptr(b), samples, int(packed), scale, n, sample_us, padding, window, ptr(lo),
                                  ptr(hi), len(lo), ptr(dec), ptr(out), device)
    if st:
        raise BrpError(st, L.brp_cuda_preprocess_error().decode())
    return dec, out


def _zap_arrays(zap):
    if zap is None:
        return np.zeros(0, np.float64), np.zeros(0, np.float64)
    if isinstance(zap, (str, bytes)) or hasattr(zap, "__fspath__"):
        return read_zap(zap)
    lo, hi = zap
    return np.ascontiguousarray(lo, np.float64), np.ascontiguousarray(hi, np.float64)
