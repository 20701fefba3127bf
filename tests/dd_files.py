"""Writers of the reference's workunit inputs for the drop-in tests: a gzip DD
file with the 1168-byte header read by src/workload.cpp:29-57 (sample time in
us at double 0, observation length at double 1, dm at double 13, scale at
double 14, sample count as uint32 at byte 128) followed by int8 samples, an
orbital bank (one "period tau psi" row per template, src/workload.cpp:96-107)
and a raw float32 file for --preprocessed."""
import gzip
import struct

import numpy as np


def write_dd(path, samples_i8, sample_us, scale=1.0, dm=0.0):
    n = len(samples_i8)
    header = bytearray(1168)
    struct.pack_into("<d", header, 0, sample_us)
    struct.pack_into("<d", header, 8, n * sample_us * 1e-6)
    struct.pack_into("<d", header, 13 * 8, dm)
    struct.pack_into("<d", header, 14 * 8, scale)
    struct.pack_into("<I", header, 128, n)
    with gzip.open(path, "wb") as f:
        f.write(bytes(header))
        f.write(np.asarray(samples_i8, dtype=np.int8).tobytes())


def write_bank(path, orbits):
    with open(path, "w") as f:
        for period, tau, psi in orbits:
            f.write("%.17g %.17g %.17g\n" % (period, tau, psi))


def write_floats(path, x):
    np.ascontiguousarray(x, dtype=np.float32).tofile(path)


def write_dd_bytes(path, raw, samples, sample_us, scale=1.0, dm=0.0):
    """As write_dd with the sample bytes given: int8 samples (.binary) or two
    4-bit samples per byte, high nibble first (.bin4)."""
    header = bytearray(1168)
    struct.pack_into("<d", header, 0, sample_us)
    struct.pack_into("<d", header, 8, samples * sample_us * 1e-6)
    struct.pack_into("<d", header, 13 * 8, dm)
    struct.pack_into("<d", header, 14 * 8, scale)
    struct.pack_into("<I", header, 128, samples)
    with gzip.open(path, "wb") as f:
        f.write(bytes(header))
        f.write(np.asarray(raw, dtype=np.uint8).tobytes())
