"""Reference ``.bin`` vector format (test infrastructure).

Layout (``matlab/writebin_vector.m:35-44``, ``matlab/readbin_vector.m:30-40``):
uint8 is_complex, uint32 n (little-endian), n float64 real parts, then n
float64 imaginary parts when is_complex.
"""

import struct

import numpy as np


def write_bin(path, v):
    v = np.asarray(v).ravel()
    cplx = np.iscomplexobj(v)
    with open(path, "wb") as f:
        f.write(struct.pack("<BI", 1 if cplx else 0, v.size))
        f.write(np.ascontiguousarray(v.real, dtype="<f8").tobytes())
        if cplx:
            f.write(np.ascontiguousarray(v.imag, dtype="<f8").tobytes())


def read_bin(path):
    with open(path, "rb") as f:
        hdr = f.read(5)
        cplx, n = struct.unpack("<BI", hdr)
        re = np.frombuffer(f.read(8 * n), dtype="<f8")
        if cplx & 1:
            im = np.frombuffer(f.read(8 * n), dtype="<f8")
            return re + 1j * im
        return re.copy()
