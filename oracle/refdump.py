"""Reader for the tagged binary dumps written by oracle/ref_driver.cpp.

ORACLE TEST INFRASTRUCTURE ONLY: used by tests to load the reference's own
state; never imported by the product package.
"""
import struct

import numpy as np

_DT = {0: np.float64, 1: np.float32, 2: np.uint8, 3: np.int64}


def read_dump(path):
    """Return {name: ndarray} for one dump file."""
    out = {}
    with open(path, "rb") as fh:
        data = fh.read()
    if data[:8] != b"PDDUMP01":
        raise ValueError(f"{path}: not a PDDUMP01 file")
    p = 8
    while p < len(data):
        (ln,) = struct.unpack_from("<I", data, p)
        p += 4
        name = data[p:p + ln].decode()
        p += ln
        dt, n = struct.unpack_from("<IQ", data, p)
        p += 12
        t = np.dtype(_DT[dt])
        out[name] = np.frombuffer(data, dtype=t, count=n, offset=p).copy()
        p += n * t.itemsize
    return out
