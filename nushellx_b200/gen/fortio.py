"""Fortran unformatted sequential records (4-byte length marker before and after
each record, little endian), the layout Intel Fortran uses for every binary file
of the reference (``form='unformatted'``)."""
import struct
import numpy as np


class RecordWriter:
    def __init__(self, path):
        self.f = open(path, "wb")

    def write(self, *items):
        payload = b"".join(_pack(x) for x in items)
        n = struct.pack("<i", len(payload))
        self.f.write(n + payload + n)

    def close(self):
        self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _pack(x):
    if isinstance(x, (bytes, bytearray)):
        return bytes(x)
    if isinstance(x, np.ndarray):
        return np.ascontiguousarray(x).tobytes()
    raise TypeError(type(x))


def i4(*v):
    return np.array(v, dtype="<i4")


def r4(*v):
    return np.array(v, dtype="<f4")


def r8(*v):
    return np.array(v, dtype="<f8")


def l4(v):
    # Intel Fortran LOGICAL(4): .TRUE. = -1, .FALSE. = 0
    return np.array([-1 if v else 0], dtype="<i4")


def read_records(path):
    """All records of a file as a list of bytes objects."""
    out = []
    with open(path, "rb") as f:
        data = f.read()
    p = 0
    while p < len(data):
        (n,) = struct.unpack_from("<i", data, p)
        rec = data[p + 4:p + 4 + n]
        (n2,) = struct.unpack_from("<i", data, p + 4 + n)
        if n2 != n:
            raise ValueError(f"{path}: record length markers differ ({n} vs {n2}) at byte {p}")
        out.append(rec)
        p += 8 + n
    return out
