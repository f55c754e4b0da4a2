"""Reader/writer for the record files exchanged with the reference oracle.

Format (little endian), one record after another:
  b"Z4CREC01", int32 name_len, name, int32 dtype (0=float64, 1=int32),
  int32 ndim, int64 dims[ndim], row-major payload.
The C++ side lives in oracle/ref/z4c_oracle_io.hpp.
"""
import struct

import numpy as np

MAGIC = b"Z4CREC01"


def read_records(path):
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    p = 0
    while p < len(data):
        if data[p:p + 8] != MAGIC:
            raise ValueError(f"bad record magic at offset {p} in {path}")
        p += 8
        (nl,) = struct.unpack_from("<i", data, p); p += 4
        name = data[p:p + nl].decode(); p += nl
        dtype, nd = struct.unpack_from("<ii", data, p); p += 8
        dims = struct.unpack_from("<" + "q" * nd, data, p); p += 8 * nd
        dt = np.float64 if dtype == 0 else np.int32
        n = int(np.prod(dims)) if nd else 1
        arr = np.frombuffer(data, dtype=dt, count=n, offset=p).reshape(dims)
        p += n * np.dtype(dt).itemsize
        out[name] = arr.copy()
    return out


def write_records(path, records):
    with open(path, "wb") as f:
        for name, arr in records.items():
            arr = np.ascontiguousarray(arr)
            if arr.dtype == np.float64:
                code = 0
            elif arr.dtype == np.int32:
                code = 1
            else:
                raise TypeError(f"{name}: unsupported dtype {arr.dtype}")
            nb = name.encode()
            f.write(MAGIC)
            f.write(struct.pack("<i", len(nb)))
            f.write(nb)
            f.write(struct.pack("<ii", code, arr.ndim))
            f.write(struct.pack("<" + "q" * arr.ndim, *arr.shape))
            f.write(arr.tobytes())
