"""Reader for the named-array files written by oracle/ref_main.cpp.

Format: magic b"BBWA0001", then records of
  u32 name_len | name | u32 dtype (0=f32, 1=f64, 2=i32) | u64 count | data.
FP64 matrices are stored column-major (Eigen's layout).
"""
import numpy as np

_DT = {0: np.float32, 1: np.float64, 2: np.int32}


def read(path):
    out = {}
    with open(path, "rb") as f:
        if f.read(8) != b"BBWA0001":
            raise ValueError("%s: not a BBWA file" % path)
        while True:
            h = f.read(4)
            if len(h) < 4:
                break
            n = int(np.frombuffer(h, np.uint32)[0])
            name = f.read(n).decode()
            dt = int(np.frombuffer(f.read(4), np.uint32)[0])
            cnt = int(np.frombuffer(f.read(8), np.uint64)[0])
            out[name] = np.frombuffer(f.read(cnt * np.dtype(_DT[dt]).itemsize), _DT[dt]).copy()
    return out
