"""Reader and writer of the .kfh container (include/kielflow_b200.h, "Files").

The reference writes HDF5 files (IO.cpp:60-505, 1295-1340); this library
writes the same hierarchy of datasets -- version, date, path, time,
domain/{type_,m_,l0_,N_,L_}{x,y,z}, parameters/..., data/{Ux,Uy,Uz,ni,Ph} --
as a flat list of named entries:

    "KFH1", u32 entry count, then per entry: u16 name length, name (UTF-8),
    u8 type (1 f64, 2 i32, 3 string, 4 i64), u8 rank, u64 dims[rank],
    little-endian payload.
"""
from __future__ import annotations

import struct

import numpy as np

_F64, _I32, _STR, _I64 = 1, 2, 3, 4
_DT = {_F64: np.float64, _I32: np.int32, _I64: np.int64}


def read(path: str) -> dict:
    """{name: value}: scalars as Python numbers, strings as str, arrays as numpy."""
    out = {}
    with open(path, "rb") as f:
        if f.read(4) != b"KFH1":
            raise ValueError(f"{path}: not a .kfh file")
        (count,) = struct.unpack("<I", f.read(4))
        for _ in range(count):
            (nl,) = struct.unpack("<H", f.read(2))
            name = f.read(nl).decode()
            typ, rank = struct.unpack("<BB", f.read(2))
            dims = struct.unpack(f"<{rank}Q", f.read(8 * rank)) if rank else ()
            n = int(np.prod(dims)) if rank else 1
            if typ == _STR:
                out[name] = f.read(n).decode()
            else:
                a = np.frombuffer(f.read(n * np.dtype(_DT[typ]).itemsize), dtype=_DT[typ])
                out[name] = a.reshape(dims).copy() if rank else a[0].item()
    return out


def write(path: str, entries) -> None:
    """entries: iterable of (name, value); float -> f64, int -> i32, str,
    numpy float arrays -> f64 arrays (np.int64 scalars -> i64)."""
    parts = [b"KFH1", struct.pack("<I", len(entries))]
    for name, v in entries:
        nb = name.encode()
        parts.append(struct.pack("<H", len(nb)) + nb)
        if isinstance(v, str):
            b = v.encode()
            parts.append(struct.pack("<BBQ", _STR, 1, len(b)) + b)
        elif isinstance(v, np.ndarray):
            a = np.ascontiguousarray(v, np.float64)
            parts.append(struct.pack(f"<BB{a.ndim}Q", _F64, a.ndim, *a.shape) + a.tobytes())
        elif isinstance(v, np.int64):
            parts.append(struct.pack("<BBq", _I64, 0, int(v)))
        elif isinstance(v, int):
            parts.append(struct.pack("<BBi", _I32, 0, v))
        else:
            parts.append(struct.pack("<BBd", _F64, 0, float(v)))
    with open(path, "wb") as f:
        f.write(b"".join(parts))
