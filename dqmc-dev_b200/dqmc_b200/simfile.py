"""Sim-file container: the named-array file the engine reads and writes.

The reference keeps a simulation in an HDF5 file whose dataset paths are
fixed by its generator (util/gen_1band_unified_hub.py:929-1160) and read and
written by src/data.c:345-789.  No HDF5 library exists on the machines this
engine runs on, so the same dataset paths, dtypes, shapes and byte order
(C order, as h5py writes numpy arrays) are kept in a flat container:

    offset 0    magic  b"DQSF0001"
    offset 8    u64    number of entries
    offset 16   u64    byte offset of the entry table (64)
    offset 64   entry table, 128 bytes per entry:
                  char[80] name   ("params/N", no leading slash)
                  u32      dtype  (DT_* below)
                  u32      ndim   (0..3)
                  u64[3]   shape
                  u64      data offset (64-byte aligned)
                  u64      data size in bytes
    data blocks

A DT_LINK entry named "params" whose data is a relative file name plays the
role of the reference's HDF5 external link (gen_1band_unified_hub.py:1046-1048):
any "params/..." lookup that misses resolves in the linked file.  Writes after
creation are in place, like the reference's H5Dwrite on existing datasets
(data.c:663-789), so a dataset's dtype and size never change.
"""
from __future__ import annotations

import os
import struct

import numpy as np

MAGIC = b"DQSF0001"
HEADER = 64
ENTRY = 128
NAME_LEN = 80
ALIGN = 64

DT_I32, DT_I64, DT_F64, DT_C128, DT_U64, DT_STR, DT_LINK = 1, 2, 3, 4, 5, 6, 7

_NP2DT = {
    np.dtype(np.int32): DT_I32,
    np.dtype(np.int64): DT_I64,
    np.dtype(np.float64): DT_F64,
    np.dtype(np.complex128): DT_C128,
    np.dtype(np.uint64): DT_U64,
}
_DT2NP = {v: k for k, v in _NP2DT.items()}

_ENTRY_FMT = "<%dsII3QQQ" % NAME_LEN
assert struct.calcsize(_ENTRY_FMT) == ENTRY


class Link:
    """Marker for a group that lives in another container file."""

    def __init__(self, filename: str):
        self.filename = filename

    def __repr__(self):
        return f"Link({self.filename!r})"


def _norm(name: str) -> str:
    return name.strip("/")


def _as_array(value):
    if isinstance(value, (Link, str, bytes)):
        return value
    if isinstance(value, bool):
        return np.array(int(value), dtype=np.int64)
    if isinstance(value, int):
        return np.array(value, dtype=np.int64)
    if isinstance(value, float):
        return np.array(value, dtype=np.float64)
    if isinstance(value, complex):
        return np.array(value, dtype=np.complex128)
    a = np.asarray(value)
    if a.dtype.kind == "b":
        a = a.astype(np.int64)
    elif a.dtype == np.int8 or a.dtype == np.int16:
        a = a.astype(np.int32)
    elif a.dtype == np.uint32:
        a = a.astype(np.int64)
    elif a.dtype == np.float32:
        a = a.astype(np.float64)
    if a.dtype.kind in "US":
        return str(a)
    if a.dtype not in _NP2DT:
        raise TypeError(f"unsupported dtype {a.dtype}")
    return a.copy(order="C")


def write(path: str, entries: dict) -> None:
    """Create (or replace) a container holding `entries` (name -> value)."""
    items = [(_norm(k), _as_array(v)) for k, v in entries.items()]
    table_end = HEADER + ENTRY * len(items)
    off = (table_end + ALIGN - 1) // ALIGN * ALIGN
    recs, blobs = [], []
    for name, v in items:
        nb = name.encode()
        if len(nb) >= NAME_LEN:
            raise ValueError(f"name too long: {name}")
        if isinstance(v, Link):
            dt, ndim, shape, data = DT_LINK, 0, (0, 0, 0), v.filename.encode()
        elif isinstance(v, (str, bytes)):
            data = v.encode() if isinstance(v, str) else v
            dt, ndim, shape = DT_STR, 0, (0, 0, 0)
        else:
            if v.ndim > 3:
                raise ValueError(f"{name}: ndim {v.ndim} > 3")
            dt, ndim = _NP2DT[v.dtype], v.ndim
            shape = tuple(v.shape) + (0,) * (3 - v.ndim)
            data = v.tobytes(order="C")
        recs.append(struct.pack(_ENTRY_FMT, nb, dt, ndim, *shape, off, len(data)))
        blobs.append((off, data))
        off = (off + len(data) + ALIGN - 1) // ALIGN * ALIGN
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(MAGIC + struct.pack("<QQ", len(items), HEADER))
        f.write(b"\0" * (HEADER - 24))
        for r in recs:
            f.write(r)
        for o, data in blobs:
            f.seek(o)
            f.write(data)
        f.truncate(max(off, table_end))
    os.replace(tmp, path)


def _table(f):
    head = f.read(HEADER)
    if len(head) < 24 or head[:8] != MAGIC:
        raise ValueError("not a DQSF container")
    n, toff = struct.unpack("<QQ", head[8:24])
    f.seek(toff)
    out = {}
    for _ in range(n):
        nb, dt, ndim, s0, s1, s2, off, size = struct.unpack(_ENTRY_FMT, f.read(ENTRY))
        name = nb.rstrip(b"\0").decode()
        out[name] = (dt, ndim, (s0, s1, s2)[:ndim], off, size)
    return out


def _decode(f, rec):
    dt, ndim, shape, off, size = rec
    f.seek(off)
    raw = f.read(size)
    if dt == DT_LINK:
        return Link(raw.decode())
    if dt == DT_STR:
        return raw.decode()
    a = np.frombuffer(raw, dtype=_DT2NP[dt]).copy()
    return a.reshape(shape) if ndim else a.reshape(())


def read(path: str, resolve_links: bool = True) -> dict:
    """Read every entry; linked groups are merged in under their own names."""
    with open(path, "rb") as f:
        tab = _table(f)
        out = {name: _decode(f, rec) for name, rec in tab.items()}
    if resolve_links:
        base = os.path.dirname(os.path.abspath(path))
        for name, v in list(out.items()):
            if isinstance(v, Link):
                other = read(os.path.join(base, v.filename))
                for k, val in other.items():
                    if k == name or k.startswith(name + "/"):
                        out.setdefault(k, val)
    return out


def load(path: str, *names):
    """Return the named datasets, resolving links (like util.load_file)."""
    d = read(path)
    return [d[_norm(n)] for n in names]


def update(path: str, values: dict) -> None:
    """Overwrite existing datasets in place (same dtype and element count)."""
    with open(path, "r+b") as f:
        tab = _table(f)
        for name, v in values.items():
            name = _norm(name)
            if name not in tab:
                raise KeyError(f"{name} not in {path}")
            dt, ndim, shape, off, size = tab[name]
            if dt in (DT_LINK, DT_STR):
                raise TypeError(f"{name} is not an array")
            a = np.asarray(v, dtype=_DT2NP[dt]).copy(order="C")
            if a.nbytes != size:
                raise ValueError(f"{name}: {a.nbytes} bytes != {size}")
            f.seek(off)
            f.write(a.tobytes())
