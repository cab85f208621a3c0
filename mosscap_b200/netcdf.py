"""NetCDF classic-format files written and read without the netCDF library.

The layout follows Unidata's published "NetCDF File Format Specification":
a big-endian header (magic, record count, dimensions, global attributes,
variables with their type, size and file offset) followed by the data of
the fixed-size variables in definition order and then the records, each
record holding one slice of every record variable in definition order.

Three versions are written: CDF-1 (32-bit offsets), CDF-2 (64-bit offsets)
and CDF-5 (64-bit sizes and counts as well). :class:`NcWriter` picks the
smallest that holds the file unless one is asked for; the netCDF library
reads all three.

Only what the hydro output needs is covered: dimensions (one of them
unlimited), text / int / double attributes and double / int variables.
"""
from __future__ import annotations

import os
import struct
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

NC_BYTE, NC_CHAR, NC_SHORT, NC_INT, NC_FLOAT, NC_DOUBLE = 1, 2, 3, 4, 5, 6
_DTYPE = {NC_BYTE: np.dtype("i1"), NC_CHAR: np.dtype("S1"), NC_SHORT: np.dtype(">i2"),
          NC_INT: np.dtype(">i4"), NC_FLOAT: np.dtype(">f4"), NC_DOUBLE: np.dtype(">f8")}
_TAG_DIMENSION, _TAG_VARIABLE, _TAG_ATTRIBUTE = 0x0A, 0x0B, 0x0C


def _pad4(n: int) -> int:
    return (n + 3) & ~3


class _Fmt:
    """Field widths of one format version."""

    def __init__(self, version: int):
        if version not in (1, 2, 5):
            raise ValueError(f"unknown NetCDF classic version {version}")
        self.version = version
        self.count = ">Q" if version == 5 else ">I"    # NON_NEG: counts, lengths, dim ids, vsize, numrecs
        self.offset = ">I" if version == 1 else ">Q"   # OFFSET: begin of a variable

    def non_neg(self, v: int) -> bytes:
        return struct.pack(self.count, v)

    def off(self, v: int) -> bytes:
        return struct.pack(self.offset, v)

    def name(self, s: str) -> bytes:
        b = s.encode("utf-8")
        return self.non_neg(len(b)) + b + b"\0" * (_pad4(len(b)) - len(b))


def _att_value(value) -> Tuple[int, bytes, int]:
    if isinstance(value, str):
        b = value.encode("utf-8")
        return NC_CHAR, b, len(b)
    a = np.atleast_1d(np.asarray(value))
    if a.dtype.kind in "iu":
        return NC_INT, a.astype(">i4").tobytes(), a.size
    if a.dtype.kind == "f":
        return NC_DOUBLE, a.astype(">f8").tobytes(), a.size
    raise TypeError(f"attribute value of type {a.dtype} is not supported")


class _Var:
    def __init__(self, name: str, dims: Sequence[str], nc_type: int):
        self.name = name
        self.dims = list(dims)
        self.nc_type = nc_type
        self.shape: Tuple[int, ...] = ()
        self.is_record = False
        self.vsize = 0
        self.begin = 0


class NcWriter:
    """Writes one classic-format file: define dimensions, attributes and
    variables, call :meth:`end_def`, then write variables and records.

    ``NcWriter.append(path)`` reopens an existing file to add records."""

    def __init__(self, path: str, version: Optional[int] = None):
        self.path = path
        self.version = version
        self.dims: List[Tuple[str, Optional[int]]] = []
        self.gatts: Dict[str, Tuple[int, bytes, int]] = {}
        self.vars: List[_Var] = []
        self.numrecs = 0
        self.recsize = 0
        self._f = None
        self._fmt: Optional[_Fmt] = None
        self._numrecs_at = 4

    # ---- define mode -------------------------------------------------------
    def create_dim(self, name: str, size: Optional[int] = None) -> None:
        """A dimension; size None makes it the (single) unlimited one."""
        if any(d[0] == name for d in self.dims):
            raise ValueError(f"dimension {name!r} exists")
        if size is None and any(d[1] is None for d in self.dims):
            raise ValueError("a classic file has at most one unlimited dimension")
        self.dims.append((name, None if size is None else int(size)))

    def has_dim(self, name: str) -> bool:
        return any(d[0] == name for d in self.dims)

    def put_att(self, name: str, value) -> None:
        """A global attribute; setting an existing one replaces its value in
        place, as nc_put_att does."""
        self.gatts[name] = _att_value(value)

    def def_var(self, name: str, dims: Sequence[str], nc_type: int = NC_DOUBLE) -> None:
        for d in dims:
            if not self.has_dim(d):
                raise ValueError(f"variable {name!r}: unknown dimension {d!r}")
        self.vars.append(_Var(name, dims, nc_type))

    def _sizes(self) -> None:
        sizes = dict(self.dims)
        for v in self.vars:
            v.is_record = bool(v.dims) and sizes[v.dims[0]] is None
            if any(sizes[d] is None for d in v.dims[1:]):
                raise ValueError(f"variable {v.name!r}: only the first dimension may be unlimited")
            v.shape = tuple(sizes[d] for d in (v.dims[1:] if v.is_record else v.dims))
            v.vsize = _pad4(int(np.prod(v.shape, dtype=np.int64)) * _DTYPE[v.nc_type].itemsize)

    def _layout(self, version: int) -> int:
        fmt = _Fmt(version)
        self._sizes()
        header = len(self._header(fmt))
        off = header
        for v in self.vars:
            if not v.is_record:
                v.begin = off
                off += v.vsize
        self.recsize = 0
        for v in self.vars:
            if v.is_record:
                v.begin = off + self.recsize
                self.recsize += v.vsize
        return off

    def _fits(self, version: int) -> bool:
        self._sizes()
        if version != 5 and any(v.vsize > 0xFFFFFFFC for v in self.vars):
            return False
        fixed_end = self._layout(version)
        if version == 5:
            return True
        if version == 1:
            return all(v.begin <= 0x7FFFFFFF for v in self.vars) and fixed_end <= 0x7FFFFFFF
        return True

    def _header(self, fmt: _Fmt) -> bytes:
        out = [b"CDF" + bytes([fmt.version]), fmt.non_neg(self.numrecs)]
        if self.dims:
            out.append(struct.pack(">I", _TAG_DIMENSION) + fmt.non_neg(len(self.dims)))
            for name, size in self.dims:
                out.append(fmt.name(name) + fmt.non_neg(0 if size is None else size))
        else:
            out.append(struct.pack(">I", 0) + fmt.non_neg(0))
        if self.gatts:
            out.append(struct.pack(">I", _TAG_ATTRIBUTE) + fmt.non_neg(len(self.gatts)))
            for name, (t, data, n) in self.gatts.items():
                out.append(fmt.name(name) + struct.pack(">I", t) + fmt.non_neg(n) + data +
                           b"\0" * (_pad4(len(data)) - len(data)))
        else:
            out.append(struct.pack(">I", 0) + fmt.non_neg(0))
        if self.vars:
            dim_ids = {d[0]: k for k, d in enumerate(self.dims)}
            out.append(struct.pack(">I", _TAG_VARIABLE) + fmt.non_neg(len(self.vars)))
            for v in self.vars:
                out.append(fmt.name(v.name) + fmt.non_neg(len(v.dims)) +
                           b"".join(fmt.non_neg(dim_ids[d]) for d in v.dims) +
                           struct.pack(">I", 0) + fmt.non_neg(0) +      # no variable attributes
                           struct.pack(">I", v.nc_type) + fmt.non_neg(v.vsize) + fmt.off(v.begin))
        else:
            out.append(struct.pack(">I", 0) + fmt.non_neg(0))
        return b"".join(out)

    def end_def(self) -> None:
        """Fixes the layout and writes the header (and zero-filled data)."""
        if self.version is None:
            self.version = next(v for v in (1, 2, 5) if self._fits(v))
        elif not self._fits(self.version):
            raise ValueError(f"the file does not fit NetCDF classic version {self.version}")
        self._fmt = _Fmt(self.version)
        fixed_end = self._layout(self.version)
        self._f = open(self.path, "w+b")
        self._f.write(self._header(self._fmt))
        self._f.truncate(fixed_end)

    # ---- data mode ---------------------------------------------------------
    def _var(self, name: str) -> _Var:
        for v in self.vars:
            if v.name == name:
                return v
        raise KeyError(name)

    def write(self, name: str, data) -> None:
        """All of a fixed-size variable."""
        v = self._var(name)
        if v.is_record:
            raise ValueError(f"{name!r} is a record variable: use write_record")
        a = np.asarray(data, dtype=_DTYPE[v.nc_type])
        if a.shape != v.shape:
            raise ValueError(f"{name!r}: shape {a.shape} != {v.shape}")
        a = np.ascontiguousarray(a).reshape(v.shape)
        self._f.seek(v.begin)
        self._write_array(a)

    def write_record(self, name: str, index: int, data) -> None:
        """Record `index` of a record variable; the record count grows to
        cover it."""
        v = self._var(name)
        if not v.is_record:
            raise ValueError(f"{name!r} is not a record variable")
        a = np.asarray(data, dtype=_DTYPE[v.nc_type])
        if a.shape != v.shape:
            raise ValueError(f"{name!r}: shape {a.shape} != {v.shape}")
        a = np.ascontiguousarray(a).reshape(v.shape)
        self._f.seek(v.begin + index * self.recsize)
        self._write_array(a)
        if index + 1 > self.numrecs:
            self.numrecs = index + 1
            # every record is complete on disk (zeros where nothing was written)
            needed = self._rec0() + self.numrecs * self.recsize
            if self._f.seek(0, os.SEEK_END) < needed:
                self._f.truncate(needed)
            self._f.seek(self._numrecs_at)
            self._f.write(self._fmt.non_neg(self.numrecs))

    def _rec0(self) -> int:
        return min(x.begin for x in self.vars if x.is_record)

    def _write_array(self, a: np.ndarray) -> None:
        flat = a.reshape(-1)
        step = max(1, (64 << 20) // max(a.itemsize, 1))
        for s in range(0, flat.size, step):
            self._f.write(flat[s:s + step].tobytes())
        pad = _pad4(a.nbytes) - a.nbytes
        if pad:
            self._f.write(b"\0" * pad)

    def close(self) -> None:
        if self._f is not None:
            self._f.flush()
            self._f.close()
            self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @classmethod
    def append(cls, path: str) -> "NcWriter":
        """Reopens a file written by this class (or any classic file with
        the supported types) to add records."""
        r = read(path)
        w = cls(path, r.version)
        w.dims = list(r.dims)
        w.gatts = {k: _att_value(v) for k, v in r.attrs.items()}
        for name, dims, t, _, _ in r.var_defs:
            w.def_var(name, dims, t)
        w._fmt = _Fmt(r.version)
        w._layout(r.version)
        for v, (_, _, _, vsize, begin) in zip(w.vars, r.var_defs):
            if v.begin != begin or v.vsize != vsize:
                raise ValueError(f"{path}: layout differs from this writer's for {v.name!r}")
        w.numrecs = r.numrecs
        w._f = open(path, "r+b")
        return w


class NcFile:
    """What :func:`read` returns: version, record count, dimensions (size
    None for the unlimited one), global attributes and the variables'
    data (record variables with the record dimension first)."""

    def __init__(self):
        self.version = 1
        self.numrecs = 0
        self.dims: List[Tuple[str, Optional[int]]] = []
        self.attrs: Dict[str, object] = {}
        self.var_defs: List[Tuple[str, List[str], int, int, int]] = []
        self.variables: Dict[str, np.ndarray] = {}
        self.var_dims: Dict[str, List[str]] = {}


def read(path: str, data: bool = True) -> NcFile:
    """Parses a classic-format file (CDF-1, CDF-2 or CDF-5)."""
    with open(path, "rb") as f:
        buf = f.read() if data else f.read(1 << 20)
    if buf[:3] != b"CDF" or buf[3] not in (1, 2, 5):
        raise ValueError(f"{path}: not a NetCDF classic file")
    fmt = _Fmt(buf[3])
    out = NcFile()
    out.version = buf[3]
    pos = 4

    def take(fmt_str):
        nonlocal pos
        (v,) = struct.unpack_from(fmt_str, buf, pos)
        pos += struct.calcsize(fmt_str)
        return v

    def name():
        nonlocal pos
        n = take(fmt.count)
        s = buf[pos:pos + n].decode("utf-8")
        pos += _pad4(n)
        return s

    out.numrecs = take(fmt.count)
    tag, n = take(">I"), take(fmt.count)
    for _ in range(n if tag == _TAG_DIMENSION else 0):
        nm = name()
        size = take(fmt.count)
        out.dims.append((nm, None if size == 0 else size))

    def atts():
        nonlocal pos
        res = {}
        tag, n = take(">I"), take(fmt.count)
        for _ in range(n if tag == _TAG_ATTRIBUTE else 0):
            nm = name()
            t = take(">I")
            cnt = take(fmt.count)
            dt = _DTYPE[t]
            raw = buf[pos:pos + cnt * dt.itemsize]
            pos += _pad4(cnt * dt.itemsize)
            res[nm] = raw.decode("utf-8") if t == NC_CHAR else np.frombuffer(raw, dt).astype(dt.newbyteorder("="))
        return res

    out.attrs = atts()
    tag, n = take(">I"), take(fmt.count)
    sizes = [d[1] for d in out.dims]
    for _ in range(n if tag == _TAG_VARIABLE else 0):
        nm = name()
        nd = take(fmt.count)
        ids = [take(fmt.count) for _ in range(nd)]
        atts()
        t = take(">I")
        vsize = take(fmt.count)
        begin = take(fmt.offset)
        dims = [out.dims[k][0] for k in ids]
        out.var_defs.append((nm, dims, t, vsize, begin))
        out.var_dims[nm] = dims
    recsize = sum(vs for (_, dims, _, vs, _) in out.var_defs
                  if dims and dict(out.dims)[dims[0]] is None)
    if data:
        for nm, dims, t, vsize, begin in out.var_defs:
            dt = _DTYPE[t]
            is_rec = bool(dims) and dict(out.dims)[dims[0]] is None
            shape = [dict(out.dims)[d] for d in (dims[1:] if is_rec else dims)]
            count = int(np.prod(shape, dtype=np.int64))
            if is_rec:
                recs = [np.frombuffer(buf, dt, count, begin + r * recsize).reshape(shape)
                        for r in range(out.numrecs)]
                arr = np.stack(recs) if recs else np.zeros([0] + shape, dt)
            else:
                arr = np.frombuffer(buf, dt, count, begin).reshape(shape)
            out.variables[nm] = arr.astype(dt.newbyteorder("="))
    return out
