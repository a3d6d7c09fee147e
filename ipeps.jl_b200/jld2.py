"""Reader for the JLD2 files iPEPS.jl writes (gs.jld2, basis.jld2, es_*.jld2).

The reference saves its results with JLD2.jldsave (src/optimize/optim_gs.jl:36,
src/optimize/optim_es.jl:70,146); JLD2 files are HDF5 files (superblock
version 2 or 3 after a 512-byte user block).  This module reads the plain
numeric datasets of such files without an HDF5 library: Float64, Float32,
Int64/Int32 and ComplexF64 arrays and scalars, in Julia (column-major) order,
from groups of any depth, and Julia structs whose fields are all references
(the saved CTMTensors: a dict of its fields) or arrays of references
(Vector{Matrix}: a list).  Datasets of other types (the Optim state, Dict
fields) are reported as Unsupported.

    data = load("simulation/test_test_D2_X32/es_0.1_0.jld2")
    effH = data["effH"]            # (31, 31) complex128, Julia layout

HDF5 pieces handled: superblock v2/v3, version-2 object headers with
continuation blocks, link messages (hard links), dataspace, datatype (fixed
point, floating point, and the two-member compound JLD2 uses for Complex,
shared through committed datatypes), compact and contiguous data layouts.
"""
from __future__ import annotations

import struct
from typing import Any, Dict, List, Optional, Tuple

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"


class JLD2Error(ValueError):
    pass


class Unsupported:
    """Placeholder for a dataset this reader does not decode."""

    def __init__(self, name: str, why: str):
        self.name, self.why = name, why

    def __repr__(self):
        return f"Unsupported({self.name!r}: {self.why})"


class _File:
    def __init__(self, data: bytes):
        self.d = data
        off = 0
        while off < len(data) and data[off:off + 8] != _SIG:
            off = 512 if off == 0 else off * 2
        if off >= len(data):
            raise JLD2Error("no HDF5 superblock found")
        ver = data[off + 8]
        if ver not in (2, 3):
            raise JLD2Error(f"HDF5 superblock version {ver} not supported (JLD2 writes 2 or 3)")
        so, sl = data[off + 9], data[off + 10]
        if so != 8 or sl != 8:
            raise JLD2Error("only 8-byte offsets and lengths are supported")
        self.base, _ext, _eof, self.root = struct.unpack_from("<QQQQ", data, off + 12)

    # ------------------------------------------------------------ object headers
    def messages(self, addr: int) -> List[Tuple[int, int, bytes]]:
        d = self.d
        a = self.base + addr
        if d[a:a + 4] != b"OHDR":
            raise JLD2Error(f"no version-2 object header at {addr:#x}")
        flags = d[a + 5]
        p = a + 6
        if flags & 0x20:
            p += 16  # access/modification/change/birth times
        if flags & 0x10:
            p += 4   # attribute phase change values
        sz = 1 << (flags & 3)
        n = int.from_bytes(d[p:p + sz], "little")
        p += sz
        out: List[Tuple[int, int, bytes]] = []
        self._read_msgs(p, p + n, flags, out)
        return out

    def _read_msgs(self, p: int, end: int, hflags: int, out: list):
        d = self.d
        while p + 4 <= end:
            t = d[p]
            size = struct.unpack_from("<H", d, p + 1)[0]
            mflags = d[p + 3]
            p += 4
            if hflags & 0x04:
                p += 2  # creation order
            body = d[p:p + size]
            p += size
            if t == 0x10:  # continuation: OCHK block
                caddr, clen = struct.unpack_from("<QQ", body, 0)
                c = self.base + caddr
                if d[c:c + 4] != b"OCHK":
                    raise JLD2Error("bad continuation block")
                self._read_msgs(c + 4, c + clen - 4, hflags, out)
            else:
                out.append((t, mflags, body))

    # ------------------------------------------------------------ messages
    @staticmethod
    def links(msgs) -> Dict[str, int]:
        res = {}
        for t, _f, b in msgs:
            if t != 0x06:
                continue
            ver, fl = b[0], b[1]
            if ver != 1:
                raise JLD2Error("link message version")
            p = 2
            ltype = 0
            if fl & 0x08:
                ltype = b[p]
                p += 1
            if fl & 0x04:
                p += 8
            if fl & 0x10:
                p += 1
            ls = 1 << (fl & 3)
            ln = int.from_bytes(b[p:p + ls], "little")
            p += ls
            name = b[p:p + ln].decode("utf-8")
            p += ln
            if ltype == 0:
                res[name] = struct.unpack_from("<Q", b, p)[0]
        return res

    def datatype(self, msgs) -> Tuple[Optional[np.dtype], str]:
        for t, f, b in msgs:
            if t != 0x03:
                continue
            if f & 0x02:  # shared: committed datatype elsewhere
                addr = struct.unpack_from("<Q", b, 2)[0]
                return self.datatype(self.messages(addr))
            return self._parse_dtype(b)
        return None, "no datatype message"

    def _parse_dtype(self, b: bytes) -> Tuple[Optional[np.dtype], str]:
        cls = b[0] & 0x0F
        bits0 = b[1]
        size = struct.unpack_from("<I", b, 4)[0]
        if cls in (0, 1) and bits0 & 1:
            return None, "big-endian data"
        if cls == 0:  # fixed point
            signed = bool(bits0 & 0x08)
            return np.dtype(("i" if signed else "u") + str(size)).newbyteorder("<"), ""
        if cls == 1:  # floating point
            if size not in (4, 8):
                return None, f"float of {size} bytes"
            return np.dtype("<f" + str(size)), ""
        if cls == 6:  # compound: JLD2 writes Complex{T} as {re, im}
            nmem = b[1] | (b[2] << 8)
            ver = b[0] >> 4
            p = 8
            mems = []
            for _ in range(nmem):
                e = b.index(b"\x00", p)
                name = b[p:e].decode()
                p = e + 1
                if ver < 3:
                    p = 8 + ((p - 8 + 7) // 8) * 8
                if ver >= 3:
                    osz = 1 if size < 256 else 2 if size < 65536 else 4
                    off = int.from_bytes(b[p:p + osz], "little")
                    p += osz
                else:
                    off = struct.unpack_from("<I", b, p)[0]
                    p += 4
                    if ver == 1:
                        p += 28
                if (b[p] & 0x0F) not in (0, 1):
                    return None, "compound type with non-numeric members"
                sub, why = self._parse_dtype(b[p:])
                msz = struct.unpack_from("<I", b, p + 4)[0]
                p += self._dtype_len(b[p:])
                mems.append((name, off, sub, msz))
            if (len(mems) == 2 and [m[0] for m in mems] == ["re", "im"] and mems[0][2] is not None
                    and mems[0][2] == mems[1][2] and mems[0][2].kind == "f"):
                return np.dtype("<c" + str(2 * mems[0][3])), ""
            return None, "compound type " + ",".join(m[0] for m in mems)
        return None, f"datatype class {cls}"

    @staticmethod
    def _dtype_len(b: bytes) -> int:
        cls = b[0] & 0x0F
        if cls == 0:
            return 8 + 4
        if cls == 1:
            return 8 + 12
        raise JLD2Error("nested compound members are not supported")

    @staticmethod
    def dataspace(msgs) -> Optional[Tuple[int, ...]]:
        for t, _f, b in msgs:
            if t != 0x01:
                continue
            ver, rank, fl = b[0], b[1], b[2]
            if ver == 1:
                p = 8
            else:
                if b[3] == 2:  # null dataspace
                    return None
                p = 4
            return tuple(struct.unpack_from("<Q", b, p + 8 * i)[0] for i in range(rank))
        return None

    def raw(self, msgs) -> Optional[bytes]:
        for t, _f, b in msgs:
            if t != 0x08:
                continue
            ver, cls = b[0], b[1]
            if ver < 3:
                raise JLD2Error("data layout message version < 3")
            if cls == 0:
                n = struct.unpack_from("<H", b, 2)[0]
                return b[4:4 + n]
            if cls == 1:
                addr, size = struct.unpack_from("<QQ", b, 2)
                if addr == 0xFFFFFFFFFFFFFFFF:
                    return b""
                a = self.base + addr
                return self.d[a:a + size]
            raise JLD2Error("chunked (compressed) datasets are not supported")
        return None


def _ref_members(f: _File, msgs) -> Optional[List[str]]:
    """Member names of a compound datatype whose members are all object
    references (a Julia struct of arrays, e.g. the saved CTMTensors)."""
    for t, fl, b in msgs:
        if t != 0x03:
            continue
        if fl & 0x02:
            return _ref_members(f, f.messages(struct.unpack_from("<Q", b, 2)[0]))
        if (b[0] & 0x0F) != 6 or (b[0] >> 4) < 3:
            return None
        nmem = b[1] | (b[2] << 8)
        size = struct.unpack_from("<I", b, 4)[0]
        osz = 1 if size < 256 else 2 if size < 65536 else 4
        p, names = 8, []
        for _ in range(nmem):
            e = b.index(b"\x00", p)
            names.append(b[p:e].decode())
            p = e + 1 + osz
            if (b[p] & 0x0F) != 7:
                return None
            p += 8  # reference datatype: header only
        return names
    return None


def _is_reference(f: _File, msgs) -> bool:
    for t, fl, b in msgs:
        if t == 0x03:
            if fl & 0x02:
                return _is_reference(f, f.messages(struct.unpack_from("<Q", b, 2)[0]))
            return (b[0] & 0x0F) == 7
    return False


def _dataset(f: _File, addr: int, name: str, depth: int = 0) -> Any:
    if depth > 8:
        return Unsupported(name, "reference chain too deep")
    msgs = f.messages(addr)
    shape = f.dataspace(msgs)
    raw = f.raw(msgs)
    if raw is None:
        return Unsupported(name, "no data")
    if shape is None:
        return None  # null dataspace (an empty Julia object)
    n = int(np.prod(shape)) if shape else 1
    members = _ref_members(f, msgs)
    if members is not None and n == 1:
        refs = struct.unpack_from("<%dQ" % len(members), raw, 0)
        return {m: _dataset(f, r, name + "." + m, depth + 1) for m, r in zip(members, refs)}
    if _is_reference(f, msgs):
        refs = struct.unpack_from("<%dQ" % n, raw, 0)
        return [_dataset(f, r, f"{name}[{i}]", depth + 1) for i, r in enumerate(refs)]
    dt, why = f.datatype(msgs)
    if dt is None:
        return Unsupported(name, why)
    arr = np.frombuffer(raw, dtype=dt, count=n)
    if len(shape) == 0:
        return arr[0].item()
    # HDF5 dims are stored reversed: the raw bytes are in Julia's column-major order
    return arr.reshape(tuple(reversed(shape)), order="F").copy()


def _walk(f: _File, addr: int, prefix: str, out: Dict[str, Any]):
    msgs = f.messages(addr)
    kinds = {t for t, _f, _b in msgs}
    if 0x08 in kinds:  # dataset
        name = prefix.rstrip("/")
        out[name] = _dataset(f, addr, name)
        return
    for name, a in f.links(msgs).items():
        if name == "_types":
            continue
        _walk(f, a, prefix + name + "/", out)


def load(path: str) -> Dict[str, Any]:
    """All datasets of a JLD2 file: name (groups joined with '/') -> numpy
    array (Julia shape and order), Python scalar, or Unsupported."""
    with open(path, "rb") as fh:
        f = _File(fh.read())
    out: Dict[str, Any] = {}
    _walk(f, f.root, "", out)
    return out
