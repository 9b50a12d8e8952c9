"""Read classic-format HDF5 result files without h5py.

Supports what the reference's result layout needs (include/wos/hdf5_io.hpp):
superblock version 0/1, symbol-table groups (v1 B-trees, symbol-table nodes,
local heaps), version-1 object headers (with continuation blocks), simple or
scalar dataspaces, IEEE floating-point and fixed-point little-endian
datatypes, and contiguous or compact data layouts.  A user block (the file
signature at 512, 1024, ... bytes) is accepted.

    >>> from walk_on_spheres_b200 import h5lite
    >>> f = h5lite.read("wos.h5")          # {"/mean": ndarray, "/metadata/seed": ...}
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5FormatError(ValueError):
    pass


class _File:
    def __init__(self, data: bytes):
        self.d = data
        self.base = self._find_signature()
        sb = self.base
        version = data[sb + 8]
        if version not in (0, 1):
            raise H5FormatError(f"superblock version {version} not supported")
        self.so, self.sl = data[sb + 13], data[sb + 14]
        if (self.so, self.sl) != (8, 8):
            raise H5FormatError("only 8-byte offsets and lengths are supported")
        p = sb + 24 + (4 if version == 1 else 0)
        self.base_addr, _, self.eof, _ = struct.unpack_from("<QQQQ", data, p)
        root = p + 32
        _, self.root_header, _, _, _, _ = struct.unpack_from("<QQIIQQ", data, root)

    def _find_signature(self) -> int:
        off = 0
        while off + 8 <= len(self.d):
            if self.d[off:off + 8] == SIGNATURE:
                return off
            off = 512 if off == 0 else off * 2
        raise H5FormatError("not an HDF5 file")

    def at(self, addr: int) -> int:
        return self.base + addr

    # ---------------------------------------------------------- object headers
    def messages(self, addr: int) -> list[tuple[int, bytes]]:
        p = self.at(addr)
        version, _, n, _, size = struct.unpack_from("<BBHII", self.d, p)
        if version != 1:
            raise H5FormatError(f"object header version {version} not supported")
        chunks = [(p + 16, size)]
        out = []
        while chunks and len(out) < n:
            q, size = chunks.pop(0)
            end = q + size
            while q + 8 <= end and len(out) < n:
                mtype, msize, _ = struct.unpack_from("<HHB", self.d, q)
                body = self.d[q + 8:q + 8 + msize]
                if mtype == 0x0010:  # continuation
                    caddr, clen = struct.unpack_from("<QQ", body, 0)
                    chunks.append((self.at(caddr), clen))
                out.append((mtype, body))
                q += 8 + msize
        return out

    # ---------------------------------------------------------- groups
    def heap_name(self, heap_addr: int, offset: int) -> str:
        p = self.at(heap_addr)
        if self.d[p:p + 4] != b"HEAP":
            raise H5FormatError("bad local heap")
        _, _, data_addr = struct.unpack_from("<QQQ", self.d, p + 8)
        q = self.at(data_addr) + offset
        e = self.d.index(b"\x00", q)
        return self.d[q:e].decode()

    def group_links(self, btree_addr: int, heap_addr: int) -> list[tuple[str, int]]:
        p = self.at(btree_addr)
        if self.d[p:p + 4] != b"TREE":
            raise H5FormatError("bad group B-tree")
        node_type, level, used = self.d[p + 4], self.d[p + 5], struct.unpack_from("<H", self.d, p + 6)[0]
        if node_type != 0:
            raise H5FormatError("not a group B-tree")
        links = []
        q = p + 24
        for i in range(used):
            child = struct.unpack_from("<Q", self.d, q + 8 + 16 * i)[0]
            if level > 0:
                links.extend(self.group_links(child, heap_addr))
                continue
            s = self.at(child)
            if self.d[s:s + 4] != b"SNOD":
                raise H5FormatError("bad symbol table node")
            nsym = struct.unpack_from("<H", self.d, s + 6)[0]
            for k in range(nsym):
                name_off, header = struct.unpack_from("<QQ", self.d, s + 8 + 40 * k)
                links.append((self.heap_name(heap_addr, name_off), header))
        return links

    # ---------------------------------------------------------- datasets
    @staticmethod
    def dtype(body: bytes) -> np.dtype:
        cls_ver = body[0]
        cls = cls_ver & 0x0F
        bits = body[1] | (body[2] << 8) | (body[3] << 16)
        size = struct.unpack_from("<I", body, 4)[0]
        if bits & 1:
            raise H5FormatError("big-endian data not supported")
        if cls == 1:
            return np.dtype(f"<f{size}")
        if cls == 0:
            return np.dtype(f"<{'i' if bits & 0x08 else 'u'}{size}")
        raise H5FormatError(f"datatype class {cls} not supported")

    @staticmethod
    def shape(body: bytes) -> tuple:
        version, rank = body[0], body[1]
        off = 8 if version == 1 else 4
        if version == 2 and body[3] == 0:
            return ()
        return tuple(struct.unpack_from("<Q", body, off + 8 * i)[0] for i in range(rank))

    def dataset(self, msgs) -> np.ndarray:
        dt = shape = layout = None
        for t, b in msgs:
            if t == 0x0003:
                dt = self.dtype(b)
            elif t == 0x0001:
                shape = self.shape(b)
            elif t == 0x0008:
                layout = b
        if dt is None or shape is None or layout is None:
            raise H5FormatError("dataset without datatype, dataspace or layout")
        n = int(np.prod(shape)) if shape else 1
        version = layout[0]
        if version == 3:
            cls = layout[1]
            if cls == 1:
                addr = struct.unpack_from("<Q", layout, 2)[0]
            elif cls == 0:
                size = struct.unpack_from("<H", layout, 2)[0]
                raw = layout[4:4 + size]
                return np.frombuffer(raw, dtype=dt, count=n).reshape(shape).copy()
            else:
                raise H5FormatError("chunked layout not supported")
        elif version in (1, 2):
            if layout[2] != 1:
                raise H5FormatError("only contiguous version-1/2 layouts are supported")
            addr = struct.unpack_from("<Q", layout, 8)[0]
        else:
            raise H5FormatError(f"layout version {version} not supported")
        if addr == UNDEF:
            return np.zeros(shape, dtype=dt)
        p = self.at(addr)
        return np.frombuffer(self.d, dtype=dt, count=n, offset=p).reshape(shape).copy()

    def walk(self, header: int, prefix: str, out: dict):
        msgs = self.messages(header)
        stab = [b for t, b in msgs if t == 0x0011]
        if stab:
            btree, heap = struct.unpack_from("<QQ", stab[0], 0)
            for name, child in self.group_links(btree, heap):
                self.walk(child, f"{prefix}/{name}", out)
        else:
            out[prefix] = self.dataset(msgs)


def read(path: str | Path) -> dict:
    """Every dataset of the file by full path ("/mean", "/metadata/seed", ...).
    Scalars come back as 0-d arrays."""
    f = _File(Path(path).read_bytes())
    out: dict = {}
    f.walk(f.root_header, "", out)
    return out
