"""Initial conditions from the reference's HDF5 snapshot files, without an
HDF5 library: a small reader of the file format's original (version 0/1
superblock) layout, the one the reference's inputs use.

readHDFFile (SPH/hdfHandler/hdfHandler.cpp:12-136) opens group "PartType0"
and reads Coordinates and Velocities (N x 3) and Densities,
InternalEnergies, Masses, Pressures, SmoothingLengths (N) as float, and
MaterialIDs (N) as int32, converting from the stored types (the demo file
stores coordinates as FP64).  `read_ic` returns the same fields, converted the
same way (FP64 -> FP32 by round to nearest), as the initial-conditions dict
that Compute takes.

Supported: superblock versions 0 and 1 with 8-byte offsets and lengths;
groups as symbol tables (v1 B-trees of symbol-table nodes and a local heap);
version-1 object headers with continuation blocks; dataspace messages v1/v2;
little-endian fixed-point and IEEE floating-point datatypes; contiguous and
compact data layouts (v1-v3).  Anything else (chunked or filtered data, the
newer superblocks and object headers) raises UnsupportedHDF5.
"""
from __future__ import annotations

import struct

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"


class UnsupportedHDF5(ValueError):
    pass


class _File:
    def __init__(self, data: bytes):
        self.d = data
        if data[:8] != SIGNATURE:
            raise UnsupportedHDF5("not an HDF5 file (no signature at offset 0)")
        sb = data[8]
        if sb not in (0, 1):
            raise UnsupportedHDF5(f"superblock version {sb} is not supported")
        if data[13] != 8 or data[14] != 8:
            raise UnsupportedHDF5("only 8-byte offsets and lengths are supported")
        base = 24 + (4 if sb == 1 else 0)  # v1 adds indexed-storage K + reserved
        # base address, free space, end of file, driver info, then the root entry
        root = base + 32
        self.root = self._entry(root)

    # little-endian readers
    def u8(self, o):
        return self.d[o]

    def u16(self, o):
        return struct.unpack_from("<H", self.d, o)[0]

    def u32(self, o):
        return struct.unpack_from("<I", self.d, o)[0]

    def u64(self, o):
        return struct.unpack_from("<Q", self.d, o)[0]

    def _entry(self, o) -> dict:
        """Symbol table entry: name offset, object header, cache type, scratch."""
        e = dict(name_off=self.u64(o), header=self.u64(o + 8), cache=self.u32(o + 16))
        if e["cache"] == 1:
            e["btree"], e["heap"] = self.u64(o + 24), self.u64(o + 32)
        return e

    def _heap_string(self, heap: int, off: int) -> str:
        if self.d[heap:heap + 4] != b"HEAP":
            raise UnsupportedHDF5("bad local heap")
        s = self.u64(heap + 24) + off
        return self.d[s:self.d.index(b"\0", s)].decode()

    def messages(self, addr: int) -> list:
        """(type, body offset, body size) of a version-1 object header."""
        if self.u8(addr) != 1:
            raise UnsupportedHDF5(f"object header version {self.u8(addr)} at {addr:#x} is not supported")
        nmsg = self.u16(addr + 2)
        blocks = [(addr + 16, self.u32(addr + 8))]
        out = []
        while blocks and len(out) < nmsg:
            a, size = blocks.pop(0)
            p = a
            while p + 8 <= a + size and len(out) < nmsg:
                t, ms = self.u16(p), self.u16(p + 2)
                body = p + 8
                out.append((t, body, ms))
                if t == 0x10:  # continuation
                    blocks.append((self.u64(body), self.u64(body + 8)))
                p = body + ms
        return out

    def group(self, btree: int, heap: int) -> dict:
        """name -> symbol table entry of a symbol-table group."""
        out = {}
        if self.d[btree:btree + 4] != b"TREE" or self.u8(btree + 4) != 0:
            raise UnsupportedHDF5("bad group B-tree")
        level, used = self.u8(btree + 5), self.u16(btree + 6)
        p = btree + 24
        for _ in range(used):
            child = self.u64(p + 8)
            p += 16
            if level > 0:
                out.update(self.group(child, heap))
                continue
            if self.d[child:child + 4] != b"SNOD":
                raise UnsupportedHDF5("bad symbol table node")
            q = child + 8
            for _ in range(self.u16(child + 6)):
                e = self._entry(q)
                out[self._heap_string(heap, e["name_off"])] = e
                q += 40
        return out

    def subgroup(self, entry: dict) -> dict:
        if entry.get("cache") == 1:
            return self.group(entry["btree"], entry["heap"])
        for t, body, _ in self.messages(entry["header"]):
            if t == 0x11:  # symbol table message
                return self.group(self.u64(body), self.u64(body + 8))
        raise UnsupportedHDF5("object is not a symbol-table group")

    def dataset(self, entry: dict) -> np.ndarray:
        shape = dtype = data = None
        for t, b, ms in self.messages(entry["header"]):
            if t == 0x01:  # dataspace
                ver, rank = self.u8(b), self.u8(b + 1)
                first = b + (8 if ver == 1 else 4)
                shape = tuple(self.u64(first + 8 * k) for k in range(rank))
            elif t == 0x03:  # datatype
                cls, ver_cls = self.u8(b) & 0x0F, self.u8(b) >> 4
                bits, size = self.u8(b + 1), self.u32(b + 4)
                if ver_cls not in (1, 2, 3) or bits & 0x01:
                    raise UnsupportedHDF5("only little-endian datatypes are supported")
                if cls == 0:
                    dtype = np.dtype(("<i" if bits & 0x08 else "<u") + str(size))
                elif cls == 1 and size in (4, 8):
                    dtype = np.dtype("<f" + str(size))
                else:
                    raise UnsupportedHDF5(f"datatype class {cls} size {size} is not supported")
            elif t == 0x08:  # data layout
                ver = self.u8(b)
                if ver == 3:
                    lc = self.u8(b + 1)
                    if lc == 1:
                        data = ("contiguous", self.u64(b + 2), self.u64(b + 10))
                    elif lc == 0:
                        data = ("compact", b + 4, self.u16(b + 2))
                    else:
                        raise UnsupportedHDF5("chunked datasets are not supported")
                elif ver in (1, 2):
                    rank, lc = self.u8(b + 1), self.u8(b + 2)
                    if lc == 1:
                        data = ("contiguous", self.u64(b + 8), None)
                    elif lc == 0:
                        o = b + 8 + 4 * rank
                        data = ("compact", o + 4, self.u32(o))
                    else:
                        raise UnsupportedHDF5("chunked datasets are not supported")
                else:
                    raise UnsupportedHDF5(f"layout message version {ver} is not supported")
            elif t == 0x0B:  # filter pipeline
                raise UnsupportedHDF5("filtered datasets are not supported")
        if shape is None or dtype is None or data is None:
            raise UnsupportedHDF5("dataset without dataspace, datatype or layout")
        count = int(np.prod(shape)) if shape else 1
        nbytes = count * dtype.itemsize
        kind, addr, size = data
        if kind == "contiguous" and addr == 0xFFFFFFFFFFFFFFFF:
            return np.zeros(shape, dtype)  # never written
        if size is not None and size < nbytes:
            raise UnsupportedHDF5("dataset storage is smaller than its dataspace")
        return np.frombuffer(self.d, dtype=dtype, count=count, offset=addr).reshape(shape).copy()


def read_group(path: str, group: str = "PartType0") -> dict:
    """Every dataset of one top-level group, in its stored type."""
    with open(path, "rb") as f:
        h = _File(f.read())
    top = h.subgroup(h.root)
    if group not in top:
        raise KeyError(f"{path}: no group {group!r} (has {sorted(top)})")
    g = h.subgroup(top[group])
    return {name: h.dataset(e) for name, e in g.items() if e.get("cache") != 1}


def read_ic(path: str) -> dict:
    """readHDFFile (hdfHandler.cpp:12-136): the PartType0 fields as the
    initial-conditions dict of Compute -- float32 (FP64 rounded to nearest),
    material ids int32."""
    g = read_group(path, "PartType0")

    def vec3(name):
        a = g[name]
        if a.ndim != 2 or a.shape[1] != 3:
            raise ValueError(f"dataset {name} does not have 3 columns")
        return a.astype(np.float32)

    def scalar(name):
        return g[name].reshape(-1).astype(np.float32)

    ic = dict(pos=vec3("Coordinates"), vel=vec3("Velocities"), rho=scalar("Densities"),
              u=scalar("InternalEnergies"), mass=scalar("Masses"), pressure=scalar("Pressures"),
              h=scalar("SmoothingLengths"), material=g["MaterialIDs"].reshape(-1).astype(np.int32))
    ic["n"] = int(ic["pos"].shape[0])
    for k, v in ic.items():
        if k != "n" and v.shape[0] != ic["n"]:
            raise ValueError(f"dataset for {k} has {v.shape[0]} rows, Coordinates has {ic['n']}")
    return ic
