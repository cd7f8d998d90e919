"""HDF5 files without the HDF5 library: a reader and a writer of the subset PyLith's output uses.

Written from the published HDF5 File Format Specification (version 3.0). The reader handles
superblocks 0-3, object headers 1 and 2 (with continuation blocks), old-style groups (symbol
tables: version-1 group B-trees, symbol-table nodes, local heaps) and new-style compact groups
(link messages), simple and scalar dataspaces, fixed-point, floating-point and string datatypes
(fixed length, and variable length through the global heap), contiguous, compact and chunked
layouts (version-1 chunk B-trees) with the deflate, shuffle and Fletcher-32 filters, and
attributes. The writer produces structures the HDF5 library itself writes: superblock 0,
version-1 object headers, compact new-style groups (link messages, as in files made with link
creation order tracked), contiguous datasets, chunked datasets that grow along their first
dimension (one chunk per step, version-1 chunk B-tree) and version-1 attributes.
"""
from __future__ import annotations

import struct
import zlib
from typing import Dict, List, Optional, Tuple

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF

# object header message types
MSG_NIL, MSG_DATASPACE, MSG_LINK_INFO, MSG_DATATYPE = 0x0, 0x1, 0x2, 0x3
MSG_FILL_OLD, MSG_FILL, MSG_LINK, MSG_EXTERNAL, MSG_LAYOUT = 0x4, 0x5, 0x6, 0x7, 0x8
MSG_GROUP_INFO, MSG_FILTERS, MSG_ATTRIBUTE, MSG_CONTINUATION = 0xA, 0xB, 0xC, 0x10
MSG_SYMBOL_TABLE, MSG_MTIME, MSG_ATTR_INFO, MSG_REFCOUNT = 0x11, 0x12, 0x15, 0x16

FILTER_DEFLATE, FILTER_SHUFFLE, FILTER_FLETCHER32 = 1, 2, 3


class H5FormatError(ValueError):
    """The file is not HDF5, or uses a part of the format this module does not read."""


def _pad8(n: int) -> int:
    return (n + 7) & ~7


# ----------------------------------------------------------------------------------------------
# Reader
# ----------------------------------------------------------------------------------------------


class _Datatype:
    """A parsed datatype message: numpy dtype for numbers and fixed strings, or vlen string."""

    def __init__(self, cls: int, size: int, dtype: Optional[np.dtype], vlen_string: bool = False):
        self.cls, self.size, self.dtype, self.vlen_string = cls, size, dtype, vlen_string


class _Object:
    """Messages of one object header, by type (in header order)."""

    def __init__(self, addr: int):
        self.addr = addr
        self.messages: List[Tuple[int, bytes]] = []

    def first(self, mtype: int) -> Optional[bytes]:
        for t, d in self.messages:
            if t == mtype:
                return d
        return None

    def all(self, mtype: int) -> List[bytes]:
        return [d for t, d in self.messages if t == mtype]


class H5File:
    """Read-only view of an HDF5 file held in memory.

    Paths are absolute ("/geometry/vertices"). `keys(group)` lists a group's links in name
    order, `dataset(path)` returns the data as a numpy array (fixed strings as bytes, variable
    strings as a list of str), `attrs(path)` the attributes of a group or dataset."""

    def __init__(self, path_or_bytes):
        self.path = None
        if isinstance(path_or_bytes, (bytes, bytearray)):
            self.buf = bytes(path_or_bytes)
        else:
            self.path = str(path_or_bytes)
            with open(path_or_bytes, "rb") as f:
                self.buf = f.read()
        self._objects: Dict[int, _Object] = {}
        self._superblock()

    # -- primitives ----------------------------------------------------------------------------
    def _u(self, off: int, size: int) -> int:
        return int.from_bytes(self.buf[off:off + size], "little")

    def _addr(self, off: int) -> int:
        return self._u(off, self.so)

    def _len(self, off: int) -> int:
        return self._u(off, self.sl)

    def _sig(self, off: int, sig: bytes) -> None:
        if self.buf[off:off + len(sig)] != sig:
            raise H5FormatError(f"expected {sig!r} at {off}, found {self.buf[off:off + len(sig)]!r}")

    # -- superblock ----------------------------------------------------------------------------
    def _superblock(self) -> None:
        base = None
        for off in (0, 512, 1024, 2048, 4096):
            if self.buf[off:off + 8] == SIGNATURE:
                base = off
                break
        if base is None:
            raise H5FormatError("no HDF5 signature")
        v = self.buf[base + 8]
        self.superblock_version = v
        if v in (0, 1):
            self.so, self.sl = self.buf[base + 13], self.buf[base + 14]
            self.group_leaf_k = self._u(base + 16, 2)
            self.group_internal_k = self._u(base + 18, 2)
            p = base + 24 + (4 if v == 1 else 0)
            self.base = self._addr(p)
            p += 4 * self.so  # base, free space, end of file, driver info
            self.root = self._addr(p + self.so)  # symbol table entry: name offset, header address
        elif v in (2, 3):
            self.so, self.sl = self.buf[base + 9], self.buf[base + 10]
            p = base + 12
            self.base = self._addr(p)
            self.root = self._addr(p + 3 * self.so)  # base, extension, end of file, root header
        else:
            raise H5FormatError(f"superblock version {v}")

    # -- object headers ------------------------------------------------------------------------
    def _object(self, addr: int) -> _Object:
        if addr in self._objects:
            return self._objects[addr]
        ob = _Object(addr)
        a = self.base + addr
        if self.buf[a:a + 4] == b"OHDR":
            self._header_v2(ob, a)
        elif self.buf[a] == 1:
            nmsg = self._u(a + 2, 2)
            size = self._u(a + 8, 4)
            blocks = [(a + 16, size)]
            while blocks and len(ob.messages) < nmsg:
                p, n = blocks.pop(0)
                end = p + n
                while p + 8 <= end and len(ob.messages) < nmsg:
                    mtype, msize = self._u(p, 2), self._u(p + 2, 2)
                    data = self.buf[p + 8:p + 8 + msize]
                    if mtype == MSG_CONTINUATION:
                        blocks.append((self.base + self._addr(p + 8), self._len(p + 8 + self.so)))
                    ob.messages.append((mtype, data))
                    p += 8 + msize
        else:
            raise H5FormatError(f"object header version {self.buf[a]} at {addr}")
        self._objects[addr] = ob
        return ob

    def _header_v2(self, ob: _Object, a: int) -> None:
        flags = self.buf[a + 5]
        p = a + 6
        if flags & 0x20:
            p += 16  # access, modification, change, birth times
        if flags & 0x10:
            p += 4  # max compact / min dense attributes
        csize = 1 << (flags & 3)
        size = self._u(p, csize)
        p += csize
        blocks = [(p, size)]
        track = bool(flags & 0x4)
        while blocks:
            p, n = blocks.pop(0)
            end = p + n
            while p + 4 + (2 if track else 0) <= end:
                mtype, msize = self.buf[p], self._u(p + 1, 2)
                p += 4 + (2 if track else 0)
                data = self.buf[p:p + msize]
                if mtype == MSG_CONTINUATION:
                    c = self.base + self._addr(p)
                    self._sig(c, b"OCHK")
                    blocks.append((c + 4, self._len(p + self.so) - 8))  # minus signature, checksum
                ob.messages.append((mtype, data))
                p += msize

    # -- groups --------------------------------------------------------------------------------
    def _links(self, ob: _Object) -> Dict[str, int]:
        out: Dict[str, int] = {}
        st = ob.first(MSG_SYMBOL_TABLE)
        if st is not None:
            btree, heap = self._u_bytes(st, 0, self.so), self._u_bytes(st, self.so, self.so)
            heap_data = self._local_heap(heap)
            self._group_btree(btree, heap_data, out)
        for d in ob.all(MSG_LINK):
            name, addr = self._link_message(d)
            if addr is not None:
                out[name] = addr
        li = ob.first(MSG_LINK_INFO)
        if li is not None:
            flags = li[1]
            fheap = self._u_bytes(li, 2 + (8 if flags & 1 else 0), self.so)
            if fheap != UNDEF:
                raise H5FormatError("dense link storage (fractal heap) is not read")
        return dict(sorted(out.items()))

    def _u_bytes(self, b: bytes, off: int, size: int) -> int:
        return int.from_bytes(b[off:off + size], "little")

    def _local_heap(self, addr: int) -> bytes:
        a = self.base + addr
        self._sig(a, b"HEAP")
        size = self._len(a + 8)
        data = self.base + self._addr(a + 8 + 2 * self.sl)
        return self.buf[data:data + size]

    def _group_btree(self, addr: int, heap: bytes, out: Dict[str, int]) -> None:
        a = self.base + addr
        self._sig(a, b"TREE")
        if self.buf[a + 4] != 0:
            raise H5FormatError("group B-tree of another node type")
        level, used = self.buf[a + 5], self._u(a + 6, 2)
        p = a + 8 + 2 * self.so + self.sl  # siblings, key 0
        for _ in range(used):
            child = self._addr(p)
            p += self.so + self.sl
            if level > 0:
                self._group_btree(child, heap, out)
            else:
                self._symbol_node(child, heap, out)

    def _symbol_node(self, addr: int, heap: bytes, out: Dict[str, int]) -> None:
        a = self.base + addr
        self._sig(a, b"SNOD")
        n = self._u(a + 6, 2)
        p = a + 8
        esize = 2 * self.so + 24
        for i in range(n):
            e = p + i * esize
            name_off, header = self._addr(e), self._addr(e + self.so)
            end = heap.index(b"\0", name_off)
            out[heap[name_off:end].decode()] = header

    def _link_message(self, d: bytes) -> Tuple[str, Optional[int]]:
        flags = d[1]
        p = 2
        ltype = 0
        if flags & 0x8:
            ltype = d[p]
            p += 1
        if flags & 0x4:
            p += 8  # creation order
        if flags & 0x10:
            p += 1  # charset
        nsize = 1 << (flags & 3)
        nlen = self._u_bytes(d, p, nsize)
        p += nsize
        name = d[p:p + nlen].decode()
        p += nlen
        if ltype != 0:
            return name, None  # soft or external link
        return name, self._u_bytes(d, p, self.so)

    def _resolve(self, path: str) -> _Object:
        ob = self._object(self.root)
        for part in filter(None, path.split("/")):
            links = self._links(ob)
            if part not in links:
                raise KeyError(path)
            ob = self._object(links[part])
        return ob

    # -- public: structure ---------------------------------------------------------------------
    def keys(self, path: str = "/") -> List[str]:
        return list(self._links(self._resolve(path)))

    def is_group(self, path: str) -> bool:
        ob = self._resolve(path)
        return ob.first(MSG_LAYOUT) is None

    def has(self, path: str) -> bool:
        try:
            self._resolve(path)
            return True
        except KeyError:
            return False

    def walk(self, path: str = "/") -> List[str]:
        """Every group and dataset path below `path`, depth first in name order."""
        out = []
        for k in self.keys(path):
            p = path.rstrip("/") + "/" + k
            out.append(p)
            if self.is_group(p):
                out += self.walk(p)
        return out

    # -- dataspace, datatype -------------------------------------------------------------------
    def _dataspace(self, d: bytes) -> Optional[Tuple[int, ...]]:
        v, rank, flags = d[0], d[1], d[2]
        if v == 1:
            p = 8
            stype = 1 if rank else 0
        elif v == 2:
            stype = d[3]
            p = 4
        else:
            raise H5FormatError(f"dataspace version {v}")
        if stype == 2:
            return None  # null dataspace
        return tuple(self._u_bytes(d, p + i * self.sl, self.sl) for i in range(rank))

    def _datatype(self, d: bytes) -> _Datatype:
        cls, bits = d[0] & 0x0F, d[1] | (d[2] << 8) | (d[3] << 16)
        size = self._u_bytes(d, 4, 4)
        order = ">" if bits & 1 else "<"
        if cls == 0:
            kind = "i" if bits & 0x8 else "u"
            return _Datatype(cls, size, np.dtype(f"{order}{kind}{size}"))
        if cls == 1:
            if size not in (2, 4, 8):
                raise H5FormatError(f"floating-point size {size}")
            return _Datatype(cls, size, np.dtype(f"{order}f{size}"))
        if cls == 3:
            return _Datatype(cls, size, np.dtype(f"S{size}"))
        if cls == 9:
            vtype = bits & 0xF
            if vtype == 1:  # string
                return _Datatype(cls, size, None, vlen_string=True)
            raise H5FormatError("variable-length sequences are not read")
        raise H5FormatError(f"datatype class {cls}")

    def _vlen_strings(self, raw: bytes, count: int) -> List[str]:
        out = []
        step = 4 + self.so + 4
        for i in range(count):
            e = i * step
            n = self._u_bytes(raw, e, 4)
            coll = self._u_bytes(raw, e + 4, self.so)
            idx = self._u_bytes(raw, e + 4 + self.so, 4)
            out.append(self._global_heap_object(coll, idx)[:n].decode())
        return out

    def _global_heap_object(self, addr: int, index: int) -> bytes:
        a = self.base + addr
        self._sig(a, b"GCOL")
        size = self._len(a + 8)
        p, end = a + 8 + self.sl, a + size
        while p + 8 + self.sl <= end:
            idx, osize = self._u(p, 2), self._len(p + 8)
            if idx == index:
                return self.buf[p + 8 + self.sl:p + 8 + self.sl + osize]
            if idx == 0:
                break
            p += 8 + self.sl + _pad8(osize)
        raise H5FormatError(f"global heap object {index} not found")

    # -- public: data --------------------------------------------------------------------------
    def dataset(self, path: str):
        ob = self._resolve(path)
        layout = ob.first(MSG_LAYOUT)
        if layout is None:
            raise H5FormatError(f"{path} is not a dataset")
        shape = self._dataspace(ob.first(MSG_DATASPACE))
        dt = self._datatype(ob.first(MSG_DATATYPE))
        if shape is None:
            return np.zeros(0, dtype=dt.dtype or np.uint8)
        count = int(np.prod(shape, dtype=np.int64))
        raw = self._raw(ob, layout, shape, dt.size, path)
        if dt.vlen_string:
            strs = self._vlen_strings(raw, count)
            return np.array(strs, dtype=object).reshape(shape)
        arr = np.frombuffer(raw[:count * dt.size], dtype=dt.dtype).reshape(shape)
        return arr.astype(arr.dtype.newbyteorder("=")) if dt.dtype.byteorder == ">" else arr.copy()

    def _external(self, efl: bytes, nbytes: int, path: str) -> bytes:
        """Data of a dataset kept in external raw files (External Data Files message): the
        slots' byte ranges, concatenated. A relative file name is looked up from the current
        directory (the HDF5 library's default) and then beside this file."""
        import os

        if efl[0] != 1:
            raise H5FormatError(f"external data files message version {efl[0]} in {path}")
        used = self._u_bytes(efl, 6, 2)
        heap = self._local_heap(self._u_bytes(efl, 8, self.so))
        out = bytearray()
        p = 8 + self.so
        for _ in range(used):
            name_off, offset, size = (self._u_bytes(efl, p + i * self.sl, self.sl) for i in range(3))
            p += 3 * self.sl
            name = heap[name_off:heap.index(b"\0", name_off)].decode()
            cands = [name] + ([os.path.join(os.path.dirname(self.path), name)] if self.path else [])
            fn = next((c for c in cands if os.path.isfile(c)), None)
            if fn is None:
                raise H5FormatError(f"external file '{name}' of {path} not found")
            with open(fn, "rb") as fh:
                fh.seek(offset)
                want = nbytes - len(out)
                out += fh.read(want if size == UNDEF else min(want, size))
            if len(out) >= nbytes:
                break
        if len(out) < nbytes:
            raise H5FormatError(f"external files of {path} hold {len(out)} of {nbytes} bytes")
        return bytes(out)

    def _raw(self, ob: _Object, layout: bytes, shape, esize: int, path: str) -> bytes:
        v = layout[0]
        nbytes = int(np.prod(shape, dtype=np.int64)) * esize
        efl = ob.first(MSG_EXTERNAL)
        if efl is not None:
            return self._external(efl, nbytes, path)
        if v == 3:
            cls = layout[1]
            if cls == 0:
                n = self._u_bytes(layout, 2, 2)
                return layout[4:4 + n]
            if cls == 1:
                addr = self._u_bytes(layout, 2, self.so)
                if addr == UNDEF:
                    return bytes(nbytes)  # never written: fill value 0
                return self.buf[self.base + addr:self.base + addr + nbytes]
            if cls == 2:
                rank = layout[2]
                btree = self._u_bytes(layout, 3, self.so)
                cdims = [self._u_bytes(layout, 3 + self.so + 4 * i, 4) for i in range(rank)]
                return self._chunked(ob, btree, shape, cdims[:-1], esize)
            raise H5FormatError(f"layout class {cls} in {path}")
        if v in (1, 2):
            rank, cls = layout[1], layout[2]
            p = 8
            if cls == 0:
                p2 = p + 4 * rank
                n = self._u_bytes(layout, p2, 4)
                return layout[p2 + 4:p2 + 4 + n]
            addr = self._u_bytes(layout, p, self.so)
            if cls == 1:
                if addr == UNDEF:
                    return bytes(nbytes)
                return self.buf[self.base + addr:self.base + addr + nbytes]
            if cls == 2:
                cdims = [self._u_bytes(layout, p + self.so + 4 * i, 4) for i in range(rank)]
                return self._chunked(ob, addr, shape, cdims[:-1], esize)
        raise H5FormatError(f"layout version {v} in {path}")

    def _filters(self, ob: _Object) -> List[Tuple[int, List[int]]]:
        d = ob.first(MSG_FILTERS)
        if d is None:
            return []
        v, n = d[0], d[1]
        p = 8 if v == 1 else 2
        out = []
        for _ in range(n):
            fid = self._u_bytes(d, p, 2)
            p += 2
            nlen = 0
            if v == 1 or fid >= 256:
                nlen = self._u_bytes(d, p, 2)
                p += 2
            p += 2  # flags
            nval = self._u_bytes(d, p, 2)
            p += 2
            p += _pad8(nlen) if v == 1 else nlen
            vals = [self._u_bytes(d, p + 4 * i, 4) for i in range(nval)]
            p += 4 * nval
            if v == 1 and nval % 2:
                p += 4
            out.append((fid, vals))
        return out

    def _chunked(self, ob: _Object, btree: int, shape, cdims, esize: int) -> bytes:
        rank = len(shape)
        out = np.zeros(int(np.prod(shape, dtype=np.int64)) * esize, dtype=np.uint8).reshape(
            tuple(shape) + (esize,))
        filters = self._filters(ob)
        if btree == UNDEF:
            return out.tobytes()
        for offs, mask, addr, size in self._chunk_entries(btree, rank):
            data = self.buf[self.base + addr:self.base + addr + size]
            for i, (fid, vals) in reversed(list(enumerate(filters))):
                if mask & (1 << i):
                    continue
                if fid == FILTER_DEFLATE:
                    data = zlib.decompress(data)
                elif fid == FILTER_SHUFFLE:
                    n = len(data) // esize
                    data = np.frombuffer(data[:n * esize], np.uint8).reshape(esize, n).T.tobytes() + data[n * esize:]
                elif fid == FILTER_FLETCHER32:
                    data = data[:-4]
                else:
                    raise H5FormatError(f"filter {fid}")
            chunk = np.frombuffer(data[:int(np.prod(cdims)) * esize], np.uint8).reshape(tuple(cdims) + (esize,))
            sl_out, sl_in = [], []
            for d in range(rank):
                lo = offs[d]
                hi = min(lo + cdims[d], shape[d])
                sl_out.append(slice(lo, hi))
                sl_in.append(slice(0, hi - lo))
            out[tuple(sl_out)] = chunk[tuple(sl_in)]
        return out.tobytes()

    def _chunk_entries(self, addr: int, rank: int):
        a = self.base + addr
        self._sig(a, b"TREE")
        if self.buf[a + 4] != 1:
            raise H5FormatError("chunk B-tree of another node type")
        level, used = self.buf[a + 5], self._u(a + 6, 2)
        ksize = 8 + 8 * (rank + 1)
        p = a + 8 + 2 * self.so
        for _ in range(used):
            size, mask = self._u(p, 4), self._u(p + 4, 4)
            offs = [self._u(p + 8 + 8 * i, 8) for i in range(rank)]
            child = self._addr(p + ksize)
            if level > 0:
                yield from self._chunk_entries(child, rank)
            else:
                yield offs, mask, child, size
            p += ksize + self.so

    def attrs(self, path: str) -> Dict[str, object]:
        ob = self._resolve(path)
        out = {}
        for d in ob.all(MSG_ATTRIBUTE):
            name, value = self._attribute(d)
            out[name] = value
        ai = ob.first(MSG_ATTR_INFO)
        if ai is not None:
            flags = ai[1]
            fheap = self._u_bytes(ai, 2 + (2 if flags & 1 else 0), self.so)
            if fheap != UNDEF:
                raise H5FormatError("dense attribute storage (fractal heap) is not read")
        return out

    def _attribute(self, d: bytes):
        v = d[0]
        nlen, tlen, slen = self._u_bytes(d, 2, 2), self._u_bytes(d, 4, 2), self._u_bytes(d, 6, 2)
        p = 8 if v in (1, 2) else 9
        pad = _pad8 if v == 1 else (lambda n: n)
        name = d[p:p + nlen].rstrip(b"\0").decode()
        p += pad(nlen)
        dt = self._datatype(d[p:p + tlen])
        p += pad(tlen)
        shape = self._dataspace(d[p:p + slen])
        p += pad(slen)
        count = 1 if not shape else int(np.prod(shape))
        raw = d[p:p + count * dt.size]
        if dt.vlen_string:
            vals = self._vlen_strings(raw, count)
            return name, vals[0] if not shape else vals
        arr = np.frombuffer(raw, dtype=dt.dtype)
        if dt.cls == 3:
            strs = [bytes(x).split(b"\0")[0].decode() for x in arr]
            return name, strs[0] if not shape or count == 1 else strs
        arr = arr.astype(arr.dtype.newbyteorder("="))
        return name, arr[0] if not shape else arr.reshape(shape)


# ----------------------------------------------------------------------------------------------
# Writer
# ----------------------------------------------------------------------------------------------

_SO = 8  # size of offsets
_SL = 8  # size of lengths
_CHUNK_K = 32  # version-0 superblocks imply indexed-storage K = 32: up to 64 entries per B-tree node
_GROUP_SPARE = 768  # bytes of free header space a new group keeps for its links
_SUPERBLOCK_SIZE = 96


def _u8(v: int) -> bytes:
    return struct.pack("<Q", v)


def _msg(mtype: int, data: bytes, flags: int = 0) -> bytes:
    """One version-1 header message: type, size, flags, reserved, data padded to 8 bytes."""
    data = data + bytes(_pad8(len(data)) - len(data))
    return struct.pack("<HHB3x", mtype, len(data), flags) + data


def _nil(size: int) -> bytes:
    return struct.pack("<HHB3x", MSG_NIL, size, 0) + bytes(size)


def _datatype_message(dtype) -> bytes:
    """Datatype message (version 1) for little-endian IEEE floats, two's-complement and
    unsigned integers and null-terminated fixed-length ASCII strings."""
    dt = np.dtype(dtype)
    big = dt.byteorder == ">"
    if dt.kind == "f":
        size = dt.itemsize
        if size == 8:
            exp_loc, exp_size, mant_size, bias, sign = 52, 11, 52, 1023, 63
        elif size == 4:
            exp_loc, exp_size, mant_size, bias, sign = 23, 8, 23, 127, 31
        else:
            raise ValueError(f"float size {size}")
        return struct.pack("<BBBBI", 0x11, 0x20 | int(big), sign, 0, size) + struct.pack(
            "<HHBBBBI", 0, 8 * size, exp_loc, exp_size, 0, mant_size, bias)
    if dt.kind in "iu":
        bits = (0x08 if dt.kind == "i" else 0) | int(big)
        return struct.pack("<BBBBI", 0x10, bits, 0, 0, dt.itemsize) + struct.pack("<HH", 0, 8 * dt.itemsize)
    if dt.kind == "S":
        return struct.pack("<BBBBI", 0x13, 0, 0, 0, dt.itemsize)
    raise ValueError(f"dtype {dt} is not written")


def _dataspace_message(shape, maxshape=None) -> bytes:
    """Dataspace message (version 1); maxshape entries None are unlimited."""
    rank = len(shape)
    flags = 1 if maxshape is not None else 0
    out = struct.pack("<BBBB4x", 1, rank, flags, 0) + b"".join(_u8(int(d)) for d in shape)
    if maxshape is not None:
        out += b"".join(_u8(UNDEF if m is None else int(m)) for m in maxshape)
    return out


def _attribute_message(name: str, value) -> bytes:
    """Attribute message (version 1): a scalar string, number, or a numeric array."""
    if isinstance(value, str):
        raw = value.encode() + b"\0"
        dt, shape, data = np.dtype(f"S{len(raw)}"), (), raw
    else:
        arr = np.asarray(value)
        if arr.dtype.kind == "U":
            raise ValueError("string arrays are written as fixed-length bytes")
        arr = arr.astype(arr.dtype.newbyteorder("<"))
        dt, shape, data = arr.dtype, arr.shape, arr.tobytes()
    nm = name.encode() + b"\0"
    tmsg, smsg = _datatype_message(dt), _dataspace_message(shape)
    head = struct.pack("<BBHHH", 1, 0, len(nm), len(tmsg), len(smsg))

    def pad(b):
        return b + bytes(_pad8(len(b)) - len(b))

    return head + pad(nm) + pad(tmsg) + pad(smsg) + data


def _fill_message(chunked: bool) -> bytes:
    # version 2: allocation time (late / incremental), write fill value if set, fill value
    # defined with size 0 (the library's default: zeros)
    return struct.pack("<BBBBI", 2, 3 if chunked else 2, 2, 1, 0)


class _Header:
    """A version-1 object header being filled: its blocks' free NIL regions and the reserved
    slot for the next continuation message."""

    def __init__(self, addr: int, nmsg: int, free_at: int, free_size: int, cont_at: int):
        self.addr = addr
        self.nmsg = nmsg
        self.free_at, self.free_size = free_at, free_size  # NIL message header offset, data size
        self.cont_at = cont_at  # offset of the 16-byte NIL kept for a continuation message


class _Series:
    """A chunked dataset growing along its first (time) dimension, one chunk per step."""

    def __init__(self, header: int, dims_at: int, layout_at: int, tail, dtype):
        self.header, self.dims_at, self.layout_at = header, dims_at, layout_at
        self.tail, self.dtype = tuple(int(t) for t in tail), np.dtype(dtype)
        self.step_bytes = int(np.prod(self.tail, dtype=np.int64)) * self.dtype.itemsize
        self.chunks: List[Tuple[int, int]] = []  # (address, bytes) per step
        self.nodes: Dict[Tuple[int, int], int] = {}  # (level, index) -> address
        self.root = UNDEF


class H5Writer:
    """Writes an HDF5 file (superblock 0, version-1 object headers, compact new-style groups,
    contiguous datasets, chunked datasets with an unlimited first dimension, version-1
    attributes). The file is complete and readable after every call; datasets grown with
    `append` hold one chunk per step indexed by a version-1 chunk B-tree."""

    def __init__(self, path: str, root_attrs: Optional[Dict[str, object]] = None):
        self.path = path
        self.f = open(path, "w+b")
        self.eof = _SUPERBLOCK_SIZE
        self.groups: Dict[str, _Header] = {}
        self.series: Dict[str, _Series] = {}
        self.f.write(bytes(_SUPERBLOCK_SIZE))
        root = self._new_group(root_attrs or {})
        self.root = root.addr
        self.groups["/"] = root
        self._superblock()

    # -- file primitives -----------------------------------------------------------------------
    def _alloc(self, n: int) -> int:
        at = self.eof
        self.eof = _pad8(self.eof + n)
        return at

    def _write(self, at: int, data: bytes) -> None:
        self.f.seek(at)
        self.f.write(data)

    def _superblock(self) -> None:
        sb = SIGNATURE + bytes([0, 0, 0, 0, 0, _SO, _SL, 0]) + struct.pack("<HHI", 4, 16, 0)
        sb += _u8(0) + _u8(UNDEF) + _u8(self.eof) + _u8(UNDEF)
        # root group symbol table entry: link name offset, object header, no cached data
        sb += _u8(0) + _u8(self.root) + struct.pack("<II", 0, 0) + bytes(16)
        assert len(sb) == _SUPERBLOCK_SIZE
        self._write(0, sb)
        self.f.seek(0, 2)
        if self.f.tell() < self.eof:
            self.f.truncate(self.eof)
        self.f.flush()

    def _object_header(self, messages: List[bytes], spare: int = 0) -> _Header:
        """Writes a version-1 object header with the messages, `spare` bytes of NIL space and a
        16-byte NIL slot for a later continuation message."""
        body = b"".join(messages)
        nmsg = len(messages)
        free_rel = None
        if spare:
            free_rel = len(body)
            body += _nil(spare)
            nmsg += 1
        cont_rel = len(body)
        body += _nil(16)
        nmsg += 1
        addr = self._alloc(16 + len(body))
        self._write(addr, struct.pack("<BBHII4x", 1, 0, nmsg, 1, len(body)) + body)
        base = addr + 16
        return _Header(addr, nmsg, base + free_rel if free_rel is not None else -1, spare, base + cont_rel)

    def _add_message(self, h: _Header, message: bytes) -> None:
        """Places one message in the header's free NIL region, or in a new continuation block."""
        n = len(message)  # a multiple of 8, as every region here
        if h.free_at >= 0 and n <= h.free_size + 8:
            rest = h.free_size + 8 - n
            if rest == 0:  # the message takes the whole NIL region
                self._write(h.free_at, message)
                h.free_at, h.free_size = -1, 0
            else:  # the message, then a smaller NIL region
                self._write(h.free_at, message + _nil(rest - 8))
                h.nmsg += 1
                self._write(h.addr + 2, struct.pack("<H", h.nmsg))
                h.free_at, h.free_size = h.free_at + n, rest - 8
            return
        # new continuation block: the message, free space, and the next continuation slot
        spare = _GROUP_SPARE
        block = message + _nil(spare) + _nil(16)
        at = self._alloc(len(block))
        self._write(at, block)
        self._write(h.cont_at, _msg(MSG_CONTINUATION, _u8(at) + _u8(len(block))))
        h.nmsg += 3
        self._write(h.addr + 2, struct.pack("<H", h.nmsg))
        h.free_at, h.free_size = at + n, spare
        h.cont_at = at + n + 8 + spare

    def _new_group(self, attrs: Dict[str, object]) -> _Header:
        link_info = struct.pack("<BB", 0, 0) + _u8(UNDEF) + _u8(UNDEF)  # no dense storage
        msgs = [_msg(MSG_LINK_INFO, link_info), _msg(MSG_GROUP_INFO, struct.pack("<BB", 0, 0))]
        msgs += [_msg(MSG_ATTRIBUTE, _attribute_message(k, v)) for k, v in attrs.items()]
        return self._object_header(msgs, spare=_GROUP_SPARE)

    def _link(self, parent: str, name: str, addr: int) -> None:
        nm = name.encode()
        if len(nm) > 255:
            raise ValueError("link names longer than 255 bytes are not written")
        self._add_message(self.groups[parent], _msg(MSG_LINK, struct.pack("<BBB", 1, 0, len(nm)) + nm + _u8(addr)))

    @staticmethod
    def _split(path: str) -> Tuple[str, str]:
        path = "/" + path.strip("/")
        parent, _, name = path.rpartition("/")
        return parent or "/", name

    def _ensure_parent(self, path: str) -> str:
        parent, name = self._split(path)
        if parent not in self.groups:
            self.create_group(parent)
        return name

    # -- public --------------------------------------------------------------------------------
    def create_group(self, path: str, attrs: Optional[Dict[str, object]] = None) -> None:
        path = "/" + path.strip("/")
        if path in self.groups:
            return
        name = self._ensure_parent(path)
        h = self._new_group(attrs or {})
        self.groups[path] = h
        self._link(self._split(path)[0], name, h.addr)
        self._superblock()

    def create_dataset(self, path: str, data, attrs: Optional[Dict[str, object]] = None) -> None:
        """A contiguous dataset holding `data` (numbers, or an array of fixed-length bytes)."""
        arr = np.asarray(data)
        if arr.dtype.kind in "iuf":
            arr = arr.astype(arr.dtype.newbyteorder("<"))
        name = self._ensure_parent(path)
        raw = np.ascontiguousarray(arr).tobytes()
        at = self._alloc(len(raw)) if raw else UNDEF
        if raw:
            self._write(at, raw)
        layout = struct.pack("<BB", 3, 1) + _u8(at) + _u8(len(raw))
        msgs = [_msg(MSG_DATASPACE, _dataspace_message(arr.shape)), _msg(MSG_DATATYPE, _datatype_message(arr.dtype)),
                _msg(MSG_FILL, _fill_message(False)), _msg(MSG_LAYOUT, layout)]
        msgs += [_msg(MSG_ATTRIBUTE, _attribute_message(k, v)) for k, v in (attrs or {}).items()]
        h = self._object_header(msgs)
        self._link(self._split(path)[0], name, h.addr)
        self._superblock()

    def create_series(self, path: str, tail, dtype=np.float64, attrs: Optional[Dict[str, object]] = None) -> None:
        """An empty chunked dataset of shape (0,) + tail, growing along its first dimension by
        `append` (one chunk of shape (1,) + tail per step)."""
        name = self._ensure_parent(path)
        tail = tuple(int(t) for t in tail)
        dt = np.dtype(dtype).newbyteorder("<")
        space = _dataspace_message((0,) + tail, (None,) + tail)
        layout = struct.pack("<BBB", 3, 2, len(tail) + 2) + _u8(UNDEF) + struct.pack(
            "<" + "I" * (len(tail) + 2), 1, *tail, dt.itemsize)
        msgs = [_msg(MSG_DATASPACE, space), _msg(MSG_DATATYPE, _datatype_message(dt)),
                _msg(MSG_FILL, _fill_message(True)), _msg(MSG_LAYOUT, layout)]
        msgs += [_msg(MSG_ATTRIBUTE, _attribute_message(k, v)) for k, v in (attrs or {}).items()]
        h = self._object_header(msgs)
        # positions of the first dimension's size and of the B-tree address
        dims_at = h.addr + 16 + 8 + 8
        layout_at = h.addr + 16 + len(msgs[0]) + len(msgs[1]) + len(msgs[2]) + 8 + 3
        self.series["/" + path.strip("/")] = _Series(h.addr, dims_at, layout_at, tail, dt)
        self._link(self._split(path)[0], name, h.addr)
        self._superblock()

    def create_external(self, path: str, filename: str, tail, dtype=">f8", max_steps: Optional[int] = None,
                        attrs: Optional[Dict[str, object]] = None) -> None:
        """A dataset of shape (1,) + tail whose data live in the raw file `filename` (External Data
        Files message, one slot from offset 0 of unlimited size), as H5Pset_external gives it;
        `extend` sets its number of steps as the caller appends raw steps to that file.
        max_steps None makes the first dimension unlimited."""
        name = self._ensure_parent(path)
        tail = tuple(int(t) for t in tail)
        dt = np.dtype(dtype)
        fname = filename.encode() + b"\0"
        heap_data = bytes(8) + fname + bytes(_pad8(len(fname)) - len(fname))
        heap_at = self._alloc(32 + len(heap_data))
        self._write(heap_at, b"HEAP" + bytes(4) + _u8(len(heap_data)) + _u8(UNDEF) + _u8(heap_at + 32) + heap_data)
        efl = struct.pack("<B3xHH", 1, 1, 1) + _u8(heap_at) + _u8(8) + _u8(0) + _u8(UNDEF)
        nbytes = int(np.prod(tail, dtype=np.int64)) * dt.itemsize
        space = _dataspace_message((1,) + tail, (max_steps,) + tail)
        layout = struct.pack("<BB", 3, 1) + _u8(UNDEF) + _u8(nbytes)
        msgs = [_msg(MSG_DATASPACE, space), _msg(MSG_DATATYPE, _datatype_message(dt)),
                _msg(MSG_FILL, _fill_message(False)), _msg(MSG_LAYOUT, layout), _msg(MSG_EXTERNAL, efl)]
        msgs += [_msg(MSG_ATTRIBUTE, _attribute_message(k, v)) for k, v in (attrs or {}).items()]
        h = self._object_header(msgs)
        dims_at = h.addr + 16 + 8 + 8
        size_at = h.addr + 16 + len(msgs[0]) + len(msgs[1]) + len(msgs[2]) + 8 + 2 + _SO
        s = _Series(h.addr, dims_at, size_at, tail, dt)
        self.series["/" + path.strip("/")] = s
        self._link(self._split(path)[0], name, h.addr)
        self._superblock()

    def extend(self, path: str, steps: int) -> None:
        """Sets the number of steps of an external dataset (its dataspace and layout size)."""
        s = self.series["/" + path.strip("/")]
        self._write(s.dims_at, _u8(steps))
        self._write(s.layout_at, _u8(steps * s.step_bytes))
        self._superblock()

    def append(self, path: str, data) -> int:
        """Adds one step to a series; returns the number of steps."""
        s = self.series["/" + path.strip("/")]
        arr = np.ascontiguousarray(np.asarray(data, dtype=s.dtype).reshape(s.tail))
        raw = arr.tobytes()
        at = self._alloc(len(raw))
        self._write(at, raw)
        s.chunks.append((at, len(raw)))
        self._chunk_index(s)
        self._write(s.dims_at, _u8(len(s.chunks)))
        self._superblock()
        return len(s.chunks)

    def _chunk_index(self, s: _Series) -> None:
        """Rewrites the right edge of the series' chunk B-tree after an append (new nodes at the
        end of the file; the root address in the layout message when the tree grows a level)."""
        rank = len(s.tail) + 1
        ksize = 8 + 8 * (rank + 1)
        cap = 2 * _CHUNK_K
        node_size = 8 + 2 * _SO + (cap + 1) * ksize + cap * _SO
        n = len(s.chunks)

        def key(size: int, t: int, past: bool = False) -> bytes:
            offs = [t] + ([d for d in s.tail] + [s.dtype.itemsize] if past else [0] * (rank))
            return struct.pack("<II", size, 0) + b"".join(_u8(o) for o in offs[:rank + 1])

        # level 0 entries: (left key step, size, child address); upper levels: first step of child
        entries = [(i, s.chunks[i][1], s.chunks[i][0]) for i in range(n)]
        level = 0
        while True:
            nodes = [entries[i:i + cap] for i in range(0, len(entries), cap)]
            for j in range(len(nodes)):  # a new node is zero-filled at its full size
                if (level, j) not in s.nodes:
                    s.nodes[(level, j)] = self._alloc(node_size)
                    self._write(s.nodes[(level, j)], bytes(node_size))
            # only the last node of a level changes, and the one before it when the last is new
            # (its right-sibling address)
            for j in range(max(0, len(nodes) - 2), len(nodes)):
                ents = nodes[j]
                body = b"TREE" + struct.pack("<BBH", 1, level, len(ents))
                body += _u8(s.nodes[(level, j - 1)] if j else UNDEF)
                body += _u8(s.nodes[(level, j + 1)] if j + 1 < len(nodes) else UNDEF)
                for step, size, child in ents:
                    body += key(size, step) + _u8(child)
                # the right key: the first step past the node's last chunk, then the chunk's
                # extent in the other dimensions
                body += key(0, ents[-1][0] + self._span(s, level, ents[-1][0]), past=True)
                self._write(s.nodes[(level, j)], body)
            parents = [(ents[0][0], ents[0][1], s.nodes[(level, j)]) for j, ents in enumerate(nodes)]
            if len(nodes) == 1:
                root = parents[0][2]
                break
            entries = parents
            level += 1
        if root != s.root:
            s.root = root
            self._write(s.layout_at, _u8(root))

    @staticmethod
    def _span(s: _Series, level: int, first: int) -> int:
        """Steps covered by the last child (starting at step `first`) of a node at `level`."""
        return min((2 * _CHUNK_K) ** level, len(s.chunks) - first)

    def close(self) -> None:
        if self.f:
            self._superblock()
            self.f.close()
            self.f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
