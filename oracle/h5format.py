"""Test infrastructure (the oracle): a pure-Python restatement of the part of the HDF5 file format
that the reference's flow-field checkpoints use, for checking the library's own reader and writer
(`astr_h5*`, astr_gpu_b200/csrc/h5file.cpp). Only tests may import it.

The reference writes its checkpoints through the HDF5 library: `write_io_tree`
(src/readwrite.F90:1920-1979) creates `flowfield.h5` with the 3-D real(8) datasets ro, u1, u2, u3, p,
t of Fortran shape (ia+1, ja+1, ka+1) (h5wa3d_r8_struct, src/hdf5io.F90:752-808), then `h5srite`
adds the 1-element datasets nstep (integer) and time (real(8)) to the same file
(h5_write1int, src/hdf5io.F90:1015-1049); `readcheckpoint` (src/readwrite.F90:1378-1528) reads them
back (h5ra3d_r8_struct / h5ra3d_r8_stream, src/hdf5io.F90:204-348). The HDF5 library itself is not
part of the reference and is absent from this image, so the format is restated from the published
HDF5 File Format Specification (The HDF Group, versions 2.0/3.0): superblock versions 0-3, version 1
and 2 object headers with continuation blocks, groups as symbol tables (version 1 B-tree of group
nodes, symbol table nodes, local heap) or compact link messages, and datasets with the dataspace,
datatype, data layout (compact or contiguous), filter pipeline and attribute messages.

Parity is pinned by reading one file written by the HDF5 library (a MATLAB 7.3 file from scipy's
test data, user block of 512 bytes, superblock version 0): the reader returns its dataset and its
attribute. No other HDF5 file exists in this image.

The writer here makes version-0 files like the library's default output, with switchable choices
(user block, layout message version, byte order, SNOD capacity, 1-D "stream" datasets) that the
library's writer does not make, and version-2 files (`write_v2`: checksummed superblock and object
headers, compact links), so that the reader under test meets more than its own writer's output.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5FormatError(ValueError):
    pass


@dataclass
class Entry:
    name: str
    address: int
    kind: str = "other"            # "dataset", "group" or "other"
    dims: tuple = ()               # HDF5 (C) order, slowest first
    dtype: np.dtype | None = None
    layout: str = ""               # "compact", "contiguous", "chunked"
    data_address: int = UNDEF
    data_size: int = 0
    filtered: bool = False
    attrs: dict = field(default_factory=dict)
    data: np.ndarray | None = None
    messages: list = field(default_factory=list)   # (type, version, flags, raw bytes)


@dataclass
class FileInfo:
    superblock_version: int
    base: int
    eof: int
    root_address: int
    group_kind: str                # "symbol_table" or "links"
    root_messages: list
    entries: dict


def _u(b, off, n):
    return int.from_bytes(b[off:off + n], "little")


_M32 = 0xFFFFFFFF


def _rot(x, k):
    return ((x << k) | (x >> (32 - k))) & _M32


def lookup3(data: bytes, initval: int = 0) -> int:
    """Bob Jenkins' lookup3 hash (hashlittle, public domain, 2006), the checksum of the HDF5
    format's version-2 structures: 12-byte blocks mixed into three 32-bit words, the last block
    zero-padded and finalised (an empty input returns the initial value)."""
    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & _M32
    i = 0
    while n - i > 12:
        a = (a + _u(data, i, 4)) & _M32
        b = (b + _u(data, i + 4, 4)) & _M32
        c = (c + _u(data, i + 8, 4)) & _M32
        a = (a - c) & _M32; a ^= _rot(c, 4); c = (c + b) & _M32
        b = (b - a) & _M32; b ^= _rot(a, 6); a = (a + c) & _M32
        c = (c - b) & _M32; c ^= _rot(b, 8); b = (b + a) & _M32
        a = (a - c) & _M32; a ^= _rot(c, 16); c = (c + b) & _M32
        b = (b - a) & _M32; b ^= _rot(a, 19); a = (a + c) & _M32
        c = (c - b) & _M32; c ^= _rot(b, 4); b = (b + a) & _M32
        i += 12
    if i == n:
        return c
    t = bytes(data[i:]) + bytes(12 - (n - i))
    a = (a + _u(t, 0, 4)) & _M32
    b = (b + _u(t, 4, 4)) & _M32
    c = (c + _u(t, 8, 4)) & _M32
    c ^= b; c = (c - _rot(b, 14)) & _M32
    a ^= c; a = (a - _rot(c, 11)) & _M32
    b ^= a; b = (b - _rot(a, 25)) & _M32
    c ^= b; c = (c - _rot(b, 16)) & _M32
    a ^= c; a = (a - _rot(c, 4)) & _M32
    b ^= a; b = (b - _rot(a, 14)) & _M32
    c ^= b; c = (c - _rot(b, 24)) & _M32
    return c


class _Reader:
    def __init__(self, raw: bytes):
        self.raw = raw
        self.base = 0

    def at(self, addr, n):
        a = self.base + addr
        if addr == UNDEF or a < 0 or a + n > len(self.raw):
            raise H5FormatError(f"read of {n} bytes at {addr:#x} outside the file")
        return self.raw[a:a + n]

    # ---- superblock
    def superblock(self):
        off = 0
        while off + 8 <= len(self.raw):
            if self.raw[off:off + 8] == SIGNATURE:
                break
            off = 512 if off == 0 else off * 2
        else:
            raise H5FormatError("no HDF5 signature")
        b = self.raw[off:off + 128]
        ver = b[8]
        if ver in (0, 1):
            if b[13] != 8 or b[14] != 8:
                raise H5FormatError("only 8-byte offsets and lengths")
            q = 24 + (4 if ver == 1 else 0)
            base, _fs, eof, _drv = (_u(b, q + 8 * i, 8) for i in range(4))
            e = q + 32
            root = _u(b, e + 8, 8)
        elif ver in (2, 3):
            if b[9] != 8 or b[10] != 8:
                raise H5FormatError("only 8-byte offsets and lengths")
            base, _ext, eof, root = (_u(b, 12 + 8 * i, 8) for i in range(4))
            if lookup3(b[:44]) != _u(b, 44, 4):
                raise H5FormatError("superblock checksum")
        else:
            raise H5FormatError(f"superblock version {ver}")
        self.base = base
        return ver, base, eof, root

    # ---- object headers: list of (type, flags, data, version)
    def object_header(self, addr):
        msgs = []
        if self.at(addr, 4) == b"OHDR":
            h = self.at(addr, 6)
            if h[4] != 2:
                raise H5FormatError("object header version")
            flags = h[5]
            pos = 6 + (16 if flags & 0x20 else 0) + (4 if flags & 0x10 else 0)
            w = 1 << (flags & 3)
            size0 = _u(self.at(addr + pos, w), 0, w)
            whole = self.at(addr, pos + w + size0 + 4)
            if lookup3(whole[:-4]) != _u(whole, len(whole) - 4, 4):
                raise H5FormatError("object header checksum")
            chunks = [(addr + pos + w, size0)]
            ohv = 2
        else:
            h = self.at(addr, 16)
            if h[0] != 1:
                raise H5FormatError("object header version")
            nmesgs = _u(h, 2, 2)
            chunks = [(addr + 16, _u(h, 8, 4))]
            ohv, flags = 1, 0
        done = 0
        hs = 8 if ohv == 1 else 4 + (2 if flags & 0x04 else 0)
        while done < len(chunks):
            start, size = chunks[done]
            done += 1
            if ohv == 2 and done > 1:      # continuation block: "OCHK", messages, checksum
                if self.at(start, 4) != b"OCHK":
                    raise H5FormatError("continuation block signature")
                start, size = start + 4, size - 8
            body = self.at(start, size)
            pos = 0
            while pos + hs <= size:
                if ohv == 1:
                    t, ms, mf = _u(body, pos, 2), _u(body, pos + 2, 2), body[pos + 4]
                else:
                    t, ms, mf = body[pos], _u(body, pos + 1, 2), body[pos + 3]
                d = body[pos + hs:pos + hs + ms]
                if len(d) != ms:
                    raise H5FormatError("message runs past its chunk")
                msgs.append((t, mf, d, start + pos + hs))
                if t == 0x10:
                    chunks.append((_u(d, 0, 8), _u(d, 8, 8)))
                pos += hs + ms
                if ohv == 1 and len(msgs) == nmesgs:
                    break
        if ohv == 1 and len(msgs) != nmesgs:
            raise H5FormatError("object header message count")
        return msgs

    # ---- group members: name -> object header address
    def local_heap(self, addr):
        h = self.at(addr, 32)
        if h[:4] != b"HEAP":
            raise H5FormatError("local heap signature")
        return self.at(_u(h, 24, 8), _u(h, 8, 8))

    def btree_members(self, addr, heap, out, depth=0):
        h = self.at(addr, 24)
        if h[:4] != b"TREE" or h[4] != 0:
            raise H5FormatError("group B-tree node")
        level, n = h[5], _u(h, 6, 2)
        body = self.at(addr + 24, 16 * n + 8)
        for i in range(n):
            child = _u(body, 8 + 16 * i, 8)
            if level > 0:
                if depth > 16:
                    raise H5FormatError("B-tree too deep")
                self.btree_members(child, heap, out, depth + 1)
            else:
                s = self.at(child, 8)
                if s[:4] != b"SNOD":
                    raise H5FormatError("symbol table node signature")
                ents = self.at(child + 8, 40 * _u(s, 6, 2))
                for k in range(_u(s, 6, 2)):
                    noff = _u(ents, 40 * k, 8)
                    name = heap[noff:heap.index(b"\0", noff)].decode()
                    out[name] = _u(ents, 40 * k + 8, 8)

    def links(self, msgs):
        out = {}
        for t, _f, d, _p in msgs:
            if t == 0x02 and len(d) >= 10:
                fheap = _u(d, 2 + (8 if d[1] & 1 else 0), 8)
                if fheap != UNDEF:
                    raise H5FormatError("dense link storage")
            if t != 0x06:
                continue
            fl = d[1]
            pos = 2
            ltype = 0
            if fl & 0x08:
                ltype = d[pos]
                pos += 1
            if fl & 0x04:
                pos += 8
            if fl & 0x10:
                pos += 1
            w = 1 << (fl & 3)
            ln = _u(d, pos, w)
            pos += w
            name = d[pos:pos + ln].decode()
            pos += ln
            if ltype == 0:
                out[name] = _u(d, pos, 8)
        return out


def _datatype(d):
    cls, b0 = d[0] & 0x0F, d[1]
    size = _u(d, 4, 4)
    order = ">" if b0 & 1 else "<"
    if cls == 0:
        return np.dtype(f"{order}{'i' if b0 & 8 else 'u'}{size}")
    if cls == 1:
        if b0 & 0x40 or size not in (4, 8):
            raise H5FormatError("floating-point layout")
        exp_loc, exp_size, mant_loc, mant_size, bias = d[12], d[13], d[14], d[15], _u(d, 16, 4)
        ieee = {8: (52, 11, 0, 52, 1023, 63), 4: (23, 8, 0, 23, 127, 31)}[size]
        if (exp_loc, exp_size, mant_loc, mant_size, bias, d[2]) != ieee:
            raise H5FormatError("non-IEEE floating point")
        return np.dtype(f"{order}f{size}")
    if cls == 3:
        return np.dtype(f"S{size}")
    return None


def _dataspace(d):
    ver, rank = d[0], d[1]
    if ver == 1:
        pos = 8
    elif ver == 2:
        if d[3] == 2:
            return None
        pos = 4
    else:
        raise H5FormatError("dataspace version")
    return tuple(_u(d, pos + 8 * i, 8) for i in range(rank))


def _layout(d, itemsize):
    ver = d[0]
    if ver in (1, 2):
        nd, cls = d[1], d[2]
        pos = 8
        addr = UNDEF
        if cls != 0:
            addr = _u(d, pos, 8)
            pos += 8
        dims = [_u(d, pos + 4 * i, 4) for i in range(nd)]
        pos += 4 * nd
        if cls == 0:
            n = _u(d, pos, 4)
            return "compact", UNDEF, n, d[pos + 4:pos + 4 + n]
        if cls == 1:
            return "contiguous", addr, int(np.prod(dims, dtype=np.int64)), None
        return "chunked", UNDEF, 0, None
    if ver in (3, 4):
        cls = d[1]
        if cls == 0:
            n = _u(d, 2, 2)
            return "compact", UNDEF, n, d[4:4 + n]
        if cls == 1:
            return "contiguous", _u(d, 2, 8), _u(d, 10, 8), None
        return "chunked", UNDEF, 0, None
    raise H5FormatError("layout version")


def _attribute(d):
    ver = d[0]
    if ver == 1:
        nl, tl, sl = _u(d, 2, 2), _u(d, 4, 2), _u(d, 6, 2)
        pad = lambda n: (n + 7) // 8 * 8
        pos = 8
        name = d[pos:pos + nl].rstrip(b"\0").decode()
        pos += pad(nl)
        dt = _datatype(d[pos:pos + tl])
        pos += pad(tl)
        dims = _dataspace(d[pos:pos + sl])
        pos += pad(sl)
        n = int(np.prod(dims, dtype=np.int64)) if dims is not None else 0
        val = np.frombuffer(d[pos:pos + n * dt.itemsize], dtype=dt) if dt is not None else None
        return name, val
    return None, None


def read(path, *, with_data=True) -> FileInfo:
    """Every member of the root group with its dataspace, datatype, layout and attributes, and the
    data of every numeric dataset (in the file's C order) unless with_data is False."""
    with open(path, "rb") as fh:
        raw = fh.read()
    r = _Reader(raw)
    ver, base, eof, root = r.superblock()
    rmsgs = r.object_header(root)
    stab = [m for m in rmsgs if m[0] == 0x11]
    members = {}
    if stab:
        d = stab[0][2]
        r.btree_members(_u(d, 0, 8), r.local_heap(_u(d, 8, 8)), members)
        kind = "symbol_table"
    else:
        members = r.links(rmsgs)
        kind = "links"
    entries = {}
    for name, addr in members.items():
        msgs = r.object_header(addr)
        e = Entry(name, addr, messages=[(t, d[0] if d else 0, f, bytes(d)) for t, f, d, _p in msgs])
        types = {t: d for t, _f, d, _p in msgs}
        if 0x11 in types or 0x02 in types or 0x06 in types:
            e.kind = "group"
        if 0x01 in types and 0x03 in types and 0x08 in types:
            e.kind = "dataset"
            e.dims = _dataspace(types[0x01]) or ()
            e.dtype = _datatype(types[0x03])
            e.filtered = 0x0B in types
            e.layout, e.data_address, e.data_size, compact = _layout(types[0x08], e.dtype.itemsize if e.dtype else 1)
            if with_data and e.dtype is not None and e.dtype.kind in "iuf" and e.layout != "chunked" and not e.filtered:
                n = int(np.prod(e.dims, dtype=np.int64))
                nb = n * e.dtype.itemsize
                if e.layout == "compact":
                    buf = compact[:nb]
                elif e.data_address == UNDEF:
                    buf = bytes(nb)
                else:
                    buf = r.at(e.data_address, nb)
                e.data = np.frombuffer(buf, dtype=e.dtype).reshape(e.dims).copy()
        for t, _f, d, _p in msgs:
            if t == 0x0C:
                k, v = _attribute(d)
                if k is not None:
                    e.attrs[k] = v
        entries[name] = e
    return FileInfo(ver, base, eof, root, kind, [(t, d[0] if d else 0, f, bytes(d)) for t, f, d, _p in rmsgs],
                    entries)


# ---------------------------------------------------------------------------------- writer

def _pad8(b: bytes) -> bytes:
    return b + bytes(-len(b) % 8)


def _dtype_message(dt: np.dtype) -> bytes:
    be = 1 if dt.byteorder == ">" else 0
    if dt.kind == "f":
        ieee = {8: (64, 52, 11, 0, 52, 1023, 63), 4: (32, 23, 8, 0, 23, 127, 31)}[dt.itemsize]
        prec, el, es, ml, ms, bias, sign = ieee
        return struct.pack("<BBBBI", 0x11, 0x20 | be, sign, 0, dt.itemsize) + struct.pack(
            "<HHBBBBI", 0, prec, el, es, ml, ms, bias)
    if dt.kind in "iu":
        return struct.pack("<BBBBI", 0x10, be | (0x08 if dt.kind == "i" else 0), 0, 0, dt.itemsize) + struct.pack(
            "<HH", 0, 8 * dt.itemsize)
    raise H5FormatError("unsupported numpy type")


def _message_v1(t, flags, body):
    body = _pad8(body)
    return struct.pack("<HHB3x", t, len(body), flags) + body


def _object_header_v1(msgs) -> bytes:
    body = b"".join(msgs)
    return struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body


def _ohdr(msgs) -> bytes:
    """A version-2 object header holding `msgs` (type, flags, body) in one chunk, checksummed."""
    body = b"".join(struct.pack("<BHB", t, len(d), f) + d for t, f, d in msgs)
    w, fl = (1, 0) if len(body) < 256 else (2, 1) if len(body) < 65536 else (4, 2)
    blob = b"OHDR" + bytes([2, fl]) + len(body).to_bytes(w, "little") + body
    return blob + struct.pack("<I", lookup3(blob))


def write_v2(path, datasets):
    """A file in the format's newer layout (what the HDF5 library writes with its latest format
    bounds): superblock version 2, version-2 object headers, the root group as compact link
    messages (with link info and group info messages), dataspace version 2, fill value version 3,
    contiguous layout version 3; every superblock and object header checksummed with lookup3."""
    out = bytearray(48)
    links = []
    for name, arr in datasets:
        a = np.asarray(arr, order="C")
        dims = a.shape
        space = struct.pack("<BBBB", 2, len(dims), 0, 1) + b"".join(struct.pack("<Q", d) for d in dims)
        fixed = [(0x01, 0, space), (0x03, 1, _dtype_message(a.dtype)), (0x05, 1, bytes([3, 0x0A]))]
        oh_at = len(out)
        oh_len = len(_ohdr(fixed + [(0x08, 0, bytes(18))]))
        data_at = oh_at + oh_len if a.nbytes else UNDEF
        out.extend(_ohdr(fixed + [(0x08, 0, struct.pack("<BBQQ", 3, 1, data_at, a.nbytes))]))
        out.extend(a.tobytes())
        nm = name.encode()
        if len(nm) > 255:
            raise H5FormatError("names up to 255 bytes")
        links.append((0x06, 0, bytes([1, 0, len(nm)]) + nm + struct.pack("<Q", oh_at)))
    root_at = len(out)
    out.extend(_ohdr([(0x02, 0, bytes([0, 0]) + struct.pack("<QQ", UNDEF, UNDEF)), (0x0A, 0, bytes([0, 0]))] + links))
    sb = SIGNATURE + bytes([2, 8, 8, 0]) + struct.pack("<QQQQ", 0, UNDEF, len(out), root_at)
    out[0:48] = sb + struct.pack("<I", lookup3(sb))
    with open(path, "wb") as fh:
        fh.write(out)


def write(path, datasets, *, user_block=0, layout_version=3, snod_capacity=8, byte_order="<", compact=(),
          chunked=(), filtered=(), shared_type=()):
    """A version-0 file whose root group holds `datasets`: a sequence of (name, numpy array); the
    array's shape is the dataspace (C order). user_block: bytes before the superblock (a power of
    two >= 512, or 0); layout_version: 2 (dims with the element size, as older libraries wrote)
    or 3; snod_capacity: entries per symbol table node (2 x the leaf K written to the superblock,
    so 8 is the library's default); byte_order: '<' or '>' for the stored numbers. Datasets named
    in `compact` keep their data inside the layout message (version 3); those in `chunked` get a
    chunked layout message, those in `filtered` a deflate filter pipeline message (header only)
    and those in `shared_type` a datatype message flagged as shared, for readers that must
    refuse them."""
    leaf_k = snod_capacity // 2
    ik = 16
    names = [n for n, _ in datasets]
    if len(set(names)) != len(names):
        raise H5FormatError("duplicate name")
    out = bytearray(user_block + 96)
    def addr():
        return len(out) - user_block
    def align():
        out.extend(bytes(-len(out) % 8))
    ohs = {}
    for name, arr in datasets:
        a = np.asarray(arr, order="C").astype(np.dtype(arr.dtype).newbyteorder(byte_order), copy=False)
        dims = a.shape
        space = struct.pack("<BBBB4x", 1, len(dims), 0, 0) + b"".join(struct.pack("<Q", d) for d in dims)
        nbytes = a.nbytes
        align()
        oh_at = addr()
        fixed = [_message_v1(0x05, 1, bytes([1, 2, 2, 1, 0, 0, 0, 0])),
                 _message_v1(0x03, 3 if name in shared_type else 1, _dtype_message(a.dtype)),
                 _message_v1(0x01, 0, space)]
        if name in filtered:
            fixed.append(_message_v1(0x0B, 0, struct.pack("<BB6xHHHHI", 1, 1, 1, 0, 0, 1, 6)))
        inline = name in compact or name in chunked
        if name in compact:
            lay_len = 4 + nbytes
        elif name in chunked:
            lay_len = 3 + 8 + 4 * (len(dims) + 1)
        elif layout_version == 2:
            lay_len = 8 + 8 + 4 * (len(dims) + 1)
        else:
            lay_len = 18
        oh_len = 16 + sum(len(m) for m in fixed) + 8 + ((lay_len + 7) // 8 * 8)
        data_at = oh_at + oh_len if nbytes and not inline else UNDEF
        if name in compact:
            lay = struct.pack("<BBH", 3, 0, nbytes) + a.tobytes()
        elif name in chunked:
            lay = struct.pack("<BBBQ", 3, 2, len(dims) + 1, UNDEF) + b"".join(
                struct.pack("<I", d) for d in (*dims, a.dtype.itemsize))
        elif layout_version == 2:
            lay = struct.pack("<BBB5xQ", 2, len(dims) + 1, 1, data_at) + b"".join(
                struct.pack("<I", d) for d in (*dims, a.dtype.itemsize))
        else:
            lay = struct.pack("<BBQQ", 3, 1, data_at, nbytes)
        oh = _object_header_v1(fixed + [_message_v1(0x08, 1, lay)])
        assert len(oh) == oh_len
        out.extend(oh)
        if not inline:
            out.extend(a.tobytes())
        ohs[name] = oh_at
    # root group: local heap, symbol table nodes, one B-tree node
    order = sorted(names, key=lambda s: s.encode())
    seg = bytearray(8)
    noff = {}
    for n in order:
        noff[n] = len(seg)
        seg.extend(_pad8(n.encode() + b"\0"))
    free_at = len(seg)
    seg.extend(struct.pack("<QQ", 1, 16))
    align()
    heap_at = addr()
    out.extend(b"HEAP" + bytes(4) + struct.pack("<QQQ", len(seg), free_at, heap_at + 32))
    out.extend(seg)
    groups = [order[i:i + snod_capacity] for i in range(0, len(order), snod_capacity)]
    if len(groups) > 2 * ik:
        raise H5FormatError("too many members for one B-tree node")
    snods = []
    for g in groups:
        align()
        snods.append(addr())
        ent = b"".join(struct.pack("<QQII16x", noff[n], ohs[n], 0, 0) for n in g)
        out.extend(b"SNOD" + struct.pack("<BBH", 1, 0, len(g)) + ent + bytes(40 * (snod_capacity - len(g))))
    align()
    tree_at = addr()
    node = bytearray(b"TREE" + struct.pack("<BBHQQ", 0, 0, len(groups), UNDEF, UNDEF))
    node += struct.pack("<Q", 0)
    for g, s in zip(groups, snods):
        node += struct.pack("<QQ", s, noff[g[-1]])
    node += bytes(24 + (2 * ik + 1) * 8 + 2 * ik * 8 - len(node))
    out.extend(node)
    align()
    root_at = addr()
    out.extend(_object_header_v1([_message_v1(0x11, 1, struct.pack("<QQ", tree_at, heap_at)),
                                  _message_v1(0x00, 0, b"")]))
    sb = SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", leaf_k, ik, 0)
    sb += struct.pack("<QQQQ", user_block, UNDEF, len(out), UNDEF)
    sb += struct.pack("<QQII", 0, root_at, 1, 0) + struct.pack("<QQ", tree_at, heap_at)
    assert len(sb) == 96
    out[user_block:user_block + 96] = sb
    with open(path, "wb") as fh:
        fh.write(out)
