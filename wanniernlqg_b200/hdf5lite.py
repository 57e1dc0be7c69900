"""Read-only reader for the subset of the HDF5 file format that operator bundles use.

The image has no HDF5 library or binding, so this module reads the container directly from the
published HDF5 File Format Specification (version 3.0 of the document): superblocks 0-3, version 1
and 2 object headers with continuation blocks, old-style groups (symbol-table messages, version 1
B-trees, local heaps), new-style groups with compact links and dense links (fractal heap plus a
version 2 B-tree name index), compact and dense attributes, contiguous, compact and version 1
B-tree chunked layouts (with the deflate filter), and the datatype classes fixed-point, floating
point, string, bitfield, compound, enumeration, variable-length and array.  Every checksummed
metadata block (superblock 2/3, object headers, fractal heap blocks, v2 B-tree nodes) is verified
with Bob Jenkins' lookup3 hash, as the format requires, so a damaged file raises instead of
returning wrong metadata.

Arrays come back in HDF5's dimension order (C order, slowest first).  A column-major writer such
as Julia stores an array of size (n1, n2, ...) as HDF5 dimensions (..., n2, n1); transpose to get
the writer's logical array.
"""
from __future__ import annotations

import mmap
import struct
import zlib

import numpy as np

_SIGNATURE = b"\x89HDF\r\n\x1a\n"


class HDF5FormatError(ValueError):
    """The file is not HDF5, is damaged, or uses a part of the format this reader does not read."""


# --------------------------------------------------------------------------------------------
# lookup3 (Bob Jenkins, 2006, public domain): hashlittle over bytes, initval 0, as the HDF5
# format uses for every metadata checksum.
# --------------------------------------------------------------------------------------------

_M = 0xFFFFFFFF


def _rot(x, k):
    return ((x << k) | (x >> (32 - k))) & _M


def lookup3(data: bytes, initval: int = 0) -> int:
    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & _M
    if n == 0:
        return c
    pad = (-n) % 12
    if n % 12 == 0:
        pad = 0
    words = struct.unpack("<%dI" % ((n + pad) // 4), bytes(data) + b"\0" * pad)
    nblocks = (n + pad) // 12
    for blk in range(nblocks - 1):
        a = (a + words[3 * blk]) & _M
        b = (b + words[3 * blk + 1]) & _M
        c = (c + words[3 * blk + 2]) & _M
        a = (a - c) & _M; a ^= _rot(c, 4); c = (c + b) & _M
        b = (b - a) & _M; b ^= _rot(a, 6); a = (a + c) & _M
        c = (c - b) & _M; c ^= _rot(b, 8); b = (b + a) & _M
        a = (a - c) & _M; a ^= _rot(c, 16); c = (c + b) & _M
        b = (b - a) & _M; b ^= _rot(a, 19); a = (a + c) & _M
        c = (c - b) & _M; c ^= _rot(b, 4); b = (b + a) & _M
    last = nblocks - 1
    a = (a + words[3 * last]) & _M
    b = (b + words[3 * last + 1]) & _M
    c = (c + words[3 * last + 2]) & _M
    c ^= b; c = (c - _rot(b, 14)) & _M
    a ^= c; a = (a - _rot(c, 11)) & _M
    b ^= a; b = (b - _rot(a, 25)) & _M
    c ^= b; c = (c - _rot(b, 16)) & _M
    a ^= c; a = (a - _rot(c, 4)) & _M
    b ^= a; b = (b - _rot(a, 14)) & _M
    c ^= b; c = (c - _rot(b, 24)) & _M
    return c


def _limit_enc_size(value: int) -> int:
    """Bytes the format uses to encode counts up to ``value`` (log2(value) / 8 + 1)."""
    return (max(int(value), 1).bit_length() - 1) // 8 + 1


# --------------------------------------------------------------------------------------------
# Datatypes
# --------------------------------------------------------------------------------------------


class Datatype:
    """A decoded datatype message: ``size`` bytes per element and a way to decode raw bytes."""

    def __init__(self, cls, size, np_dtype=None, **extra):
        self.cls = cls
        self.size = size
        self.np_dtype = np_dtype
        self.__dict__.update(extra)

    def decode(self, f: "File", raw: bytes, count: int):
        """Decode ``count`` packed elements; returns a numpy array (or list of objects)."""
        if self.cls == 3:  # fixed-length string
            out = []
            for i in range(count):
                s = bytes(raw[i * self.size:(i + 1) * self.size])
                if self.pad in (0, 1):
                    s = s.split(b"\0", 1)[0]
                else:
                    s = s.rstrip(b" ")
                out.append(s.decode("utf-8" if self.cset == 1 else "ascii", "replace"))
            return np.array(out, dtype=object)
        if self.cls == 9:
            out = []
            osz = f.size_of_offsets
            for i in range(count):
                base = i * self.size
                n = struct.unpack_from("<I", raw, base)[0]
                addr = f._unpack_addr(raw, base + 4)
                index = struct.unpack_from("<I", raw, base + 4 + osz)[0]
                if addr is None or n == 0:
                    payload = b""
                else:
                    payload = f._global_heap_object(addr, index)
                if self.vtype == 1:
                    s = payload[:n]
                    if self.pad in (0, 1):
                        s = s.split(b"\0", 1)[0]
                    out.append(s.decode("utf-8" if self.cset == 1 else "ascii", "replace"))
                else:
                    out.append(self.base.decode(f, payload, n))
            return np.array(out, dtype=object) if self.vtype == 1 else out
        if self.cls == 8:
            values = self.base.decode(f, raw, count)
            if sorted(self.names) == ["FALSE", "TRUE"]:
                true_value = self.values[self.names.index("TRUE")]
                return np.asarray(values) == true_value
            return values
        if self.cls == 10:
            inner = int(np.prod(self.dims))
            arr = self.base.decode(f, raw, count * inner)
            return np.asarray(arr).reshape((count,) + tuple(self.dims))
        if self.cls == 6 and self.np_dtype is None:
            raise HDF5FormatError("compound datatype with non-numeric members is not supported")
        arr = np.frombuffer(raw, dtype=self.np_dtype, count=count)
        if self.cls == 6 and self.complex_dtype is not None:
            arr = arr.view(self.complex_dtype).reshape(arr.shape)
        return arr


def _parse_datatype(f: "File", buf, pos: int):
    """Parse a datatype message at ``buf[pos:]``; returns (Datatype, bytes consumed)."""
    class_ver = buf[pos]
    cls = class_ver & 0x0F
    version = class_ver >> 4
    bits = buf[pos + 1] | (buf[pos + 2] << 8) | (buf[pos + 3] << 16)
    size = struct.unpack_from("<I", buf, pos + 4)[0]
    p = pos + 8
    if cls in (0, 4):  # fixed-point, bitfield
        if bits & 1:
            raise HDF5FormatError("big-endian integers are not supported")
        signed = bool(bits & 0x08) if cls == 0 else False
        if size not in (1, 2, 4, 8):
            raise HDF5FormatError("integer of %d bytes" % size)
        dt = np.dtype(("<i%d" if signed else "<u%d") % size)
        return Datatype(cls, size, dt), 8 + 4
    if cls == 1:
        if bits & 0x41:
            raise HDF5FormatError("non-little-endian floating point is not supported")
        if size not in (2, 4, 8):
            raise HDF5FormatError("floating point of %d bytes" % size)
        return Datatype(cls, size, np.dtype("<f%d" % size)), 8 + 12
    if cls == 3:
        return Datatype(cls, size, None, pad=bits & 0x0F, cset=(bits >> 4) & 0x0F), 8
    if cls == 6:
        nmembers = bits & 0xFFFF
        names, offsets, formats = [], [], []
        for _ in range(nmembers):
            end = bytes(buf[p:p + 4096]).index(b"\0")
            name = bytes(buf[p:p + end]).decode("utf-8")
            if version in (1, 2):
                p += (end + 8) // 8 * 8
                offset = struct.unpack_from("<I", buf, p)[0]
                p += 4
                if version == 1:
                    ndims = buf[p]
                    p += 1 + 3 + 4 + 4 + 16
                    if ndims:
                        raise HDF5FormatError("compound members with array dimensions")
            else:
                p += end + 1
                nb = 1 if size < 256 else 2 if size < 65536 else 3 if size < (1 << 24) else 4
                offset = int.from_bytes(bytes(buf[p:p + nb]), "little")
                p += nb
            member, used = _parse_datatype(f, buf, p)
            p += used
            names.append(name)
            offsets.append(offset)
            formats.append(member.np_dtype)
        complex_dtype = None
        if all(fm is not None for fm in formats):
            np_dtype = np.dtype({"names": names, "formats": formats, "offsets": offsets,
                                 "itemsize": size})
            if (len(names) == 2 and formats[0] == formats[1] and formats[0].kind == "f"
                    and offsets == [0, formats[0].itemsize] and size == 2 * formats[0].itemsize):
                complex_dtype = np.dtype("<c%d" % size)
        else:
            np_dtype = None
        return Datatype(cls, size, np_dtype, names=names, complex_dtype=complex_dtype), p - pos
    if cls == 8:
        nmembers = bits & 0xFFFF
        base, used = _parse_datatype(f, buf, p)
        p += used
        names = []
        for _ in range(nmembers):
            end = bytes(buf[p:p + 4096]).index(b"\0")
            names.append(bytes(buf[p:p + end]).decode("utf-8"))
            p += (end + 8) // 8 * 8 if version in (1, 2) else end + 1
        values = list(np.frombuffer(bytes(buf[p:p + nmembers * base.size]), dtype=base.np_dtype))
        p += nmembers * base.size
        return Datatype(cls, size, base.np_dtype, base=base, names=names, values=values), p - pos
    if cls == 9:
        base, used = _parse_datatype(f, buf, p)
        p += used
        return Datatype(cls, size, None, base=base, vtype=bits & 0x0F, pad=(bits >> 4) & 0x0F,
                        cset=(bits >> 8) & 0x0F), p - pos
    if cls == 10:
        ndims = buf[p]
        if version == 2:
            p += 4
            dims = struct.unpack_from("<%dI" % ndims, buf, p)
            p += 8 * ndims
        else:
            p += 1
            dims = struct.unpack_from("<%dI" % ndims, buf, p)
            p += 4 * ndims
        base, used = _parse_datatype(f, buf, p)
        p += used
        return Datatype(cls, size, None, base=base, dims=dims), p - pos
    raise HDF5FormatError("datatype class %d is not supported" % cls)


def _parse_dataspace(f: "File", buf, pos: int):
    """Returns the dimensions (a tuple; () for a scalar, None for a null dataspace)."""
    version = buf[pos]
    ndims = buf[pos + 1]
    L = f.size_of_lengths
    if version == 1:
        p = pos + 8
        kind = 1 if ndims else 0
    elif version == 2:
        kind = buf[pos + 3]
        p = pos + 4
    else:
        raise HDF5FormatError("dataspace version %d" % version)
    if kind == 2:
        return None
    dims = tuple(int.from_bytes(bytes(buf[p + i * L:p + (i + 1) * L]), "little")
                 for i in range(ndims))
    return dims


# --------------------------------------------------------------------------------------------
# Objects
# --------------------------------------------------------------------------------------------


class _Message:
    __slots__ = ("type", "flags", "pos", "size")

    def __init__(self, mtype, flags, pos, size):
        self.type, self.flags, self.pos, self.size = mtype, flags, pos, size


class Node:
    """A group or dataset: its header messages, attributes and (for groups) links."""

    def __init__(self, f: "File", address: int, name: str):
        self.file = f
        self.address = address
        self.name = name
        self.messages = f._object_messages(address)
        self._attrs = None

    def _first(self, mtype):
        for m in self.messages:
            if m.type == mtype:
                return m
        return None

    @property
    def attrs(self) -> dict:
        if self._attrs is None:
            self._attrs = self.file._attributes(self)
        return self._attrs


class Group(Node):
    def __init__(self, f, address, name):
        super().__init__(f, address, name)
        self._link_cache = None

    def links(self) -> dict:
        if self._link_cache is None:
            self._link_cache = self.file._links(self)
        return self._link_cache

    def keys(self):
        return list(self.links().keys())

    def __contains__(self, path: str) -> bool:
        try:
            self[path]
        except KeyError:
            return False
        return True

    def __getitem__(self, path: str):
        node = self
        for part in [p for p in path.split("/") if p]:
            if not isinstance(node, Group):
                raise KeyError(path)
            links = node.links()
            if part not in links:
                raise KeyError(path)
            node = self.file._open(links[part], (node.name.rstrip("/") + "/" + part))
        return node


class Dataset(Node):
    def __init__(self, f, address, name):
        super().__init__(f, address, name)
        dt = self._first(0x03)
        ds = self._first(0x01)
        lay = self._first(0x08)
        if dt is None or ds is None or lay is None:
            raise HDF5FormatError("%s: dataset header lacks a datatype, dataspace or layout" % name)
        self.dtype, _ = _parse_datatype(f, f.buf, dt.pos)
        self.shape = _parse_dataspace(f, f.buf, ds.pos)
        self._layout = f._parse_layout(lay.pos)
        pipe = self._first(0x0B)
        self._filters = f._parse_filters(pipe.pos) if pipe is not None else []

    @property
    def size(self) -> int:
        return 0 if self.shape is None else int(np.prod(self.shape, dtype=np.int64))

    def contiguous_offset(self):
        """File offset of a contiguous, allocated, unfiltered dataset, else None."""
        kind = self._layout[0]
        if kind == "contiguous" and self._layout[1] is not None and not self._filters:
            return self._layout[1]
        return None

    def read(self):
        count = self.size
        nbytes = count * self.dtype.size
        kind = self._layout[0]
        if self.shape is None:
            return None
        if kind == "compact":
            raw = bytes(self.file.buf[self._layout[1]:self._layout[1] + nbytes])
        elif kind == "contiguous":
            addr = self._layout[1]
            if addr is None:
                raw = b"\0" * nbytes
            elif self.dtype.np_dtype is not None and self.dtype.cls in (0, 1, 4, 6):
                raw = self.file.buf[addr:addr + nbytes]
            else:
                raw = bytes(self.file.buf[addr:addr + nbytes])
        elif kind in ("chunked", "chunked-v1"):
            raw = self.file._read_chunked(self, nbytes)
        else:
            raise HDF5FormatError("%s: layout %s is not supported" % (self.name, kind))
        if len(raw) < nbytes:
            raise HDF5FormatError("%s: data runs past the end of the file" % self.name)
        arr = self.dtype.decode(self.file, raw, count)
        if isinstance(arr, np.ndarray):
            return arr.reshape(self.shape) if self.shape else arr.reshape(())[()]
        return arr if self.shape else arr[0]


class File(Group):
    """An open HDF5 file (memory-mapped, read-only)."""

    def __init__(self, path: str):
        self._fh = open(path, "rb")
        try:
            self.buf = mmap.mmap(self._fh.fileno(), 0, access=mmap.ACCESS_READ)
        except ValueError as exc:  # empty file
            self._fh.close()
            raise HDF5FormatError("%s: not an HDF5 file" % path) from exc
        self.path = path
        self._gheaps = {}
        root = self._superblock()
        Group.__init__(self, self, root, "/")

    def close(self):
        try:
            self.buf.close()
        finally:
            self._fh.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- primitive reads ---------------------------------------------------------------------

    def _unpack_addr(self, buf, pos):
        v = int.from_bytes(bytes(buf[pos:pos + self.size_of_offsets]), "little")
        if v == (1 << (8 * self.size_of_offsets)) - 1:
            return None
        return v + self.base_address

    def _len(self, pos):
        return int.from_bytes(bytes(self.buf[pos:pos + self.size_of_lengths]), "little")

    def _check(self, start, end, what):
        stored = struct.unpack_from("<I", self.buf, end)[0]
        if lookup3(self.buf[start:end]) != stored:
            raise HDF5FormatError("%s at %d: checksum mismatch" % (what, start))

    def _sig(self, pos, sig, what):
        if bytes(self.buf[pos:pos + 4]) != sig:
            raise HDF5FormatError("%s at %d: bad signature" % (what, pos))

    # ---- superblock ----------------------------------------------------------------------------

    def _superblock(self):
        start = None
        for off in [0] + [512 << i for i in range(24)]:
            if off + 8 > len(self.buf):
                break
            if bytes(self.buf[off:off + 8]) == _SIGNATURE:
                start = off
                break
        if start is None:
            raise HDF5FormatError("%s: not an HDF5 file" % self.path)
        b = self.buf
        version = b[start + 8]
        self.superblock_version = version
        if version in (0, 1):
            self.size_of_offsets = b[start + 13]
            self.size_of_lengths = b[start + 14]
            p = start + 24 + (4 if version == 1 else 0)
            self.base_address = 0
            base = int.from_bytes(bytes(b[p:p + self.size_of_offsets]), "little")
            self.base_address = base
            O = self.size_of_offsets
            p += 4 * O  # base, free-space, end-of-file, driver information
            root = self._unpack_addr(b, p + O)  # symbol table entry: link name offset, header
            return root
        if version in (2, 3):
            self.size_of_offsets = b[start + 9]
            self.size_of_lengths = b[start + 10]
            O = self.size_of_offsets
            p = start + 12
            self.base_address = 0
            self.base_address = int.from_bytes(bytes(b[p:p + O]), "little")
            root = self._unpack_addr(b, p + 3 * O)
            self._check(start, p + 4 * O, "superblock")
            return root
        raise HDF5FormatError("superblock version %d is not supported" % version)

    # ---- object headers ----------------------------------------------------------------------

    def _object_messages(self, address):
        b = self.buf
        msgs = []
        if bytes(b[address:address + 4]) == b"OHDR":
            version = b[address + 4]
            if version != 2:
                raise HDF5FormatError("object header version %d" % version)
            flags = b[address + 5]
            p = address + 6
            if flags & 0x20:
                p += 16
            if flags & 0x10:
                p += 4
            nsize = 1 << (flags & 3)
            chunk0 = int.from_bytes(bytes(b[p:p + nsize]), "little")
            p += nsize
            self._check(address, p + chunk0, "object header")
            blocks = [(p, p + chunk0)]
            order = bool(flags & 0x04)
            i = 0
            while i < len(blocks):
                s, e = blocks[i]
                q = s
                hdr = 6 if order else 4
                while q + hdr <= e:
                    mtype = b[q]
                    size = struct.unpack_from("<H", b, q + 1)[0]
                    mflags = b[q + 3]
                    q += hdr
                    if mtype == 0x10:
                        caddr = self._unpack_addr(b, q)
                        clen = int.from_bytes(
                            bytes(b[q + self.size_of_offsets:q + self.size_of_offsets
                                    + self.size_of_lengths]), "little")
                        self._sig(caddr, b"OCHK", "continuation block")
                        self._check(caddr, caddr + clen - 4, "continuation block")
                        blocks.append((caddr + 4, caddr + clen - 4))
                    elif mtype != 0:
                        msgs.append(_Message(mtype, mflags, q, size))
                    q += size
                i += 1
            return msgs
        version = b[address]
        if version != 1:
            raise HDF5FormatError("object header at %d: version %d" % (address, version))
        hsize = struct.unpack_from("<I", b, address + 8)[0]
        blocks = [(address + 16, address + 16 + hsize)]
        i = 0
        while i < len(blocks):
            s, e = blocks[i]
            q = s
            while q + 8 <= e:
                mtype, size, mflags = struct.unpack_from("<HHB", b, q)
                q += 8
                if mtype == 0x10:
                    caddr = self._unpack_addr(b, q)
                    clen = int.from_bytes(
                        bytes(b[q + self.size_of_offsets:q + self.size_of_offsets
                                + self.size_of_lengths]), "little")
                    blocks.append((caddr, caddr + clen))
                elif mtype != 0:
                    msgs.append(_Message(mtype, mflags, q, size))
                q += size
            i += 1
        return msgs

    def _open(self, address, name):
        msgs = self._object_messages(address)
        types = {m.type for m in msgs}
        if 0x08 in types:
            return Dataset(self, address, name)
        if types & {0x02, 0x06, 0x11, 0x0A} or not types - {0x0C, 0x15, 0x12, 0x16}:
            return Group(self, address, name)
        raise HDF5FormatError("%s: object is neither a group nor a dataset" % name)

    # ---- links ---------------------------------------------------------------------------------

    def _parse_link(self, buf, pos):
        version = buf[pos]
        if version != 1:
            raise HDF5FormatError("link message version %d" % version)
        flags = buf[pos + 1]
        p = pos + 2
        ltype = 0
        if flags & 0x08:
            ltype = buf[p]
            p += 1
        if flags & 0x04:
            p += 8
        if flags & 0x10:
            p += 1
        nlen_size = 1 << (flags & 3)
        nlen = int.from_bytes(bytes(buf[p:p + nlen_size]), "little")
        p += nlen_size
        name = bytes(buf[p:p + nlen]).decode("utf-8")
        p += nlen
        if ltype == 0:
            return name, self._unpack_addr(buf, p)
        return name, None  # soft and external links are not followed

    def _links(self, group: Group):
        links = {}
        stab = group._first(0x11)
        if stab is not None:
            btree = self._unpack_addr(self.buf, stab.pos)
            heap = self._unpack_addr(self.buf, stab.pos + self.size_of_offsets)
            self._symbol_table_links(btree, heap, links)
            return links
        for m in group.messages:
            if m.type == 0x06:
                name, addr = self._parse_link(self.buf, m.pos)
                if addr is not None:
                    links[name] = addr
        info = group._first(0x02)
        if info is not None:
            flags = self.buf[info.pos + 1]
            p = info.pos + 2 + (8 if flags & 1 else 0)
            heap = self._unpack_addr(self.buf, p)
            name_tree = self._unpack_addr(self.buf, p + self.size_of_offsets)
            if heap is not None and name_tree is not None:
                fh = _FractalHeap(self, heap)
                for rec in self._btree2_records(name_tree):
                    obj = fh.get(rec[4:])
                    name, addr = self._parse_link(obj, 0)
                    if addr is not None:
                        links[name] = addr
        return links

    def _local_heap(self, address):
        self._sig(address, b"HEAP", "local heap")
        L = self.size_of_lengths
        return self._unpack_addr(self.buf, address + 8 + 2 * L)

    def _symbol_table_links(self, btree, heap, links):
        data = self._local_heap(heap)
        b = self.buf
        O, L = self.size_of_offsets, self.size_of_lengths

        def name_at(off):
            end = bytes(b[data + off:data + off + 4096]).index(b"\0")
            return bytes(b[data + off:data + off + end]).decode("utf-8")

        def walk(node):
            self._sig(node, b"TREE", "group B-tree node")
            ntype, level = b[node + 4], b[node + 5]
            used = struct.unpack_from("<H", b, node + 6)[0]
            if ntype != 0:
                raise HDF5FormatError("group B-tree node of type %d" % ntype)
            p = node + 8 + 2 * O
            for i in range(used):
                child = self._unpack_addr(b, p + L + i * (L + O))
                if level > 0:
                    walk(child)
                else:
                    self._sig(child, b"SNOD", "symbol table node")
                    n = struct.unpack_from("<H", b, child + 6)[0]
                    q = child + 8
                    for _ in range(n):
                        name_off = int.from_bytes(bytes(b[q:q + O]), "little")
                        links[name_at(name_off)] = self._unpack_addr(b, q + O)
                        q += 2 * O + 24

        walk(btree)

    # ---- attributes ----------------------------------------------------------------------------

    def _parse_attribute(self, buf, pos):
        version = buf[pos]
        flags = buf[pos + 1]
        nsize, tsize, ssize = struct.unpack_from("<HHH", buf, pos + 2)
        if flags & 0x03 and version > 1:
            raise HDF5FormatError("shared attribute datatypes or dataspaces are not supported")
        if version == 1:
            p = pos + 8
            name = bytes(buf[p:p + nsize]).split(b"\0", 1)[0].decode("utf-8")
            p += (nsize + 7) // 8 * 8
            dt, _ = _parse_datatype(self, buf, p)
            p += (tsize + 7) // 8 * 8
            dims = _parse_dataspace(self, buf, p)
            p += (ssize + 7) // 8 * 8
        elif version in (2, 3):
            p = pos + 8 + (1 if version == 3 else 0)
            name = bytes(buf[p:p + nsize]).split(b"\0", 1)[0].decode("utf-8")
            p += nsize
            dt, _ = _parse_datatype(self, buf, p)
            p += tsize
            dims = _parse_dataspace(self, buf, p)
            p += ssize
        else:
            raise HDF5FormatError("attribute message version %d" % version)
        if dims is None:
            return name, None
        count = int(np.prod(dims, dtype=np.int64)) if dims else 1
        raw = bytes(buf[p:p + count * dt.size])
        value = dt.decode(self, raw, count)
        if isinstance(value, np.ndarray):
            value = value.reshape(dims) if dims else value.reshape(())[()]
        elif not dims:
            value = value[0]
        return name, value

    def _attributes(self, node: Node):
        attrs = {}
        for m in node.messages:
            if m.type == 0x0C:
                if m.flags & 0x02:
                    raise HDF5FormatError("shared attribute messages are not supported")
                name, value = self._parse_attribute(self.buf, m.pos)
                attrs[name] = value
        info = node._first(0x15)
        if info is not None:
            flags = self.buf[info.pos + 1]
            p = info.pos + 2 + (2 if flags & 1 else 0)
            heap = self._unpack_addr(self.buf, p)
            name_tree = self._unpack_addr(self.buf, p + self.size_of_offsets)
            if heap is not None and name_tree is not None:
                fh = _FractalHeap(self, heap)
                for rec in self._btree2_records(name_tree):
                    obj = fh.get(rec[:8])
                    name, value = self._parse_attribute(obj, 0)
                    attrs[name] = value
        return attrs

    # ---- version 2 B-trees ---------------------------------------------------------------------

    def _btree2_records(self, address):
        b = self.buf
        O = self.size_of_offsets
        self._sig(address, b"BTHD", "v2 B-tree header")
        node_size = struct.unpack_from("<I", b, address + 6)[0]
        rec_size = struct.unpack_from("<H", b, address + 10)[0]
        depth = struct.unpack_from("<H", b, address + 12)[0]
        p = address + 16
        root = self._unpack_addr(b, p)
        root_nrec = struct.unpack_from("<H", b, p + O)[0]
        self._check(address, p + O + 2 + self.size_of_lengths, "v2 B-tree header")
        # Per-depth record capacities, from which the field widths of child pointers follow.
        max_nrec = [(node_size - 10) // rec_size]
        cum_max = [max_nrec[0]]
        cum_size = [0]
        max_nrec_size = _limit_enc_size(max_nrec[0])
        for d in range(1, depth + 1):
            ptr = O + max_nrec_size + (cum_size[d - 1] if d > 1 else 0)
            m = (node_size - (10 + ptr)) // (rec_size + ptr)
            max_nrec.append(m)
            cum_max.append((m + 1) * cum_max[d - 1] + m)
            cum_size.append(_limit_enc_size(cum_max[d]))
        records = []

        def walk(addr, nrec, d):
            if addr is None:
                return
            if d == 0:
                self._sig(addr, b"BTLF", "v2 B-tree leaf")
                q = addr + 6
                for i in range(nrec):
                    records.append(bytes(b[q + i * rec_size:q + (i + 1) * rec_size]))
                self._check(addr, q + nrec * rec_size, "v2 B-tree leaf")
                return
            self._sig(addr, b"BTIN", "v2 B-tree internal node")
            q = addr + 6
            for i in range(nrec):
                records.append(bytes(b[q + i * rec_size:q + (i + 1) * rec_size]))
            q += nrec * rec_size
            children = []
            for _ in range(nrec + 1):
                caddr = self._unpack_addr(b, q)
                q += O
                cn = int.from_bytes(bytes(b[q:q + max_nrec_size]), "little")
                q += max_nrec_size
                if d > 1:
                    q += cum_size[d - 1]
                children.append((caddr, cn))
            self._check(addr, q, "v2 B-tree internal node")
            for caddr, cn in children:
                walk(caddr, cn, d - 1)

        walk(root, root_nrec, depth)
        return records

    # ---- global heap ---------------------------------------------------------------------------

    def _global_heap_object(self, address, index):
        objs = self._gheaps.get(address)
        if objs is None:
            self._sig(address, b"GCOL", "global heap collection")
            L = self.size_of_lengths
            size = self._len(address + 8)
            end = address + size
            p = address + 8 + L
            objs = {}
            while p + 8 + L <= end:
                idx = struct.unpack_from("<H", self.buf, p)[0]
                osize = self._len(p + 8)
                if idx == 0:
                    break
                objs[idx] = bytes(self.buf[p + 8 + L:p + 8 + L + osize])
                p += 8 + L + (osize + 7) // 8 * 8
            self._gheaps[address] = objs
        if index not in objs:
            raise HDF5FormatError("global heap object %d missing at %d" % (index, address))
        return objs[index]

    # ---- layouts and filters ---------------------------------------------------------------------

    def _parse_layout(self, pos):
        b = self.buf
        version = b[pos]
        O, L = self.size_of_offsets, self.size_of_lengths
        if version in (1, 2):
            ndims = b[pos + 1]
            cls = b[pos + 2]
            p = pos + 8
            addr = None
            if cls != 0:
                addr = self._unpack_addr(b, p)
                p += O
            dims = struct.unpack_from("<%dI" % ndims, b, p)
            p += 4 * ndims
            if cls == 0:
                size = struct.unpack_from("<I", b, p)[0]
                return ("compact", p + 4, size)
            if cls == 1:
                return ("contiguous", addr, None)
            return ("chunked-v1", addr, dims)
        if version in (3, 4):
            cls = b[pos + 1]
            p = pos + 2
            if cls == 0:
                size = struct.unpack_from("<H", b, p)[0]
                return ("compact", p + 2, size)
            if cls == 1:
                return ("contiguous", self._unpack_addr(b, p), self._len(p + O))
            if cls == 2 and version == 3:
                ndims = b[p]
                addr = self._unpack_addr(b, p + 1)
                dims = struct.unpack_from("<%dI" % ndims, b, p + 1 + O)
                return ("chunked", "btree1", addr, dims)
            if cls == 2:
                flags, ndims, enc = b[p], b[p + 1], b[p + 2]
                q = p + 3
                dims = tuple(int.from_bytes(bytes(b[q + i * enc:q + (i + 1) * enc]), "little")
                             for i in range(ndims))
                q += ndims * enc
                itype = b[q]
                q += 1
                if itype == 1:  # single chunk
                    fsize = fmask = None
                    if flags & 0x02:
                        fsize = self._len(q)
                        fmask = struct.unpack_from("<I", b, q + L)[0]
                        q += L + 4
                    return ("chunked", "single", self._unpack_addr(b, q), dims, fsize, fmask)
                if itype == 2:  # implicit
                    return ("chunked", "implicit", self._unpack_addr(b, q), dims)
                return ("chunked", "index%d" % itype, None, dims)
        raise HDF5FormatError("data layout version %d class %d is not supported"
                              % (version, b[pos + 1]))

    def _parse_filters(self, pos):
        b = self.buf
        version = b[pos]
        n = b[pos + 1]
        p = pos + (8 if version == 1 else 2)
        filters = []
        for _ in range(n):
            fid = struct.unpack_from("<H", b, p)[0]
            if version == 1 or fid >= 256:
                nlen = struct.unpack_from("<H", b, p + 2)[0]
                flags, ncd = struct.unpack_from("<HH", b, p + 4)
                p += 8 + ((nlen + 7) // 8 * 8 if version == 1 else nlen)
            else:
                flags, ncd = struct.unpack_from("<HH", b, p + 2)
                p += 6
            p += 4 * ncd
            if version == 1 and ncd % 2:
                p += 4
            filters.append((fid, flags))
        return filters

    def _unfilter(self, ds, data, mask):
        for i, (fid, _) in reversed(list(enumerate(ds._filters))):
            if mask & (1 << i):
                continue
            if fid == 1:
                data = zlib.decompress(data)
            elif fid == 2:  # shuffle
                n = ds.dtype.size
                arr = np.frombuffer(data, dtype=np.uint8)
                data = arr.reshape(n, -1).T.tobytes()
            else:
                raise HDF5FormatError("filter %d is not supported" % fid)
        return data

    def _read_chunked(self, ds, nbytes):
        lay = ds._layout
        shape = ds.shape
        esize = ds.dtype.size
        out = np.zeros(nbytes, dtype=np.uint8)
        if lay[1] == "single":
            addr, dims = lay[2], lay[3]
            if addr is None:
                return out.tobytes()
            csize = lay[4] if lay[4] is not None else int(np.prod(dims)) * esize
            data = self._unfilter(ds, bytes(self.buf[addr:addr + csize]), lay[5] or 0)
            chunks = [((0,) * len(shape), data)]
            cdims = dims
        elif lay[1] == "btree1" or lay[0] == "chunked-v1":
            addr, cdims = (lay[2], lay[3]) if lay[0] == "chunked" else (lay[1], lay[2])
            cdims = tuple(cdims[:len(shape)])
            chunks = []
            if addr is not None:
                self._chunk_btree1(ds, addr, len(shape), chunks)
        else:
            raise HDF5FormatError("%s: chunk index %s is not supported" % (ds.name, lay[1]))
        full = out.reshape(tuple(shape) + (esize,)) if shape else out
        for offs, data in chunks:
            chunk = np.frombuffer(data, dtype=np.uint8)[:int(np.prod(cdims)) * esize]
            chunk = chunk.reshape(tuple(cdims) + (esize,))
            sl_dst, sl_src = [], []
            for d, (o, c, n) in enumerate(zip(offs, cdims, shape)):
                hi = min(o + c, n)
                sl_dst.append(slice(o, hi))
                sl_src.append(slice(0, hi - o))
            full[tuple(sl_dst)] = chunk[tuple(sl_src)]
        return out.tobytes()

    def _chunk_btree1(self, ds, node, rank, chunks):
        b = self.buf
        O = self.size_of_offsets
        self._sig(node, b"TREE", "chunk B-tree node")
        ntype, level = b[node + 4], b[node + 5]
        used = struct.unpack_from("<H", b, node + 6)[0]
        if ntype != 1:
            raise HDF5FormatError("chunk B-tree node of type %d" % ntype)
        ksize = 8 + 8 * (rank + 1)
        p = node + 8 + 2 * O
        for i in range(used):
            kpos = p + i * (ksize + O)
            csize, mask = struct.unpack_from("<II", b, kpos)
            offs = struct.unpack_from("<%dQ" % rank, b, kpos + 8)
            child = self._unpack_addr(b, kpos + ksize)
            if level > 0:
                self._chunk_btree1(ds, child, rank, chunks)
            else:
                data = self._unfilter(ds, bytes(b[child:child + csize]), mask)
                chunks.append((offs, data))


class _FractalHeap:
    """Managed and tiny objects of a fractal heap (dense link and attribute storage)."""

    def __init__(self, f: File, address: int):
        self.f = f
        b = f.buf
        O, L = f.size_of_offsets, f.size_of_lengths
        f._sig(address, b"FRHP", "fractal heap header")
        self.id_len, self.filter_len = struct.unpack_from("<HH", b, address + 5)
        self.flags = b[address + 9]
        self.max_man = struct.unpack_from("<I", b, address + 10)[0]
        self.huge_tree = f._unpack_addr(b, address + 14 + L)
        self._huge = None
        p = address + 14 + L + O + L + O + 8 * L
        self.width = struct.unpack_from("<H", b, p)[0]
        self.start = f._len(p + 2)
        self.max_direct = f._len(p + 2 + L)
        self.max_heap_bits = struct.unpack_from("<H", b, p + 2 + 2 * L)[0]
        q = p + 2 + 2 * L + 4
        self.root = f._unpack_addr(b, q)
        self.root_rows = struct.unpack_from("<H", b, q + O)[0]
        end = q + O + 2
        if self.filter_len:
            raise HDF5FormatError("filtered fractal heaps are not supported")
        f._check(address, end, "fractal heap header")
        self.off_size = (self.max_heap_bits + 7) // 8
        dblk_off = (self.max_direct.bit_length() - 1 + 7) // 8
        self.len_size = min(dblk_off, _limit_enc_size(self.max_man))
        self.max_dblock_rows = (self.max_direct.bit_length() - self.start.bit_length()) + 2

    def _row_size(self, r):
        return self.start if r < 2 else self.start << (r - 1)

    def get(self, heap_id: bytes) -> bytes:
        flag = heap_id[0]
        kind = (flag >> 4) & 3
        if kind == 2:  # tiny
            if self.id_len <= 18:
                n = (flag & 0x0F) + 1
                return bytes(heap_id[1:1 + n])
            n = (((flag & 0x0F) << 8) | heap_id[1]) + 1
            return bytes(heap_id[2:2 + n])
        if kind == 1:
            return self._huge_object(heap_id)
        if kind != 0:
            raise HDF5FormatError("fractal heap ID of unknown type")
        off = int.from_bytes(bytes(heap_id[1:1 + self.off_size]), "little")
        length = int.from_bytes(
            bytes(heap_id[1 + self.off_size:1 + self.off_size + self.len_size]), "little")
        return self._read(off, length)

    def _huge_object(self, heap_id):
        """Objects above the managed-size limit live outside the heap blocks: the ID holds their
        address and length directly when it is wide enough, else a key into the heap's v2 B-tree
        of huge objects (record type 1: address, length, ID)."""
        f = self.f
        O, L = f.size_of_offsets, f.size_of_lengths
        if self.id_len >= 1 + O + L:
            addr = f._unpack_addr(heap_id, 1)
            length = int.from_bytes(bytes(heap_id[1 + O:1 + O + L]), "little")
        else:
            if self._huge is None:
                if self.huge_tree is None:
                    raise HDF5FormatError("huge fractal heap object without its B-tree")
                self._huge = {}
                for rec in f._btree2_records(self.huge_tree):
                    if len(rec) != O + 2 * L:
                        raise HDF5FormatError("filtered huge fractal heap objects are not supported")
                    key = int.from_bytes(rec[O + L:O + 2 * L], "little")
                    self._huge[key] = (f._unpack_addr(rec, 0),
                                       int.from_bytes(rec[O:O + L], "little"))
            key = int.from_bytes(bytes(heap_id[1:1 + min(self.id_len - 1, L)]), "little")
            if key not in self._huge:
                raise HDF5FormatError("huge fractal heap object %d not indexed" % key)
            addr, length = self._huge[key]
        return bytes(f.buf[addr:addr + length])

    def _read(self, off, length):
        if self.root_rows == 0:
            return self._from_direct(self.root, 0, self.start, off, length)
        return self._from_indirect(self.root, 0, self.root_rows, off, length)

    def _from_direct(self, addr, block_off, size, off, length):
        b = self.f.buf
        self.f._sig(addr, b"FHDB", "fractal heap direct block")
        if self.flags & 0x02:
            hdr = 5 + self.f.size_of_offsets + self.off_size
            stored = struct.unpack_from("<I", b, addr + hdr)[0]
            image = bytearray(b[addr:addr + size])
            image[hdr:hdr + 4] = b"\0\0\0\0"
            if lookup3(bytes(image)) != stored:
                raise HDF5FormatError("fractal heap direct block at %d: checksum mismatch" % addr)
        rel = off - block_off
        if rel < 0 or rel + length > size:
            raise HDF5FormatError("fractal heap object outside its direct block")
        return bytes(b[addr + rel:addr + rel + length])

    def _from_indirect(self, addr, block_off, nrows, off, length):
        f = self.f
        b = f.buf
        O = f.size_of_offsets
        f._sig(addr, b"FHIB", "fractal heap indirect block")
        p = addr + 5 + O + self.off_size
        ndirect = min(nrows, self.max_dblock_rows) * self.width
        nindirect = max(nrows - self.max_dblock_rows, 0) * self.width
        f._check(addr, p + (ndirect + nindirect) * O, "fractal heap indirect block")
        child_off = block_off
        entry = 0
        for r in range(nrows):
            size = self._row_size(r)
            for _ in range(self.width):
                if child_off <= off < child_off + size:
                    caddr = f._unpack_addr(b, p + entry * O)
                    if caddr is None:
                        raise HDF5FormatError("fractal heap object in an unallocated block")
                    if r < self.max_dblock_rows:
                        return self._from_direct(caddr, child_off, size, off, length)
                    rows = (size.bit_length() - (self.start * self.width).bit_length()) + 1
                    return self._from_indirect(caddr, child_off, rows, off, length)
                child_off += size
                entry += 1
        raise HDF5FormatError("fractal heap offset %d outside the heap" % off)


def open_file(path: str) -> File:
    """Open an HDF5 file for reading."""
    return File(path)


# --------------------------------------------------------------------------------------------
# Writer: superblock 2, version 2 object headers, compact links and attributes, contiguous
# datasets.  Enough for operator bundles; read back by the reader above.
# --------------------------------------------------------------------------------------------

_UNDEF = b"\xff" * 8


class WGroup:
    """A group to be written: ``attrs`` (name -> value) and ``children`` (name -> WGroup or
    array).  Values are str, bool, int, float, or numpy arrays of integer, float64 or complex128
    type; arrays are written with their numpy (C-order) shape as the HDF5 dimensions."""

    def __init__(self):
        self.attrs = {}
        self.children = {}

    def create_group(self, name: str) -> "WGroup":
        g = WGroup()
        self.children[name] = g
        return g


def _w_datatype(value):
    """(datatype message bytes, element bytes encoder) for a value or array."""
    if isinstance(value, str):
        raw = value.encode("utf-8") + b"\0"
        return (bytes([0x13, 0x10, 0, 0]) + struct.pack("<I", len(raw))), raw
    arr = np.asarray(value)
    if arr.dtype == np.bool_:
        arr = arr.astype(np.uint8)
    kind, size = arr.dtype.kind, arr.dtype.itemsize
    if kind in "iu":
        dt = (bytes([0x10, 0x08 if kind == "i" else 0, 0, 0]) + struct.pack("<I", size)
              + struct.pack("<HH", 0, 8 * size))
        return dt, np.ascontiguousarray(arr, dtype=arr.dtype.newbyteorder("<")).tobytes()
    if kind == "f" and size == 8:
        return _F64, np.ascontiguousarray(arr, dtype="<f8").tobytes()
    if kind == "c" and size == 16:
        dt = (bytes([0x36, 2, 0, 0]) + struct.pack("<I", 16) + b"r\0" + b"\x00" + _F64
              + b"i\0" + b"\x08" + _F64)
        return dt, np.ascontiguousarray(arr, dtype="<c16").tobytes()
    raise HDF5FormatError("cannot write values of type %s" % arr.dtype)


_F64 = (bytes([0x11, 0x20, 63, 0]) + struct.pack("<I", 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11,
                                                                        0, 52, 1023))


def _w_dataspace(shape):
    return (bytes([2, len(shape), 0, 1 if shape else 0])
            + b"".join(struct.pack("<Q", int(d)) for d in shape))


def _w_message(mtype, data, flags=0):
    return struct.pack("<BHB", mtype, len(data), flags) + data


def _w_attribute(name, value):
    dt, raw = _w_datatype(value)
    shape = () if isinstance(value, str) or np.ndim(value) == 0 else np.shape(value)
    ds = _w_dataspace(shape)
    nm = name.encode("utf-8") + b"\0"
    return _w_message(0x0C, bytes([3, 0]) + struct.pack("<HHH", len(nm), len(dt), len(ds))
                      + b"\x01" + nm + dt + ds + raw)


class _Writer:
    def __init__(self):
        self.buf = bytearray(48)  # superblock, filled last

    def _put(self, data: bytes) -> int:
        while len(self.buf) % 8:
            self.buf.append(0)
        addr = len(self.buf)
        self.buf += data
        return addr

    def _header(self, messages) -> int:
        body = b"".join(messages)
        head = b"OHDR" + bytes([2, 0x02]) + struct.pack("<I", len(body)) + body
        return self._put(head + struct.pack("<I", lookup3(head)))

    def dataset(self, value, attrs) -> int:
        dt, raw = _w_datatype(value)
        shape = np.shape(value)
        addr = self._put(raw) if raw else None
        layout = (bytes([3, 1]) + (struct.pack("<Q", addr) if addr is not None else _UNDEF)
                  + struct.pack("<Q", len(raw)))
        msgs = [_w_message(0x01, _w_dataspace(shape)), _w_message(0x03, dt, 1),
                _w_message(0x05, bytes([3, 0x0A]), 1), _w_message(0x08, layout)]
        msgs += [_w_attribute(k, v) for k, v in attrs.items()]
        return self._header(msgs)

    def group(self, g: WGroup) -> int:
        links = []
        for name, child in g.children.items():
            addr = self.group(child) if isinstance(child, WGroup) else self.dataset(child, {})
            nm = name.encode("utf-8")
            if len(nm) < 256:
                links.append(_w_message(0x06, bytes([1, 0, len(nm)]) + nm + struct.pack("<Q", addr)))
            else:
                links.append(_w_message(0x06, bytes([1, 1]) + struct.pack("<H", len(nm)) + nm
                                        + struct.pack("<Q", addr)))
        msgs = [_w_message(0x02, bytes([0, 0]) + _UNDEF + _UNDEF), _w_message(0x0A, bytes([0, 0]))]
        msgs += links + [_w_attribute(k, v) for k, v in g.attrs.items()]
        return self._header(msgs)


def write_file(path: str, root: WGroup) -> None:
    """Write ``root`` and everything below it as a new HDF5 file."""
    w = _Writer()
    root_addr = w.group(root)
    sb = (_SIGNATURE + bytes([2, 8, 8, 0]) + struct.pack("<Q", 0) + _UNDEF
          + struct.pack("<Q", len(w.buf)) + struct.pack("<Q", root_addr))
    w.buf[0:48] = sb + struct.pack("<I", lookup3(sb))
    with open(path, "wb") as fh:
        fh.write(bytes(w.buf))
