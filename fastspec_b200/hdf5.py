"""Line lists in FastSpec's HDF5 layout, without an HDF5 library.

The reference reads its line lists from HDF5 files with one group /Lines holding one 1-D dataset per
column (ReadHDF, ioutils.f90:524-1159; written by python/vald2hdf.py and python/mol2hdf.py of the
reference): atomic lists {EL (fixed-length string), ION (int16), W (float64), E, LGGF, GRAD, GQST, GVDW
(float32)} plus JLO/JUP/GLO/GUP (float32) for Zeeman lists and ISOT (int16) for unscaled isotopes;
molecular single-species lists {W, E, LGGF, GRAD}.  Group attributes: NL, NAME, ID, ION, WL_VAC, HFLAG,
FILE, DATE, PROVENANCE, FORMAT_VERSION, WMIN, WMAX; each dataset carries a UNIT string.

Neither h5py nor libhdf5 is available here, so this module restates the parts of the published HDF5
file format (version 0 superblock) that these files use:

* reading: the version 0 superblock, version 1 object headers with continuation blocks, symbol-table
  groups (version 1 B-tree of group nodes, symbol-table nodes, local heap), dataspace, datatype
  (fixed-point, floating-point, fixed-length string), data layout version 3 (compact, contiguous,
  chunked with a version 1 B-tree of chunk nodes), the filter pipeline (deflate, shuffle, fletcher32
  skipped) and attribute messages (versions 1-3);
* writing: the same structures with contiguous, unfiltered datasets, which any HDF5 reader accepts
  (the reference program reads them; ``tests/golden/make_atmospheres.py`` checks that).

All multi-byte fields are little-endian, offsets and lengths 8 bytes.
"""
import struct
import zlib

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"


class HDF5Error(ValueError):
    """The file is not an HDF5 file of the supported subset."""


# ============================================================================================
# reading
# ============================================================================================

class _Reader:
    def __init__(self, path):
        with open(path, "rb") as f:
            self.b = f.read()
        if self.b[:8] != SIGNATURE:
            raise HDF5Error("%s: not an HDF5 file" % path)
        sb = self.b[8]
        if sb not in (0, 1):
            raise HDF5Error("%s: superblock version %d (only 0 and 1 are read)" % (path, sb))
        self.so, self.sl = self.b[13], self.b[14]
        if self.so != 8 or self.sl != 8:
            raise HDF5Error("offset/length sizes %d/%d (only 8/8 are read)" % (self.so, self.sl))
        p = 24 + (4 if sb == 1 else 0)
        self.base = self._u(p, 8)
        p += 32                                     # base, free-space, end-of-file, driver addresses
        self.root = self._entry(p)

    def _u(self, p, n):
        return int.from_bytes(self.b[p:p + n], "little")

    def _entry(self, p):
        """Symbol table entry: (name offset in the local heap, object header address, cache type,
        scratch B-tree address, scratch heap address)."""
        name, oh, cache = self._u(p, 8), self._u(p + 8, 8), self._u(p + 16, 4)
        bt, hp = (self._u(p + 24, 8), self._u(p + 32, 8)) if cache == 1 else (None, None)
        return dict(name=name, header=oh, cache=cache, btree=bt, heap=hp)

    # ---- object headers --------------------------------------------------------------------
    def messages(self, addr):
        """(type, flags, bytes) of every message of the version 1 object header at addr."""
        b = self.b
        if b[addr] != 1:
            raise HDF5Error("object header version %d at %d (only 1 is read)" % (b[addr], addr))
        nmsg = self._u(addr + 2, 2)
        size = self._u(addr + 8, 4)
        blocks = [(addr + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            p, n = blocks.pop(0)
            end = p + n
            while p + 8 <= end and len(out) < nmsg:
                mt, ms, mf = self._u(p, 2), self._u(p + 2, 2), b[p + 4]
                data = b[p + 8:p + 8 + ms]
                p += 8 + ms
                if mt == 0x10:                       # continuation: another block of messages
                    blocks.append(struct.unpack_from("<QQ", data))
                out.append((mt, mf, data))
        return out

    # ---- groups ----------------------------------------------------------------------------
    def _heap_string(self, heap, off):
        if self.b[heap:heap + 4] != b"HEAP":
            raise HDF5Error("local heap signature missing")
        data = self._u(heap + 24, 8)
        s = data + off
        e = self.b.index(b"\x00", s)
        return self.b[s:e].decode("ascii")

    def group_members(self, btree, heap):
        """name -> object header address of the links of a symbol-table group."""
        out = {}
        self._walk_group(btree, heap, out)
        return out

    def _walk_group(self, node, heap, out):
        b = self.b
        if b[node:node + 4] != b"TREE" or b[node + 4] != 0:
            raise HDF5Error("group B-tree node expected at %d" % node)
        level, used = b[node + 5], self._u(node + 6, 2)
        p = node + 24 + 8                            # past the header and key 0
        for _ in range(used):
            child = self._u(p, 8)
            p += 16                                  # child address, next key
            if level > 0:
                self._walk_group(child, heap, out)
                continue
            if b[child:child + 4] != b"SNOD":
                raise HDF5Error("symbol-table node expected at %d" % child)
            nsym = self._u(child + 6, 2)
            for k in range(nsym):
                e = self._entry(child + 8 + 40 * k)
                out[self._heap_string(heap, e["name"])] = e["header"]

    def group(self, addr):
        for mt, _, d in self.messages(addr):
            if mt == 0x11:
                bt, hp = struct.unpack_from("<QQ", d)
                return self.group_members(bt, hp)
        raise HDF5Error("object at %d is not a symbol-table group" % addr)

    # ---- datatypes, dataspaces, values -----------------------------------------------------
    @staticmethod
    def dtype(d):
        cls, ver = d[0] & 0x0F, d[0] >> 4
        bits = d[1] | (d[2] << 8) | (d[3] << 16)
        size = struct.unpack_from("<I", d, 4)[0]
        order = ">" if bits & 1 else "<"
        if cls == 0:
            return np.dtype("%s%s%d" % (order, "i" if bits & 8 else "u", size)), 12
        if cls == 1:
            if size not in (4, 8):
                raise HDF5Error("float of %d bytes" % size)
            return np.dtype("%sf%d" % (order, size)), 20
        if cls == 3:
            return np.dtype("S%d" % size), 8
        raise HDF5Error("datatype class %d (version %d) is not read" % (cls, ver))

    @staticmethod
    def dataspace(d):
        ver, rank, flags = d[0], d[1], d[2]
        if ver == 1:
            p = 8
        elif ver == 2:
            p = 4
            if d[3] == 0:
                return ()
        else:
            raise HDF5Error("dataspace version %d" % ver)
        dims = struct.unpack_from("<%dQ" % rank, d, p)
        return tuple(int(x) for x in dims)

    def attributes(self, addr):
        out = {}
        for mt, _, d in self.messages(addr):
            if mt != 0x0C:
                continue
            ver = d[0]
            nlen, tlen, slen = struct.unpack_from("<HHH", d, 2)
            if ver == 1:
                pad = lambda n: (n + 7) & ~7
                p = 8
                name = d[p:p + nlen].rstrip(b"\x00").decode("ascii"); p += pad(nlen)
                dt, _ = self.dtype(d[p:p + tlen]); p += pad(tlen)
                shape = self.dataspace(d[p:p + slen]); p += pad(slen)
            elif ver in (2, 3):
                p = 8 if ver == 2 else 9
                name = d[p:p + nlen].rstrip(b"\x00").decode("ascii"); p += nlen
                dt, _ = self.dtype(d[p:p + tlen]); p += tlen
                shape = self.dataspace(d[p:p + slen]); p += slen
            else:
                raise HDF5Error("attribute message version %d" % ver)
            n = int(np.prod(shape)) if shape else 1
            v = np.frombuffer(d, dtype=dt, count=n, offset=p)
            if dt.kind == "S":
                v = [x.split(b"\x00")[0].decode("ascii", "replace") for x in v]
                out[name] = v[0] if not shape or n == 1 else v
            else:
                out[name] = v[0].item() if not shape or n == 1 else v.copy()
        return out

    def dataset(self, addr):
        dt = shape = layout = None
        filters = []
        for mt, _, d in self.messages(addr):
            if mt == 0x01:
                shape = self.dataspace(d)
            elif mt == 0x03:
                dt, _ = self.dtype(d)
            elif mt == 0x08:
                layout = d
            elif mt == 0x0B:
                filters = self._filters(d)
        if dt is None or shape is None or layout is None:
            raise HDF5Error("object at %d is not a dataset" % addr)
        n = int(np.prod(shape)) if shape else 1
        if layout[0] != 3:
            raise HDF5Error("data layout version %d (only 3 is read)" % layout[0])
        cls = layout[1]
        if cls == 0:                                 # compact
            size = struct.unpack_from("<H", layout, 2)[0]
            raw = layout[4:4 + size]
        elif cls == 1:                               # contiguous
            a, size = struct.unpack_from("<QQ", layout, 2)
            raw = b"" if a == UNDEF else self.b[a:a + size]
        elif cls == 2:                               # chunked
            rank = layout[2]
            bt = struct.unpack_from("<Q", layout, 3)[0]
            cdims = struct.unpack_from("<%dI" % rank, layout, 11)
            if rank != 2:
                raise HDF5Error("chunked datasets of rank %d are not read" % (rank - 1))
            return self._chunked(bt, cdims[0], dt, n, filters).reshape(shape)
        else:
            raise HDF5Error("layout class %d" % cls)
        if len(raw) < n * dt.itemsize:               # never written: the fill value (zero)
            return np.zeros(shape, dt)
        return np.frombuffer(raw, dtype=dt, count=n).reshape(shape).copy()

    @staticmethod
    def _filters(d):
        ver, nf = d[0], d[1]
        p = 8 if ver == 1 else 2
        out = []
        for _ in range(nf):
            if ver == 1:
                fid, nlen, flags, ncd = struct.unpack_from("<HHHH", d, p)
                p += 8 + ((nlen + 7) & ~7)
            else:
                fid = struct.unpack_from("<H", d, p)[0]
                if fid < 256:
                    flags, ncd = struct.unpack_from("<HH", d, p + 2)
                    p += 6
                else:
                    nlen, flags, ncd = struct.unpack_from("<HHH", d, p + 2)
                    p += 8 + nlen
            cd = struct.unpack_from("<%dI" % ncd, d, p)
            p += 4 * ncd
            if ver == 1 and ncd % 2:
                p += 4
            out.append((fid, cd))
        return out

    def _chunked(self, bt, chunk, dt, n, filters):
        out = np.zeros(n, dt)
        raw = out.view(np.uint8)
        for off, size, mask, addr in self._chunks(bt):
            data = self.b[addr:addr + size]
            for i in reversed(range(len(filters))):
                if mask & (1 << i):
                    continue
                fid, cd = filters[i]
                if fid == 1:                          # deflate
                    data = zlib.decompress(data)
                elif fid == 2:                        # shuffle: bytes transposed by element
                    s = dt.itemsize
                    m = len(data) // s
                    data = np.frombuffer(data[:m * s], np.uint8).reshape(s, m).T.tobytes() + data[m * s:]
                elif fid == 3:                        # fletcher32: trailing checksum, not verified
                    data = data[:-4]
                else:
                    raise HDF5Error("filter %d is not supported" % fid)
            e0 = off
            cnt = min(chunk, n - e0)
            if cnt > 0:
                raw[e0 * dt.itemsize:(e0 + cnt) * dt.itemsize] = np.frombuffer(data[:cnt * dt.itemsize], np.uint8)
        return out

    def _chunks(self, node):
        b = self.b
        if b[node:node + 4] != b"TREE" or b[node + 4] != 1:
            raise HDF5Error("chunk B-tree node expected at %d" % node)
        level, used = b[node + 5], self._u(node + 6, 2)
        ksize = 8 + 8 * 2                            # chunk size, filter mask, offsets (rank 1 + element)
        p = node + 24
        for _ in range(used):
            size, mask = struct.unpack_from("<II", b, p)
            off = struct.unpack_from("<Q", b, p + 8)[0]
            child = self._u(p + ksize, 8)
            p += ksize + 8
            if level > 0:
                yield from self._chunks(child)
            else:
                yield off, size, mask, child


def read_lines(path):
    """(columns, attributes, units) of the /Lines group of a FastSpec HDF5 line list: numpy arrays by
    column name (EL decoded to str), the group attributes, and each column's UNIT attribute.  A file
    cut short, or with damaged structures, raises HDF5Error."""
    try:
        return _read_lines(path)
    except HDF5Error:
        raise
    except (struct.error, IndexError, zlib.error, ValueError, KeyError) as e:
        raise HDF5Error("%s: truncated or damaged HDF5 file (%s: %s)" % (path, type(e).__name__, e)) from None


def _read_lines(path):
    r = _Reader(path)
    top = r.group(r.root["header"])
    if "Lines" not in top:
        raise HDF5Error("%s: no /Lines group" % path)
    g = top["Lines"]
    members = r.group(g)
    cols, units = {}, {}
    for name, addr in members.items():
        a = r.dataset(addr)
        if a.dtype.kind == "S":
            a = np.array([x.split(b"\x00")[0].decode("ascii") for x in a])
        cols[name] = a
        units[name] = r.attributes(addr).get("UNIT")
    return cols, r.attributes(g), units


# ============================================================================================
# writing
# ============================================================================================

def _pad8(b):
    return b + b"\x00" * (-len(b) % 8)


def _dtype_msg(dt):
    dt = np.dtype(dt)
    if dt.kind in "iu":
        bits = 0x08 if dt.kind == "i" else 0
        return struct.pack("<B3sI", 0x10, bytes([bits, 0, 0]), dt.itemsize) + struct.pack("<HH", 0, 8 * dt.itemsize)
    if dt.kind == "f":
        if dt.itemsize == 4:
            fields = bytes([0x20, 31, 0]), (0, 32, 23, 8, 0, 23, 127)
        else:
            fields = bytes([0x20, 63, 0]), (0, 64, 52, 11, 0, 52, 1023)
        return (struct.pack("<B3sI", 0x11, fields[0], dt.itemsize) +
                struct.pack("<HHBBBBI", *fields[1]))
    if dt.kind == "S":                                # null-terminated ASCII
        return struct.pack("<B3sI", 0x13, bytes([0, 0, 0]), dt.itemsize)
    raise HDF5Error("cannot write dtype %s" % dt)


def _space_msg(n):
    if n is None:                                     # scalar
        return struct.pack("<BBBBI", 1, 0, 0, 0, 0)
    return struct.pack("<BBBBIQQ", 1, 1, 1, 0, 0, n, n)


def _msg(mtype, data, flags=0):
    data = _pad8(data)
    return struct.pack("<HHB3x", mtype, len(data), flags) + data


def _attr_msg(name, value):
    if isinstance(value, str):
        raw = value.encode("ascii") + b"\x00"
        dt, data, n = np.dtype("S%d" % len(raw)), raw, None
    else:
        v = np.asarray(value)
        dt, data, n = v.dtype, v.tobytes(), None if v.ndim == 0 else v.size
    nm = name.encode("ascii") + b"\x00"
    t, s = _dtype_msg(dt), _space_msg(n)
    body = struct.pack("<BBHHH", 1, 0, len(nm), len(t), len(s)) + _pad8(nm) + _pad8(t) + _pad8(s) + data
    return _msg(0x0C, body)


class _Writer:
    def __init__(self):
        self.buf = bytearray(b"\x00" * 96)            # superblock, filled at the end

    def put(self, data, align=8):
        self.buf += b"\x00" * (-len(self.buf) % align)
        a = len(self.buf)
        self.buf += data
        return a

    def header(self, msgs):
        body = b"".join(msgs)
        return self.put(struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body)

    def group(self, members):
        """Symbol-table group of the given {name: object header address}; returns (header address,
        B-tree address, heap address).  One symbol-table node holds every link (leaf K = 32)."""
        names = sorted(members)
        heap = bytearray(b"\x00" * 8)                # offset 0: the empty name
        offs = {}
        for nm in names:
            offs[nm] = len(heap)
            heap += _pad8(nm.encode("ascii") + b"\x00")
        heap_data = self.put(bytes(heap))
        # no free block: the free-list head is 1 (the HDF5 library's end-of-free-list marker)
        heap_addr = self.put(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), 1, heap_data))
        ents = b"".join(struct.pack("<QQI4x16x", offs[nm], members[nm], 0) for nm in names)
        ents += b"\x00" * (40 * (64 - len(names)))
        snod = self.put(b"SNOD" + struct.pack("<BBH", 1, 0, len(names)) + ents)
        key_hi = offs[names[-1]] if names else 0
        tree = self.put(b"TREE" + struct.pack("<BBHQQ", 0, 0, 1, UNDEF, UNDEF) +
                        struct.pack("<QQQ", 0, snod, key_hi) + b"\x00" * (8 * 2 * 64))
        return tree, heap_addr

    def finish(self, root_header, root_tree, root_heap):
        sb = SIGNATURE + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, 32, 16, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, len(self.buf), UNDEF)
        sb += struct.pack("<QQI4xQQ", 0, root_header, 1, root_tree, root_heap)
        assert len(sb) == 96
        self.buf[:96] = sb
        return bytes(self.buf)


def write_lines(path, columns, attrs, units=None):
    """Write a FastSpec line list: group /Lines with one contiguous 1-D dataset per column (numpy
    arrays of equal length; str arrays become fixed-length ASCII) and the group attributes (str,
    numpy scalars or arrays)."""
    w = _Writer()
    members = {}
    n = None
    for name, col in columns.items():
        a = np.asarray(col)
        if a.dtype.kind == "U":
            a = np.char.encode(a, "ascii")
            a = a.astype("S%d" % (max(1, a.dtype.itemsize) + 1))
        a = np.ascontiguousarray(a, a.dtype.newbyteorder("<") if a.dtype.kind in "iuf" else a.dtype)
        if n is None:
            n = len(a)
        elif len(a) != n:
            raise HDF5Error("column %s has %d rows, not %d" % (name, len(a), n))
        data_addr = w.put(a.tobytes(), align=16) if n else UNDEF
        msgs = [_msg(0x01, _space_msg(n)), _msg(0x03, _dtype_msg(a.dtype), flags=1),
                _msg(0x05, struct.pack("<BBBB", 2, 1, 1, 0)),   # fill value: early allocation, never written
                _msg(0x08, struct.pack("<BBQQ", 3, 1, data_addr, a.nbytes))]
        if units and name in units:
            msgs.append(_attr_msg("UNIT", units[name]))
        members[name] = w.header(msgs)
    tree, heap = w.group(members)
    gmsgs = [_msg(0x11, struct.pack("<QQ", tree, heap))] + [_attr_msg(k, v) for k, v in attrs.items()]
    lines_hdr = w.header(gmsgs)
    rtree, rheap = w.group({"Lines": lines_hdr})
    root = w.header([_msg(0x11, struct.pack("<QQ", rtree, rheap))])
    with open(path, "wb") as f:
        f.write(w.finish(root, rtree, rheap))
