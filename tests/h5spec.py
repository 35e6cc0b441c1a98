"""An independent HDF5 reader for the tests, written in Python from the public HDF5 file
format specification: it parses the subset the library writes (superblock version 0,
version-1 object headers, symbol-table groups, contiguous datasets, version-1 attribute
messages) and asserts the structural rules a libhdf5 reader relies on while it parses:
signature and versions, message sizes multiples of 8, the message count of each header,
the local heap's free-list head, sorted symbol-table entries, B-tree keys bracketing the
names, contiguous storage exactly the dataspace times the element size, and the
end-of-file address equal to the file size.

read(path) -> {"/group/name": numpy array (structured for compounds), ...,
               "/group@attr": numpy array, ...}
"""
import struct

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class Corrupt(AssertionError):
    pass


def _check(cond, what):
    if not cond:
        raise Corrupt(what)


def _u(b, off, n):
    return int.from_bytes(b[off:off + n], "little")


def _dtype(b, off):
    """(numpy dtype, bytes used) of a datatype message at b[off:]."""
    cls, ver = b[off] & 15, b[off] >> 4
    bits = b[off + 1:off + 4]
    size = _u(b, off + 4, 4)
    if cls == 1:
        _check(ver == 1, "float datatype version")
        _check(bits[0] & 1 == 0, "little-endian float")
        _check(bits[0] & 0x30 == 0x20, "implied-msb mantissa")
        _check(bits[1] == size * 8 - 1, "sign bit position")
        bo, prec, eloc, esz, mloc, msz, bias = struct.unpack_from("<HHBBBBI", b, off + 8)
        want = {8: (0, 64, 52, 11, 0, 52, 1023), 4: (0, 32, 23, 8, 0, 23, 127)}[size]
        _check((bo, prec, eloc, esz, mloc, msz, bias) == want, "IEEE float properties")
        return np.dtype("<f%d" % size), 20
    if cls == 0:
        _check(size == 4 and bits[0] == 0x08, "32-bit signed little-endian integer")
        _check(struct.unpack_from("<HH", b, off + 8) == (0, 32), "integer bit offset / precision")
        return np.dtype("<i4"), 12
    _check(cls == 6 and ver == 1, "compound datatype version 1")
    nm = bits[0] | bits[1] << 8
    q = off + 8
    names, formats, offsets = [], [], []
    for _ in range(nm):
        end = b.index(b"\0", q)
        name = b[q:end].decode()
        q += ((end - q) + 8) // 8 * 8
        moff = _u(b, q, 4)
        _check(b[q + 4] == 0, "no member array dimensions")
        q += 32
        mt, used = _dtype(b, q)
        q += used
        names.append(name)
        formats.append(mt)
        offsets.append(moff)
    dt = np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": size})
    return dt, q - off


def _space(b, off):
    _check(b[off] == 1, "dataspace version 1")
    rank = b[off + 1]
    _check(b[off + 2] == 0, "no maximum dimensions")
    return tuple(_u(b, off + 8 + 8 * i, 8) for i in range(rank))


def _header(b, addr):
    _check(b[addr] == 1, "object header version 1")
    nmsgs = _u(b, addr + 2, 2)
    _check(_u(b, addr + 4, 4) >= 1, "reference count")
    size = _u(b, addr + 8, 4)
    p, end, msgs = addr + 16, addr + 16 + size, []
    while p < end:
        typ, ln = _u(b, p, 2), _u(b, p + 2, 2)
        _check(ln % 8 == 0, "message size a multiple of 8")
        msgs.append((typ, p + 8, ln))
        p += 8 + ln
    _check(p == end, "messages fill the header exactly")
    _check(len(msgs) == nmsgs, "message count")
    return msgs


def _heap(b, addr):
    _check(b[addr:addr + 4] == b"HEAP" and b[addr + 4] == 0, "local heap")
    size, free, data = _u(b, addr + 8, 8), _u(b, addr + 16, 8), _u(b, addr + 24, 8)
    _check(free == 1 or free < size, "free-list head (1 = none)")
    _check(b[data] == 0, "offset 0 holds the empty name")
    return data, size


def _name(b, data, off):
    return b[data + off:b.index(b"\0", data + off)].decode()


def _group(b, btree, heap):
    data, _ = _heap(b, heap)
    _check(b[btree:btree + 4] == b"TREE" and b[btree + 4] == 0, "group B-tree node")
    level, used = b[btree + 5], _u(b, btree + 6, 2)
    _check(level == 0, "one-level group B-tree")
    out = {}
    for i in range(used):
        k0 = _u(b, btree + 24 + 16 * i, 8)
        snod = _u(b, btree + 32 + 16 * i, 8)
        k1 = _u(b, btree + 40 + 16 * i, 8)
        _check(b[snod:snod + 4] == b"SNOD" and b[snod + 4] == 1, "symbol-table node version 1")
        ns = _u(b, snod + 6, 2)
        names = []
        for e in range(ns):
            ent = snod + 8 + 40 * e
            name = _name(b, data, _u(b, ent, 8))
            names.append(name)
            out[name] = (_u(b, ent + 8, 8), _u(b, ent + 16, 4), _u(b, ent + 24, 8), _u(b, ent + 32, 8))
        _check(names == sorted(names, key=lambda s: s.encode()), "entries sorted by name")
        _check(_name(b, data, k0) < names[0] if names else True, "left key below the first name")
        _check(_name(b, data, k1) == names[-1], "right key = the last name")
    return out


def _object(b, addr, path, out):
    msgs = _header(b, addr)
    types = [m[0] for m in msgs]
    for typ, off, ln in msgs:
        if typ == 12:  # attribute, version 1
            _check(b[off] == 1, "attribute version 1")
            nlen, tlen, slen = _u(b, off + 2, 2), _u(b, off + 4, 2), _u(b, off + 6, 2)
            q = off + 8
            name = b[q:q + nlen - 1].decode()
            _check(b[q + nlen - 1] == 0, "attribute name terminated")
            q += (nlen + 7) // 8 * 8
            dt, used = _dtype(b, q)
            _check(used == tlen, "attribute datatype size")
            q += (tlen + 7) // 8 * 8
            shape = _space(b, q)
            q += (slen + 7) // 8 * 8
            n = int(np.prod(shape)) if shape else 1
            out[path + "@" + name] = np.frombuffer(b, dt, n, q).reshape(shape)
    if 17 in types:
        _, off, _ = msgs[types.index(17)]
        btree, heap = _u(b, off, 8), _u(b, off + 8, 8)
        for name, (oh, cache, sb, sh) in _group(b, btree, heap).items():
            sub = _header(b, oh)
            if any(t == 17 for t, _, _ in sub):
                _check(cache == 1, "group entries cache their B-tree and heap")
                o = next(x for x in sub if x[0] == 17)[1]
                _check((sb, sh) == (_u(b, o, 8), _u(b, o + 8, 8)), "cached addresses match")
            _object(b, oh, path.rstrip("/") + "/" + name, out)
        return
    _check(1 in types and 3 in types and 8 in types, "dataset: dataspace, datatype, layout")
    shape = _space(b, msgs[types.index(1)][1])
    dt, _ = _dtype(b, msgs[types.index(3)][1])
    off = msgs[types.index(8)][1]
    _check(b[off] == 3 and b[off + 1] == 1, "layout version 3, contiguous")
    addr_, size = _u(b, off + 2, 8), _u(b, off + 10, 8)
    _check(size == int(np.prod(shape)) * dt.itemsize, "storage = elements x element size")
    _check(addr_ + size <= len(b), "data inside the file")
    out[path] = np.frombuffer(b, dt, int(np.prod(shape)), addr_).reshape(shape)


def read(path):
    with open(path, "rb") as f:
        b = f.read()
    _check(b[:8] == SIG, "signature")
    _check(tuple(b[8:16]) == (0, 0, 0, 0, 0, 8, 8, 0), "superblock version 0, 8-byte offsets")
    _check(_u(b, 16, 2) > 0 and _u(b, 18, 2) > 0, "group K values")
    base, free, eof, drv = struct.unpack_from("<4Q", b, 24)
    _check(base == 0 and free == UNDEF and drv == UNDEF, "base / free-space / driver addresses")
    _check(eof == len(b), "end-of-file address = file size")
    root = _u(b, 64, 8)
    _check(_u(b, 72, 4) == 1, "root entry caches its symbol table")
    out = {}
    _object(b, root, "/", out)
    return out
