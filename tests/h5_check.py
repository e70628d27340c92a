"""A second, independent reader of the HDF5 subset the library writes and
reads (superblock 0, symbol-table root group, version-1 object headers,
contiguous and chunked/deflate datasets, version-1 attributes), written in
Python from the published file format specification. Tests run it on the
files the library writes and on files written by the HDF5 library itself,
so that the library's own writer and reader are not only checked against
each other."""
import struct
import zlib

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


def _u(b, at, n):
    return int.from_bytes(b[at:at + n], "little")


def _dtype(d):
    cls, size = d[0] & 0x0F, _u(d, 4, 4)
    if d[1] & 1:
        raise ValueError("big-endian")
    if cls == 1:
        return np.dtype({4: "<f4", 8: "<f8"}[size])
    if cls == 0:
        signed = bool(d[1] & 0x08)
        return np.dtype(("<i" if signed else "<u") + str(size))
    if cls == 4:
        return np.dtype("<u" + str(size))
    raise ValueError(f"class {cls}")


def _space(d):
    ver, rank = d[0], d[1]
    at = 8 if ver == 1 else 4
    return tuple(_u(d, at + 8 * i, 8) for i in range(rank))


class H5:
    def __init__(self, path):
        self.b = open(path, "rb").read()
        b = self.b
        assert b[:8] == SIG, "signature"
        self.superblock = dict(version=b[8], offset_size=b[13], length_size=b[14], leaf_k=_u(b, 16, 2),
                               internal_k=_u(b, 18, 2), base=_u(b, 24, 8), eof=_u(b, 40, 8))
        assert self.superblock["version"] == 0 and b[13] == 8 and b[14] == 8
        assert self.superblock["eof"] == len(b), "end-of-file address"
        root = _u(b, 64, 8)
        msgs = self.messages(root)
        st = [d for t, d in msgs if t == 0x11][0]
        btree, heap = _u(st, 0, 8), _u(st, 8, 8)
        assert b[heap:heap + 4] == b"HEAP"
        hsize, free, hdata = _u(b, heap + 8, 8), _u(b, heap + 16, 8), _u(b, heap + 24, 8)
        self.heap = dict(size=hsize, free=free, data=hdata)
        assert free == 1 or free < hsize, "heap free list"
        self.entries = {}
        stack = [btree]
        while stack:
            node = stack.pop()
            assert b[node:node + 4] == b"TREE" and b[node + 4] == 0
            level, used = b[node + 5], _u(b, node + 6, 2)
            for i in range(used):
                child = _u(b, node + 24 + 8 + 16 * i, 8)
                if level:
                    stack.append(child)
                    continue
                assert b[child:child + 4] == b"SNOD"
                names = []
                for k in range(_u(b, child + 6, 2)):
                    e = child + 8 + 40 * k
                    off = _u(b, e, 8)
                    nm = b[hdata + off: b.index(b"\0", hdata + off)].decode()
                    names.append(nm)
                    self.entries[nm] = _u(b, e + 8, 8)
                assert names == sorted(names), "symbol-table entries in name order"

    def messages(self, at):
        b = self.b
        assert b[at] == 1, "object header version 1"
        n, size = _u(b, at + 2, 2), _u(b, at + 8, 4)
        blocks, out = [(at + 16, size)], []
        for start, length in blocks:
            p = start
            while p + 8 <= start + length and len(out) < n:
                t, s = _u(b, p, 2), _u(b, p + 2, 2)
                assert s % 8 == 0, "message sizes are multiples of 8 in version-1 headers"
                d = b[p + 8:p + 8 + s]
                out.append((t, d))
                if t == 0x10:
                    blocks.append((_u(d, 0, 8), _u(d, 8, 8)))
                p += 8 + s
        return out

    def dataset(self, name):
        msgs = self.messages(self.entries[name])
        dt = _dtype([d for t, d in msgs if t == 3][0])
        shape = _space([d for t, d in msgs if t == 1][0])
        lay = [d for t, d in msgs if t == 8][0]
        filt = [d for t, d in msgs if t == 0x0B]
        assert lay[0] == 3
        count = int(np.prod(shape)) if shape else 1
        if lay[1] == 1:
            addr, size = _u(lay, 2, 8), _u(lay, 10, 8)
            assert size == count * dt.itemsize
            if size == 0:
                return np.zeros(shape, dt)
            return np.frombuffer(self.b[addr:addr + size], dt).reshape(shape).copy()
        assert lay[1] == 2
        r1 = lay[2]
        addr = _u(lay, 3, 8)
        chunk = tuple(_u(lay, 11 + 4 * i, 4) for i in range(r1 - 1))
        ids = []
        if filt:
            d = filt[0]
            assert d[0] == 1
            p = 8
            for _ in range(d[1]):
                fid, nl, nv = _u(d, p, 2), _u(d, p + 2, 2), _u(d, p + 6, 2)
                ids.append(fid)
                p += 8 + ((nl + 7) // 8) * 8 + 4 * nv + (4 if nv % 2 else 0)
        out = np.zeros(shape, dt)
        self._chunks(addr, len(shape), chunk, dt, ids, out)
        return out

    def _chunks(self, node, rank, chunk, dt, ids, out):
        b = self.b
        assert b[node:node + 4] == b"TREE" and b[node + 4] == 1
        level, used = b[node + 5], _u(b, node + 6, 2)
        key = 8 + 8 * (rank + 1)
        p = node + 24
        for _ in range(used):
            size, mask = _u(b, p, 4), _u(b, p + 4, 4)
            off = [_u(b, p + 8 + 8 * k, 8) for k in range(rank)]
            child = _u(b, p + key, 8)
            if level:
                self._chunks(child, rank, chunk, dt, ids, out)
            else:
                raw = b[child:child + size]
                for k in reversed(range(len(ids))):
                    if mask & (1 << k):
                        continue
                    assert ids[k] == 1, "deflate only"
                    raw = zlib.decompress(raw)
                a = np.frombuffer(raw, dt).reshape(chunk)
                sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(off, chunk, out.shape))
                out[sl] = a[tuple(slice(0, s.stop - s.start) for s in sl)]
            p += key + 8

    def attrs(self, name):
        res = {}
        for t, d in self.messages(self.entries[name]):
            if t != 0x0C:
                continue
            assert d[0] == 1
            nl, tl, sl = _u(d, 2, 2), _u(d, 4, 2), _u(d, 6, 2)
            pad = lambda x: (x + 7) // 8 * 8
            p = 8
            nm = d[p:p + nl].rstrip(b"\0").decode()
            p += pad(nl)
            dt = _dtype(d[p:p + tl])
            p += pad(tl)
            shape = _space(d[p:p + sl])
            p += pad(sl)
            cnt = int(np.prod(shape)) if shape else 1
            res[nm] = np.frombuffer(d[p:p + cnt * dt.itemsize], dt).copy()
        return res
