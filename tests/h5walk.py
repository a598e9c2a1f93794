"""A second, independent reader of the HDF5 subset state files use, written
in Python from the HDF5 file-format specification (superblock v0/v1, v1
object headers, symbol-table groups, v1 B-trees, contiguous and chunked
layouts with shuffle / deflate / Blosc filters). Test infrastructure only:
it cross-checks libopendynamo's writer field by field (signatures, sizes,
addresses, end-of-file) and locates chunks so tests can rewrite them.
"""

from __future__ import annotations

import ctypes
import struct
import zlib

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIG = b"\x89HDF\r\n\x1a\n"


class Walker:
    def __init__(self, data: bytes):
        self.b = data
        assert self.b[:8] == SIG, "signature"
        self.sb_version = self.b[8]
        assert self.sb_version in (0, 1)
        assert self.b[13] == 8 and self.b[14] == 8, "offset/length sizes"
        self.leaf_k, self.internal_k = struct.unpack_from("<HH", self.b, 16)
        off = 24 if self.sb_version == 0 else 28
        self.base, self.freespace, self.eof, self.driver = struct.unpack_from("<QQQQ", self.b, off)
        self.root_entry = off + 32
        _, self.root_ohdr = struct.unpack_from("<QQ", self.b, self.root_entry)

    # --- object headers
    def messages(self, addr):
        ver, _, n, _, size = struct.unpack_from("<BBHII", self.b, addr)
        assert ver == 1, f"object header version {ver}"
        out, blocks = [], [(addr + 16, size)]
        while blocks and len(out) < n:
            p, sz = blocks.pop(0)
            end = p + sz
            while p + 8 <= end and len(out) < n:
                mtype, msz, flags = struct.unpack_from("<HHB", self.b, p)
                assert msz % 8 == 0, "v1 message sizes are multiples of 8"
                body = self.b[p + 8:p + 8 + msz]
                if mtype == 0x10:
                    blocks.append(struct.unpack_from("<QQ", body, 0))
                out.append((mtype, body))
                p += 8 + msz
            assert p == end or len(out) == n
        assert len(out) == n
        return out

    def attributes(self, addr):
        out = {}
        for mtype, body in self.messages(addr):
            if mtype != 0x0C:
                continue
            ver, _, nl, dl, sl = struct.unpack_from("<BBHHH", body, 0)
            assert ver == 1
            pad = lambda x: (x + 7) // 8 * 8
            p = 8
            name = body[p:p + nl].rstrip(b"\0").decode()
            p += pad(nl)
            dt = body[p:p + dl]
            p += pad(dl)
            ds = body[p:p + sl]
            p += pad(sl)
            cls = dt[0] & 0x0F
            size = struct.unpack_from("<I", dt, 4)[0]
            assert ds[1] == 0, "scalar dataspace"
            raw = body[p:p + size]
            if cls == 0:
                assert size == 8 and dt[1] & 0x08 == 0  # unsigned
                val = struct.unpack("<Q", raw)[0]
            elif cls == 1:
                assert size == 8
                val = struct.unpack("<d", raw)[0]
            elif cls == 3:
                val = raw.rstrip(b"\0").decode()
            else:
                raise AssertionError(f"attribute class {cls}")
            out[name] = (cls, size, val)
        return out

    # --- groups
    def group_members(self, ohdr):
        stab = [body for t, body in self.messages(ohdr) if t == 0x11]
        assert len(stab) == 1
        btree, heap = struct.unpack_from("<QQ", stab[0], 0)
        assert self.b[heap:heap + 4] == b"HEAP"
        dsize, free, daddr = struct.unpack_from("<QQQ", self.b, heap + 8)
        assert daddr + dsize <= self.eof
        names = self.b[daddr:daddr + dsize]
        assert names[0] == 0, "heap offset 0 holds the empty name"
        out = {}
        self._group_node(btree, names, out)
        return out

    def _group_node(self, addr, names, out):
        assert self.b[addr:addr + 4] == b"TREE" and self.b[addr + 4] == 0
        level = self.b[addr + 5]
        used = struct.unpack_from("<H", self.b, addr + 6)[0]
        assert 1 <= used <= 2 * self.internal_k
        p = addr + 24
        keys, kids = [], []
        for i in range(used):
            keys.append(struct.unpack_from("<Q", self.b, p)[0])
            kids.append(struct.unpack_from("<Q", self.b, p + 8)[0])
            p += 16
        keys.append(struct.unpack_from("<Q", self.b, p)[0])
        for kid in kids:
            if level:
                self._group_node(kid, names, out)
                continue
            assert self.b[kid:kid + 4] == b"SNOD" and self.b[kid + 4] == 1
            ns = struct.unpack_from("<H", self.b, kid + 6)[0]
            assert 1 <= ns <= 2 * self.leaf_k
            prev = ""
            for k in range(ns):
                e = kid + 8 + 40 * k
                noff, oh, cache = struct.unpack_from("<QQI", self.b, e)
                name = names[noff:names.index(b"\0", noff)].decode()
                assert name > prev, "symbol table entries are sorted"
                prev = name
                out[name] = oh
            last = names[keys[-1]:names.index(b"\0", keys[-1])].decode()
            assert last == prev, "right key names the last member"

    # --- datasets
    def dataset(self, ohdr):
        info = {"filters": []}
        for t, body in self.messages(ohdr):
            if t == 0x01:
                ver, rank, flags = body[0], body[1], body[2]
                assert ver == 1 and 1 <= rank <= 3
                dims = struct.unpack_from(f"<{rank}Q", body, 8)
                if flags & 1:
                    assert struct.unpack_from(f"<{rank}Q", body, 8 + 8 * rank) == dims, "fixed size"
                info["dims"] = dims
                info["n"] = int(np.prod(dims))
            elif t == 0x03:
                assert body[0] == 0x11, "float class, version 1"
                info["size"] = struct.unpack_from("<I", body, 4)[0]
                off, prec, eloc, esz, mloc, msz, bias = struct.unpack_from("<HHBBBBI", body, 8)
                assert (prec, eloc, esz, msz, bias) in ((32, 23, 8, 23, 127), (64, 52, 11, 52, 1023))
                assert body[1] == 0x20 and body[2] == prec - 1
            elif t == 0x08:
                assert body[0] == 3
                info["layout"] = body[1]
                if body[1] == 1:
                    info["addr"], info["bytes"] = struct.unpack_from("<QQ", body, 2)
                else:
                    nd = body[2]
                    info["btree"] = struct.unpack_from("<Q", body, 3)[0]
                    *cd, info["esize"] = struct.unpack_from(f"<{nd}I", body, 11)
                    info["cdims"] = tuple(cd)
                    info["chunk"] = int(np.prod(cd))
            elif t == 0x0B:
                assert body[0] == 1
                nf = body[1]
                p = 8
                for _ in range(nf):
                    fid, nl, fl, ncv = struct.unpack_from("<HHHH", body, p)
                    p += 8 + (nl + 7) // 8 * 8
                    cv = list(struct.unpack_from(f"<{ncv}I", body, p))
                    p += 4 * ncv + (4 if ncv % 2 else 0)
                    info["filters"].append((fid, cv))
        return info

    def chunks(self, btree, rank=1):
        """[(element offset, address, size, mask, key position)] of a chunk
        index; the offset is a tuple of `rank` element offsets for rank > 1.
        Checks that the keys are increasing (row-major) and that every node's
        closing key lies beyond its last child."""
        out = []
        self._chunk_node(btree, out, rank)
        for a, b in zip(out, out[1:]):
            ka = a[0] if rank > 1 else (a[0],)
            kb = b[0] if rank > 1 else (b[0],)
            assert ka < kb, "chunk keys in row-major order"
        return out

    def _chunk_node(self, addr, out, rank):
        assert self.b[addr:addr + 4] == b"TREE" and self.b[addr + 4] == 1
        level = self.b[addr + 5]
        used = struct.unpack_from("<H", self.b, addr + 6)[0]
        ksz = 8 + 8 * (rank + 1)
        p = addr + 24
        first = len(out)
        for i in range(used):
            size, mask = struct.unpack_from("<II", self.b, p)
            offs = struct.unpack_from(f"<{rank + 1}Q", self.b, p + 8)
            child = struct.unpack_from("<Q", self.b, p + ksz)[0]
            assert offs[-1] == 0
            if level:
                self._chunk_node(child, out, rank)
            else:
                assert child + size <= self.eof
                out.append((offs[0] if rank == 1 else tuple(offs[:rank]), child, size, mask, p))
            p += ksz + 8
        closing = struct.unpack_from(f"<{rank + 1}Q", self.b, p + 8)[:rank]
        last = out[-1][0] if rank > 1 else (out[-1][0],)
        assert len(out) > first and tuple(closing) > tuple(last), "closing key beyond the last child"

    def _decode(self, info, raw):
        es = info["size"]
        for k, (fid, cv) in reversed(list(enumerate(info["filters"]))):
            if info.get("mask", 0) & (1 << k):
                continue
            if fid == 1:
                raw = zlib.decompress(raw)
            elif fid == 2:
                raw = _unshuffle(raw, es)
            elif fid == 32001:
                raw = blosc_decode(raw)
            else:
                raise AssertionError(f"filter {fid}")
        return raw

    def read_array(self, ohdr):
        """A float dataset of rank 1 to 3 as a numpy array of its dims."""
        info = self.dataset(ohdr)
        es, dims = info["size"], info["dims"]
        dt = np.float32 if es == 4 else np.float64
        if info["layout"] == 1:
            return np.frombuffer(self.b[info["addr"]:info["addr"] + info["n"] * es], dtype=dt).reshape(dims).copy()
        rank = len(dims)
        cd = info["cdims"]
        out = np.zeros(dims, dt)
        for off, addr, size, mask, _ in self.chunks(info["btree"], rank):
            off = off if rank > 1 else (off,)
            raw = self._decode(dict(info, mask=mask), self.b[addr:addr + size])
            assert len(raw) == int(np.prod(cd)) * es, "whole chunks"
            blk = np.frombuffer(raw, dtype=dt).reshape(cd)
            sl = tuple(slice(o, min(o + c, d)) for o, c, d in zip(off, cd, dims))
            out[sl] = blk[tuple(slice(0, s.stop - s.start) for s in sl)]
        return out

    def read_plane(self, ohdr):
        info = self.dataset(ohdr)
        es, n = info["size"], info["n"]
        if info["layout"] == 1:
            assert info["bytes"] == n * es
            return self.b[info["addr"]:info["addr"] + n * es]
        out = bytearray(n * es)
        for off, addr, size, mask, _ in self.chunks(info["btree"]):
            raw = self.b[addr:addr + size]
            for k, (fid, cv) in reversed(list(enumerate(info["filters"]))):
                if mask & (1 << k):
                    continue
                if fid == 1:
                    raw = zlib.decompress(raw)
                elif fid == 2:
                    raw = _unshuffle(raw, es)
                elif fid == 32001:
                    raw = blosc_decode(raw)
                else:
                    raise AssertionError(f"filter {fid}")
            cnt = min(info["chunk"], n - off)
            out[off * es:(off + cnt) * es] = raw[:cnt * es]
        return bytes(out)


def _shuffle(raw: bytes, es: int) -> bytes:
    ne = len(raw) // es
    a = np.frombuffer(raw[:ne * es], np.uint8).reshape(ne, es)
    return a.T.tobytes() + raw[ne * es:]


def _unshuffle(raw: bytes, es: int) -> bytes:
    ne = len(raw) // es
    a = np.frombuffer(raw[:ne * es], np.uint8).reshape(es, ne)
    return a.T.tobytes() + raw[ne * es:]


def _codec(name):
    return ctypes.CDLL(name)


def blosc_decode(frame: bytes) -> bytes:
    """c-blosc 1.x frame decoder (split and unsplit blocks, lz4 / zstd)."""
    flags, ts = frame[2], frame[3]
    nbytes, bsize, ctbytes = struct.unpack_from("<III", frame, 4)
    assert ctbytes == len(frame)
    if flags & 0x2:
        return frame[16:16 + nbytes]
    codec = flags >> 5
    nblocks = (nbytes + bsize - 1) // bsize
    out = bytearray(nbytes)
    for bi in range(nblocks):
        bs = min(bsize, nbytes - bi * bsize)
        leftover = bs < bsize
        split = not (flags & 0x10) and not leftover and ts <= 16 and bsize // ts >= 128
        ns = ts if split else 1
        neb = bs // ns
        pos = struct.unpack_from("<I", frame, 16 + 4 * bi)[0]
        tmp = bytearray()
        for _ in range(ns):
            cs = struct.unpack_from("<I", frame, pos)[0]
            pos += 4
            src = frame[pos:pos + cs]
            pos += cs
            if cs == neb:
                tmp += src
            elif codec == 1:
                dst = ctypes.create_string_buffer(neb)
                r = _codec("liblz4.so.1").LZ4_decompress_safe(src, dst, cs, neb)
                assert r == neb
                tmp += dst.raw
            elif codec == 4:
                dst = ctypes.create_string_buffer(neb)
                z = _codec("libzstd.so.1")
                z.ZSTD_decompress.restype = ctypes.c_size_t
                r = z.ZSTD_decompress(dst, ctypes.c_size_t(neb), src, ctypes.c_size_t(cs))
                assert r == neb
                tmp += dst.raw
            else:
                raise AssertionError(f"codec {codec}")
        if flags & 0x1:
            tmp = _unshuffle(bytes(tmp), ts)
        out[bi * bsize:bi * bsize + bs] = tmp
    return bytes(out)


def blosc_encode_split(data: bytes, typesize: int, codec: str = "lz4", blocksize: int = 1 << 14) -> bytes:
    """c-blosc 1.x frame with byte shuffle and split streams (one per byte
    of the type), the layout c-blosc writes by default for typesize <= 16."""
    nbytes = len(data)
    nblocks = (nbytes + blocksize - 1) // blocksize
    code = {"lz4": 1, "zstd": 4}[codec]
    body = bytearray()
    starts = []
    hdr_len = 16 + 4 * nblocks
    for bi in range(nblocks):
        blk = data[bi * blocksize:(bi + 1) * blocksize]
        bs = len(blk)
        ne = bs // typesize
        sh = _shuffle(bytes(blk), typesize)
        leftover = bs < blocksize
        ns = typesize if (not leftover and blocksize // typesize >= 128) else 1
        neb = bs // ns
        starts.append(hdr_len + len(body))
        for s in range(ns):
            src = sh[s * neb:(s + 1) * neb]
            if codec == "lz4":
                lib = _codec("liblz4.so.1")
                cap = lib.LZ4_compressBound(neb)
                dst = ctypes.create_string_buffer(cap)
                cs = lib.LZ4_compress_default(src, dst, neb, cap)
            else:
                lib = _codec("libzstd.so.1")
                lib.ZSTD_compressBound.restype = ctypes.c_size_t
                lib.ZSTD_compress.restype = ctypes.c_size_t
                cap = lib.ZSTD_compressBound(ctypes.c_size_t(neb))
                dst = ctypes.create_string_buffer(cap)
                cs = lib.ZSTD_compress(dst, ctypes.c_size_t(cap), src, ctypes.c_size_t(neb), 3)
            if 0 < cs < neb:
                body += struct.pack("<I", cs) + dst.raw[:cs]
            else:
                body += struct.pack("<I", neb) + src
    flags = 0x1 | (code << 5)
    frame = struct.pack("<BBBBIII", 2, 1, flags, typesize, nbytes, blocksize, hdr_len + len(body))
    frame += b"".join(struct.pack("<I", s) for s in starts) + bytes(body)
    return frame
