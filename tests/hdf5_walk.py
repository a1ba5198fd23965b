"""A second, independent reading of the HDF5 structures that checkpoint files
use (test helper): superblock versions 0-1, the root group as a symbol table
(version-1 B-tree of type 0, symbol-table nodes, local heap), version-1
object headers with continuation blocks, dataspace versions 1-2, datatype
class 1 and layout versions 1-3.  It follows the HDF5 file format
specification directly, in Python, so that it shares no code with the
library's C reader, and it returns what it saw (every message of every
header) for the structure tests.
"""
from __future__ import annotations

import struct

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5:
    def __init__(self, path: str):
        with open(path, "rb") as f:
            self.b = f.read()
        off = 0
        while self.b[off:off + 8] != SIG:
            off = 512 if off == 0 else 2 * off
            if off + 8 > len(self.b):
                raise ValueError("no superblock")
        self.sb_off = off
        sb = self.b[off:]
        self.sb_version = sb[8]
        if self.sb_version > 1:
            raise ValueError("superblock version")
        self.size_off, self.size_len = sb[13], sb[14]
        assert self.size_off == 8 and self.size_len == 8
        self.leaf_k, self.internal_k = struct.unpack_from("<HH", sb, 16)
        self.flags = struct.unpack_from("<I", sb, 20)[0]
        a = 24 if self.sb_version == 0 else 28
        self.base, self.freespace, self.eof, self.driver = struct.unpack_from("<4Q", sb, a)
        e = a + 32
        self.root_name_off, self.root_header, self.root_cache = struct.unpack_from("<QQI", sb, e)
        self.root_scratch = struct.unpack_from("<QQ", sb, e + 24)
        self.root = self.header(self.root_header)
        stab = [m for m in self.root["messages"] if m[0] == 0x11]
        assert len(stab) == 1, "root group without a symbol table"
        self.btree, self.heap_addr = struct.unpack_from("<QQ", stab[0][2])
        self.heap = self.local_heap(self.heap_addr)
        self.links = {}
        self.snods = []
        self.walk(self.btree)

    def at(self, addr: int, n: int) -> bytes:
        a = self.base + addr
        if addr == UNDEF or a + n > len(self.b):
            raise ValueError(f"address {addr} + {n} outside the file")
        return self.b[a:a + n]

    def local_heap(self, addr: int) -> dict:
        h = self.at(addr, 32)
        assert h[:4] == b"HEAP" and h[4] == 0
        size, free, data = struct.unpack_from("<QQQ", h, 8)
        return {"size": size, "free": free, "data_addr": data, "data": self.at(data, size)}

    def name(self, off: int) -> str:
        d = self.heap["data"]
        return d[off:d.index(b"\0", off)].decode()

    def walk(self, addr: int) -> None:
        node = self.at(addr, 24)
        assert node[:4] == b"TREE" and node[4] == 0, "not a group B-tree node"
        level, used = node[5], struct.unpack_from("<H", node, 6)[0]
        body = self.at(addr + 24, 16 * used + 8)
        keys = [struct.unpack_from("<Q", body, 16 * i)[0] for i in range(used + 1)]
        kids = [struct.unpack_from("<Q", body, 16 * i + 8)[0] for i in range(used)]
        for c in kids:
            if level > 0:
                self.walk(c)
                continue
            s = self.at(c, 8)
            assert s[:4] == b"SNOD" and s[4] == 1
            n = struct.unpack_from("<H", s, 6)[0]
            names = []
            for i in range(n):
                off, hdr, cache = struct.unpack_from("<QQI", self.at(c + 8 + 40 * i, 40))
                names.append(self.name(off))
                self.links[self.name(off)] = hdr
            self.snods.append({"addr": c, "names": names, "keys": [self.name(k) for k in keys]})

    def header(self, addr: int) -> dict:
        p = self.at(addr, 16)
        version, nmsg, refcount, size = p[0], *struct.unpack_from("<HII", p, 2)
        assert version == 1, "only version-1 object headers"
        msgs, chunks = [], [(addr + 16, size)]
        while chunks and len(msgs) < nmsg:
            a, n = chunks.pop(0)
            blk = self.at(a, n)
            pos = 0
            while pos + 8 <= n and len(msgs) < nmsg:
                t, ln, fl = struct.unpack_from("<HHB", blk, pos)
                body = blk[pos + 8:pos + 8 + ln]
                if t == 0x10:
                    chunks.append(struct.unpack_from("<QQ", body))
                msgs.append((t, fl, body))
                pos += 8 + ln
        return {"version": version, "nmsg": nmsg, "refcount": refcount, "size": size, "messages": msgs}

    def dataset(self, name: str) -> tuple[np.ndarray, dict]:
        h = self.header(self.links[name])
        msgs = {t: body for t, _, body in h["messages"]}
        sp = msgs[0x01]
        rank = sp[1]
        off = 8 if sp[0] == 1 else 4
        dims = struct.unpack_from(f"<{rank}Q", sp, off)
        dt = msgs[0x03]
        assert dt[0] & 0x0F == 1 and struct.unpack_from("<I", dt, 4)[0] == 8 and not dt[1] & 1
        lay = msgs[0x08]
        if lay[0] == 3:
            assert lay[1] == 1, "contiguous layout only"
            addr, size = struct.unpack_from("<QQ", lay, 2)
        else:
            nd = lay[1]
            addr = struct.unpack_from("<Q", lay, 8)[0]
            size = int(np.prod(struct.unpack_from(f"<{nd}I", lay, 16)))
        data = np.frombuffer(self.at(addr, size), "<f8").reshape(dims)
        return data, h
