"""Test infrastructure: a reader of the part of the HDF5 file format that
mp_hdf5_* write, following the published HDF5 file format specification
(version 0 superblock; a group stored as a symbol table: version 1 B-tree of
group nodes, symbol table nodes "SNOD", local heap "HEAP"; version 1 object
headers with dataspace, datatype, fill value and layout messages; contiguous
storage).  No HDF5 library is installed here, so the tests read the files
with this and check every structural field they can: signatures, versions,
sizes, sorted names, addresses inside the file.  It is not the HDF5 library:
compatibility with it is argued from the specification, not tested."""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"


class FormatError(AssertionError):
    pass


def _check(cond, msg):
    if not cond:
        raise FormatError(msg)


class Reader:
    def __init__(self, path: str):
        with open(path, "rb") as f:
            self.b = f.read()
        self._superblock()

    def u(self, off, n):
        _check(0 <= off and off + n <= len(self.b), f"read of {n} bytes at {off} outside the file ({len(self.b)})")
        return int.from_bytes(self.b[off:off + n], "little")

    def _superblock(self):
        b = self.b
        _check(b[:8] == SIGNATURE, "superblock signature")
        _check(b[8] == 0, "superblock version 0")
        _check(b[9] == 0 and b[10] == 0 and b[12] == 0, "free-space, root entry and shared header versions 0")
        _check(b[13] == 8 and b[14] == 8, "8-byte offsets and lengths")
        self.leaf_k, self.internal_k = self.u(16, 2), self.u(18, 2)
        _check(self.leaf_k > 0 and self.internal_k > 0, "group K values")
        _check(self.u(24, 8) == 0, "base address 0")
        _check(self.u(32, 8) == UNDEF and self.u(48, 8) == UNDEF, "no free-space info, no driver block")
        _check(self.u(40, 8) == len(b), "end-of-file address equals the file size")
        # root group symbol table entry
        self.root_header = self.u(64, 8)
        _check(self.u(72, 4) == 1, "root entry caches its symbol table")
        self.btree, self.heap = self.u(80, 8), self.u(88, 8)

    def _heap(self):
        h = self.heap
        _check(self.b[h:h + 4] == b"HEAP" and self.b[h + 4] == 0, "local heap signature and version")
        size, free, data = self.u(h + 8, 8), self.u(h + 16, 8), self.u(h + 24, 8)
        _check(free == 1 or free < size, "local heap free list head")
        _check(self.b[data] == 0, "heap offset 0 holds the empty string")
        return data, size

    def name_at(self, off):
        data, size = self._heap()
        _check(off < size, "heap offset inside the data segment")
        end = self.b.index(b"\0", data + off)
        return self.b[data + off:end].decode()

    def _object_messages(self, addr):
        b = self.b
        _check(b[addr] == 1, "object header version 1")
        nmsg, _ref, size = self.u(addr + 2, 2), self.u(addr + 4, 4), self.u(addr + 8, 4)
        p, end, msgs = addr + 16, addr + 16 + size, []
        for _ in range(nmsg):
            mtype, msize, flags = self.u(p, 2), self.u(p + 2, 2), b[p + 4]
            _check(msize % 8 == 0, "message data padded to 8 bytes")
            msgs.append((mtype, flags, b[p + 8:p + 8 + msize]))
            p += 8 + msize
        _check(p == end, "object header size matches its messages")
        return msgs

    def root_symbol_table(self):
        msgs = self._object_messages(self.root_header)
        st = [m for m in msgs if m[0] == 0x0011]
        _check(len(st) == 1, "root group has one symbol table message")
        bt, hp = struct.unpack("<QQ", st[0][2][:16])
        _check((bt, hp) == (self.btree, self.heap), "superblock scratch pad matches the symbol table message")
        return bt, hp

    def _btree_children(self, addr):
        b = self.b
        _check(b[addr:addr + 4] == b"TREE", "B-tree signature")
        _check(b[addr + 4] == 0, "B-tree of group nodes")
        level, used = b[addr + 5], self.u(addr + 6, 2)
        _check(self.u(addr + 8, 8) == UNDEF and self.u(addr + 16, 8) == UNDEF, "single node: no siblings")
        _check(used <= 2 * self.internal_k, "entries fit the node")
        keys, kids, p = [self.u(addr + 24, 8)], [], addr + 32
        for _ in range(used):
            kids.append(self.u(p, 8))
            keys.append(self.u(p + 8, 8))
            p += 16
        _check(keys[0] == 0, "key 0 is the empty string")
        node_size = 24 + (2 * self.internal_k + 1) * 8 + 2 * self.internal_k * 8
        _check(addr + node_size <= len(b), "the node's full size lies in the file")
        out = []
        for q, c in enumerate(kids):
            if level > 0:
                out.extend(self._btree_children(c))
            else:
                out.append((c, keys[q + 1]))
        return out

    def datasets(self):
        """{name: numpy array} of the root group, in name order."""
        self.root_symbol_table()
        out, last = {}, ""
        for snod, key in self._btree_children(self.btree):
            b = self.b
            _check(b[snod:snod + 4] == b"SNOD" and b[snod + 4] == 1, "symbol table node signature and version")
            n = self.u(snod + 6, 2)
            _check(n <= 2 * self.leaf_k, "entries fit the symbol table node")
            names = []
            for e in range(n):
                ent = snod + 8 + 40 * e
                name = self.name_at(self.u(ent, 8))
                _check(name > last, "names sorted across the group")
                last = name
                names.append(name)
                out[name] = self._dataset(self.u(ent + 8, 8))
            _check(self.name_at(key) == names[-1], "B-tree key is the last name of its child")
        return out

    def _dataset(self, addr):
        msgs = {m[0]: m[2] for m in self._object_messages(addr)}
        for t in (0x0001, 0x0003, 0x0005, 0x0008):
            _check(t in msgs, f"dataset message 0x{t:04x} present")
        sp = msgs[0x0001]
        _check(sp[0] == 1, "dataspace version 1")
        rank = sp[1]
        dims = struct.unpack(f"<{rank}Q", sp[8:8 + 8 * rank])
        ty = msgs[0x0003]
        _check(ty[0] == 0x11, "floating point datatype, version 1")
        _check(ty[1] & 1 == 0, "little endian")
        size, off, prec, eloc, esize, mloc, msize, bias = struct.unpack("<IHHBBBBI", ty[4:20])
        _check((size, off, prec, eloc, esize, mloc, msize, bias) == (8, 0, 64, 52, 11, 0, 52, 1023) and ty[3] == 0 and
               ty[2] == 63, "IEEE 754 double")
        _check(msgs[0x0005][0] == 2, "fill value message version 2")
        ly = msgs[0x0008]
        _check(ly[0] == 3 and ly[1] == 1, "layout version 3, contiguous")
        daddr, dsize = struct.unpack("<QQ", ly[2:18])
        _check(dsize == 8 * int(np.prod(dims)), "data size of the dataspace")
        _check(daddr + dsize <= len(self.b), "data inside the file")
        return np.frombuffer(self.b, dtype="<f8", count=int(np.prod(dims)), offset=daddr).reshape(dims).copy()


def read_datasets(path: str) -> dict:
    return Reader(path).datasets()
