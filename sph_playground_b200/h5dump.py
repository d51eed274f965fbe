"""The dump file, output/dump_full.h5 (utils/dumper.f90:14-225), without libhdf5.

The reference writes two float64 datasets at the root of an HDF5 file:
``state`` (49,) and ``store`` (N, 32) (Fortran store(32, N) seen row-major),
both chunked with unlimited maximum dimensions, so that a later run (and the
driver's AddParticles) can resize them.  Neither h5py nor libhdf5 is part of
this project's environment, so this module writes and reads that file
directly from the HDF5 file-format specification (version 0 superblock, the
layout the HDF5 1.6-1.8 libraries write by default):

* superblock v0 with the root group's symbol-table entry;
* root group: a version 1 object header holding a symbol-table message, a
  local heap with the link names and a group B-tree (version 1, type 0)
  pointing to one symbol-table node;
* each dataset: a version 1 object header with dataspace (current and
  unlimited maximum dimensions), IEEE float64 little-endian datatype, fill
  value and chunked layout (version 3) messages; one chunk covering the
  whole dataset, indexed by a chunk B-tree (version 1, type 1).

The reader handles what that writer produces plus the other layouts a v0
file commonly holds (contiguous layout message versions 1-3, continuation
messages, version 1-2 dataspaces), which is enough to read files written by
the HDF5 library in the same style; it is checked against such a file.
"""
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIG = b"\x89HDF\r\n\x1a\n"
GROUP_LEAF_K, GROUP_INTERNAL_K, CHUNK_K = 4, 16, 32


def _pad8(b):
    return b + b"\0" * (-len(b) % 8)


def _msg(mtype, data, flags=0):
    data = _pad8(data)
    return struct.pack("<HHB3x", mtype, len(data), flags) + data


def _ohdr_v1(messages):
    body = b"".join(messages)
    return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(body)) + body


def _f64_type():
    # class 1 (floating point), version 1; little-endian, mantissa
    # normalisation 2 (implied leading 1), sign bit 63; size 8; bit offset 0,
    # precision 64, exponent at bit 52 of 11 bits, mantissa at 0 of 52 bits,
    # exponent bias 1023
    return struct.pack("<B3BI", 0x11, 0x20, 63, 0, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)


def write(path, datasets):
    """Write {name: float64 array} as chunked datasets with unlimited
    maximum dimensions at the root of a new HDF5 file."""
    names = sorted(datasets)
    arrays = [np.ascontiguousarray(datasets[n], dtype="<f8") for n in names]
    out = bytearray()

    def alloc(n):
        a = len(out)
        out.extend(b"\0" * n)
        return a

    sb = alloc(56 + 40)
    # local heap: "" at 0, then the names; a trailing free block as the
    # library leaves one
    heap_data = bytearray(b"\0" * 8)
    name_off = []
    for n in names:
        name_off.append(len(heap_data))
        heap_data += _pad8(n.encode() + b"\0")
    free_at = len(heap_data)
    heap_data += struct.pack("<QQ", 1, 64) + b"\0" * 48
    heap_hdr = alloc(32)
    heap_seg = alloc(len(heap_data))
    out[heap_seg:heap_seg + len(heap_data)] = heap_data
    out[heap_hdr:heap_hdr + 32] = b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), free_at, heap_seg)
    # dataset chunks, chunk B-trees, object headers
    ohdr_addr = []
    for a in arrays:
        rank = a.ndim
        data_at = alloc(a.nbytes)
        out[data_at:data_at + a.nbytes] = a.tobytes()
        ksize = 8 + 8 * (rank + 1)
        node_size = 24 + (2 * CHUNK_K + 1) * ksize + 2 * CHUNK_K * 8
        bt = alloc(node_size)
        key0 = struct.pack("<II", a.nbytes, 0) + struct.pack("<%dQ" % (rank + 1), *([0] * (rank + 1)))
        key1 = struct.pack("<II", 0, 0) + struct.pack("<%dQ" % (rank + 1), *(list(a.shape) + [0]))
        node = b"TREE" + struct.pack("<BBHQQ", 1, 0, 1, UNDEF, UNDEF) + key0 + struct.pack("<Q", data_at) + key1
        out[bt:bt + len(node)] = node
        space = struct.pack("<BBBB4x", 1, rank, 1, 0) + struct.pack("<%dQ" % rank, *a.shape) \
            + struct.pack("<%dQ" % rank, *([UNDEF] * rank))
        fill = struct.pack("<BBBBI", 1, 2, 2, 1, 0)
        layout = struct.pack("<BBBQ", 3, 2, rank + 1, bt) + struct.pack("<%dI" % (rank + 1), *(list(a.shape) + [8]))
        oh = _ohdr_v1([_msg(1, space), _msg(3, _f64_type(), 1), _msg(5, fill, 1), _msg(8, layout)])
        at = alloc(len(oh))
        out[at:at + len(oh)] = oh
        ohdr_addr.append(at)
    # symbol-table node with the datasets, the group B-tree over it
    snod_size = 8 + 2 * GROUP_LEAF_K * 40
    snod = alloc(snod_size)
    ent = b"".join(struct.pack("<QQII16x", name_off[i], ohdr_addr[i], 0, 0) for i in range(len(names)))
    out[snod:snod + 8 + len(ent)] = b"SNOD" + struct.pack("<BBH", 1, 0, len(names)) + ent
    gbt_size = 24 + (2 * GROUP_INTERNAL_K + 1) * 8 + 2 * GROUP_INTERNAL_K * 8
    gbt = alloc(gbt_size)
    node = b"TREE" + struct.pack("<BBHQQ", 0, 0, 1, UNDEF, UNDEF) + struct.pack("<QQQ", 0, snod, name_off[-1])
    out[gbt:gbt + len(node)] = node
    root = _ohdr_v1([_msg(0x11, struct.pack("<QQ", gbt, heap_hdr), 1)])
    root_at = alloc(len(root))
    out[root_at:root_at + len(root)] = root
    # superblock v0: versions, offset / length sizes 8, group K values, flags
    # 0, base 0, no free-space info, end of file, no driver block, root entry
    sbb = SIG + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, GROUP_LEAF_K, GROUP_INTERNAL_K, 0)
    sbb += struct.pack("<QQQQ", 0, UNDEF, len(out), UNDEF)
    sbb += struct.pack("<QQII", 0, root_at, 1, 0) + struct.pack("<QQ", gbt, heap_hdr)
    out[sb:sb + len(sbb)] = sbb
    with open(path, "wb") as f:
        f.write(out)


class _File:
    def __init__(self, buf):
        self.b = buf
        at = 0
        while self.b[at:at + 8] != SIG:  # a user block moves the superblock by a power of 2
            at = 512 if at == 0 else 2 * at
            if at >= len(self.b):
                raise ValueError("not an HDF5 file")
        if self.b[at + 8] != 0:
            raise ValueError("superblock version %d is not supported" % self.b[at + 8])
        so, sl = self.b[at + 13], self.b[at + 14]
        if (so, sl) != (8, 8):
            raise ValueError("offset / length sizes other than 8 are not supported")
        self.base = struct.unpack_from("<Q", self.b, at + 24)[0]
        self.root_entry = at + 56

    def u(self, fmt, at):
        return struct.unpack_from("<" + fmt, self.b, self.base + at)

    def messages(self, oh):
        ver, _, nmsg, _, size = self.u("BBHII", oh)
        if ver != 1:
            raise ValueError("object header version %d is not supported" % ver)
        blocks, out = [(oh + 16, size)], []
        while blocks and len(out) < nmsg:
            at, size = blocks.pop(0)
            end = at + size
            while at + 8 <= end and len(out) < nmsg:
                mt, ms, _ = self.u("HHB", at)
                if mt == 0x10:  # continuation
                    blocks.append(self.u("QQ", at + 8))
                out.append((mt, at + 8, ms))
                at += 8 + ms
        return out

    def group(self, btree, heap):
        _, _, _, _, dseg = self.u("4sB3xQQQ", heap)
        names = {}

        def walk(node):
            sig, ntype, level, used = self.u("4sBBH", node)
            if sig != b"TREE" or ntype != 0:
                raise ValueError("bad group B-tree")
            for i in range(used):
                child = self.u("Q", node + 24 + 8 + i * 16)[0]
                if level > 0:
                    walk(child)
                    continue
                sig2, _, _, nsym = self.u("4sBBH", child)
                if sig2 != b"SNOD":
                    raise ValueError("bad symbol-table node")
                for k in range(nsym):
                    noff, ohdr = self.u("QQ", child + 8 + 40 * k)
                    s = self.base + dseg + noff
                    name = bytes(self.b[s:self.b.index(b"\0", s)]).decode()
                    names[name] = ohdr
        walk(btree)
        return names

    def dataset(self, oh):
        shape = dtype = None
        layout = None
        for mt, at, _ in self.messages(oh):
            if mt == 1:
                ver, rank, flags = self.u("BBB", at)
                off = at + (8 if ver == 1 else 4)
                shape = self.u("%dQ" % rank, off)
            elif mt == 3:
                cls_ver, b0, _, _, size = self.u("BBBBI", at)
                if cls_ver & 0x0F != 1 or size != 8 or b0 & 1:
                    raise ValueError("only little-endian float64 data are supported")
                dtype = "<f8"
            elif mt == 8:
                layout = at
        if shape is None or dtype is None or layout is None:
            raise ValueError("dataset without dataspace, datatype or layout")
        n = int(np.prod(shape)) if shape else 1
        ver = self.u("B", layout)[0]
        if ver in (1, 2):
            rank, cls = self.u("BB", layout + 1)
            addr = self.u("Q", layout + 8)[0]
            if cls != 1:
                raise ValueError("layout class %d (version %d) is not supported" % (cls, ver))
            return self._read(addr, n, dtype).reshape(shape)
        cls = self.u("B", layout + 1)[0]
        if cls == 1:  # contiguous
            addr = self.u("Q", layout + 2)[0]
            return self._read(addr, n, dtype).reshape(shape)
        if cls != 2:
            raise ValueError("layout class %d is not supported" % cls)
        dims = self.u("B", layout + 2)[0]
        bt = self.u("Q", layout + 3)[0]
        chunk = self.u("%dI" % dims, layout + 11)[: dims - 1]
        out = np.zeros(shape, dtype=dtype)
        rank = dims - 1

        def walk(node):
            sig, ntype, level, used = self.u("4sBBH", node)
            if sig != b"TREE" or ntype != 1:
                raise ValueError("bad chunk B-tree")
            ks = 8 + 8 * dims
            for i in range(used):
                kat = node + 24 + i * (ks + 8)
                csize, mask = self.u("II", kat)
                offs = self.u("%dQ" % dims, kat + 8)[:rank]
                child = self.u("Q", kat + ks)[0]
                if level > 0:
                    walk(child)
                    continue
                if mask:
                    raise ValueError("filtered chunks are not supported")
                blk = self._read(child, int(np.prod(chunk)), dtype).reshape(chunk)
                sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, chunk, shape))
                out[sl] = blk[tuple(slice(0, x.stop - x.start) for x in sl)]
        walk(bt)
        return out

    def _read(self, addr, n, dtype):
        s = self.base + addr
        return np.frombuffer(bytes(self.b[s:s + 8 * n]), dtype=dtype).copy()


def read(path):
    """{name: array} of the float64 datasets at the root of an HDF5 file."""
    with open(path, "rb") as f:
        h = _File(f.read())
    _, ohdr, cache, _, btree, heap = struct.unpack_from("<QQII QQ".replace(" ", ""), h.b,
                                                       h.root_entry)
    if cache != 1:
        # no cached scratch pad: take the symbol-table message of the root header
        for mt, at, _ in h.messages(ohdr):
            if mt == 0x11:
                btree, heap = h.u("QQ", at)
    out = {}
    for name, oh in h.group(btree, heap).items():
        try:
            out[name] = h.dataset(oh)
        except ValueError:
            continue  # groups and non-float64 objects are skipped
    return out
