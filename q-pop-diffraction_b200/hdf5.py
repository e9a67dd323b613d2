"""
Minimal HDF5 reading and writing without h5py or libhdf5.

Covers what Q-POP-FerroDyn fields and Q-POP-Diffraction output use (src/python/io_utils.py:30-141):
files with the version-0 superblock that h5py writes by default, groups held in symbol tables,
version-1 object headers (with continuation blocks), contiguous, compact and chunked datasets
(version-1 B-tree chunk index) with the shuffle and deflate filters, little-endian IEEE floats and
integers, and scalar numeric or fixed-length string attributes.

Reading:  ``read_dataset(path, name)``, ``read_attrs(path)``, ``list_datasets(path)``.
Writing:  ``write_file(path, datasets, attrs)`` writes contiguous or chunked (shuffle + deflate)
datasets and root attributes in the same version-0 layout; ``write_diffraction_output`` writes the
reference's result file (``/intensity`` as (nz, ny, nx), ``/q_x``, ``/q_y``, ``/q_z``, attributes
``Timestep`` and ``q_units``) and its XDMF sidecar (src/python/io_utils.py:95-141).
"""

from __future__ import annotations

import os
import struct
import zlib

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class HDF5Error(ValueError):
    pass


# ------------------------------------------------------------------------------------------------
# Reading
# ------------------------------------------------------------------------------------------------

class _Reader:
    def __init__(self, path):
        with open(path, "rb") as fh:
            self.b = fh.read()
        self.path = str(path)
        b = self.b
        if b[:8] != SIGNATURE:
            raise HDF5Error(f"{path}: not an HDF5 file")
        if b[8] != 0:
            raise HDF5Error(f"{path}: superblock version {b[8]} is not supported (version 0 only)")
        self.so, self.sl = b[13], b[14]
        if self.so != 8 or self.sl != 8:
            raise HDF5Error(f"{path}: only 8-byte offsets and lengths are supported")
        self.base = self._u(24, 8)
        # root group symbol table entry at 56: link name offset, object header address, cache type, scratch
        self.root_header = self._u(64, 8)
        cache_type = self._u(72, 4)
        self.root_btree = self._u(80, 8) if cache_type == 1 else None
        self.root_heap = self._u(88, 8) if cache_type == 1 else None

    def _u(self, off, n):
        return int.from_bytes(self.b[off:off + n], "little")

    # --- groups -------------------------------------------------------------------------------
    def _heap_string(self, heap, off):
        if self.b[heap:heap + 4] != b"HEAP":
            raise HDF5Error(f"{self.path}: bad local heap")
        data = self._u(heap + 24, 8)
        end = self.b.index(b"\0", data + off)
        return self.b[data + off:end].decode()

    def _group_entries(self, btree, heap):
        out = {}
        stack = [btree]
        while stack:
            node = stack.pop()
            if self.b[node:node + 4] != b"TREE":
                raise HDF5Error(f"{self.path}: bad group B-tree node")
            level, used = self.b[node + 5], self._u(node + 6, 2)
            p = node + 8 + 16 + 8  # header, siblings, key 0
            for _ in range(used):
                child = self._u(p, 8)
                p += 16  # child, next key
                if level > 0:
                    stack.append(child)
                else:
                    out.update(self._snod(child, heap))
        return out

    def _snod(self, addr, heap):
        if self.b[addr:addr + 4] != b"SNOD":
            raise HDF5Error(f"{self.path}: bad symbol table node")
        n = self._u(addr + 6, 2)
        out = {}
        p = addr + 8
        for _ in range(n):
            name = self._heap_string(heap, self._u(p, 8))
            out[name] = self._u(p + 8, 8)
            p += 40
        return out

    def root(self):
        if self.root_btree is None:
            msgs = self.messages(self.root_header)
            st = next((m for t, m in msgs if t == 0x11), None)
            if st is None:
                raise HDF5Error(f"{self.path}: root group has no symbol table")
            self.root_btree, self.root_heap = self._u(st, 8), self._u(st + 8, 8)
        return self._group_entries(self.root_btree, self.root_heap)

    def lookup(self, name):
        entries = self.root()
        cur = None
        parts = [p for p in name.strip("/").split("/") if p]
        table = entries
        for i, part in enumerate(parts):
            if part not in table:
                raise HDF5Error(f"{self.path}: no object {name!r}")
            cur = table[part]
            if i < len(parts) - 1:
                st = next((m for t, m in self.messages(cur) if t == 0x11), None)
                if st is None:
                    raise HDF5Error(f"{self.path}: {part!r} is not a group")
                table = self._group_entries(self._u(st, 8), self._u(st + 8, 8))
        return cur

    # --- object headers -------------------------------------------------------------------------
    def messages(self, addr):
        b = self.b
        if b[addr] != 1:
            raise HDF5Error(f"{self.path}: object header version {b[addr]} is not supported")
        nmsg = self._u(addr + 2, 2)
        size = self._u(addr + 8, 4)
        blocks = [(addr + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            p = start
            while p + 8 <= start + length and len(out) < nmsg:
                mtype, msize = self._u(p, 2), self._u(p + 2, 2)
                data = p + 8
                if mtype == 0x10:  # continuation
                    blocks.append((self._u(data, 8), self._u(data + 8, 8)))
                out.append((mtype, data))
                p = data + msize
        return out

    # --- datasets -------------------------------------------------------------------------------
    def _dataspace(self, p):
        b = self.b
        ver, rank, flags = b[p], b[p + 1], b[p + 2]
        q = p + (8 if ver == 1 else 4)
        if ver == 2 and b[p + 3] == 0:
            return ()
        return tuple(self._u(q + 8 * i, 8) for i in range(rank))

    def _datatype(self, p):
        b = self.b
        cls = b[p] & 0x0F
        bits0 = b[p + 1]
        size = self._u(p + 4, 4)
        if bits0 & 1:
            raise HDF5Error(f"{self.path}: big-endian data is not supported")
        if cls == 1:
            return np.dtype(f"<f{size}")
        if cls == 0:
            return np.dtype(f"<{'i' if bits0 & 0x08 else 'u'}{size}")
        if cls == 3:
            return np.dtype(f"S{size}")
        raise HDF5Error(f"{self.path}: datatype class {cls} is not supported")

    def _filters(self, p):
        b = self.b
        ver, n = b[p], b[p + 1]
        q = p + (8 if ver == 1 else 2)
        out = []
        for _ in range(n):
            fid = self._u(q, 2)
            if ver == 1 or fid >= 256:
                namelen = self._u(q + 2, 2)
                nvals = self._u(q + 6, 2)
                q += 8 + ((namelen + 7) // 8 * 8 if ver == 1 else namelen)
            else:
                nvals = self._u(q + 4, 2)
                q += 6
            vals = [self._u(q + 4 * i, 4) for i in range(nvals)]
            q += 4 * nvals + (4 if ver == 1 and nvals % 2 else 0)
            out.append((fid, vals))
        return out

    def _chunks(self, btree, rank):
        """(offsets, filter mask, address, size) of every chunk under a version-1 chunk B-tree."""
        out = []
        stack = [btree]
        keylen = 8 + 8 * (rank + 1)
        while stack:
            node = stack.pop()
            if self.b[node:node + 4] != b"TREE" or self.b[node + 4] != 1:
                raise HDF5Error(f"{self.path}: bad chunk B-tree node")
            level, used = self.b[node + 5], self._u(node + 6, 2)
            p = node + 24
            for _ in range(used):
                size, mask = self._u(p, 4), self._u(p + 4, 4)
                offs = tuple(self._u(p + 8 + 8 * i, 8) for i in range(rank))
                child = self._u(p + keylen, 8)
                if level > 0:
                    stack.append(child)
                else:
                    out.append((offs, mask, child, size))
                p += keylen + 8
        return out

    def dataset(self, name):
        msgs = self.messages(self.lookup(name))
        kinds = {t: d for t, d in msgs}
        if 0x01 not in kinds or 0x03 not in kinds or 0x08 not in kinds:
            raise HDF5Error(f"{self.path}: {name!r} is not a dataset")
        shape = self._dataspace(kinds[0x01])
        dtype = self._datatype(kinds[0x03])
        filters = self._filters(kinds[0x0B]) if 0x0B in kinds else []
        lp = kinds[0x08]
        ver, cls = self.b[lp], self.b[lp + 1]
        if ver != 3:
            raise HDF5Error(f"{self.path}: layout message version {ver} is not supported")
        count = int(np.prod(shape)) if shape else 1
        if cls == 0:  # compact
            size = self._u(lp + 2, 2)
            return np.frombuffer(self.b[lp + 4:lp + 4 + size], dtype=dtype, count=count).reshape(shape).copy()
        if cls == 1:  # contiguous
            addr = self._u(lp + 2, 8)
            if addr == UNDEF:
                return np.zeros(shape, dtype=dtype)
            return np.frombuffer(self.b, dtype=dtype, count=count, offset=addr).reshape(shape).copy()
        if cls != 2:
            raise HDF5Error(f"{self.path}: layout class {cls} is not supported")
        rank = self.b[lp + 2] - 1
        btree = self._u(lp + 3, 8)
        chunk = tuple(self._u(lp + 11 + 4 * i, 4) for i in range(rank))
        out = np.zeros(shape, dtype=dtype)
        if btree == UNDEF:
            return out
        for offs, mask, addr, size in self._chunks(btree, rank):
            raw = self.b[addr:addr + size]
            for k, (fid, vals) in reversed(list(enumerate(filters))):
                if mask & (1 << k):
                    continue
                if fid == 1:
                    raw = zlib.decompress(raw)
                elif fid == 2:
                    es = vals[0] if vals else dtype.itemsize
                    a = np.frombuffer(raw, dtype=np.uint8)
                    raw = a.reshape(es, -1).T.tobytes()
                else:
                    raise HDF5Error(f"{self.path}: filter {fid} is not supported")
            block = np.frombuffer(raw, dtype=dtype, count=int(np.prod(chunk))).reshape(chunk)
            sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, chunk, shape))
            out[sl] = block[tuple(slice(0, x.stop - x.start) for x in sl)]
        return out

    def attrs(self, addr=None):
        out = {}
        for t, p in self.messages(self.root_header if addr is None else addr):
            if t != 0x0C:
                continue
            ver = self.b[p]
            nlen, tlen, slen = self._u(p + 2, 2), self._u(p + 4, 2), self._u(p + 6, 2)
            pad = (lambda x: (x + 7) // 8 * 8) if ver == 1 else (lambda x: x)
            q = p + 8 + (1 if ver == 3 else 0)
            name = self.b[q:q + nlen].split(b"\0")[0].decode()
            q += pad(nlen)
            dtype = self._datatype(q)
            q += pad(tlen)
            shape = self._dataspace(q)
            q += pad(slen)
            count = int(np.prod(shape)) if shape else 1
            val = np.frombuffer(self.b, dtype=dtype, count=count, offset=q)
            if dtype.kind == "S":
                out[name] = val[0].split(b"\0")[0].decode()
            else:
                out[name] = val.reshape(shape)[()] if shape else val[0]
        return out


def read_dataset(path, name):
    """The dataset `name` of an HDF5 file as a NumPy array."""
    return _Reader(path).dataset(name)


def read_attrs(path, name=None):
    """Attributes of the root group (or of object `name`)."""
    r = _Reader(path)
    return r.attrs(None if name is None else r.lookup(name))


def list_datasets(path):
    """Names of the objects in the root group."""
    return sorted(_Reader(path).root())


# ------------------------------------------------------------------------------------------------
# Writing (version-0 superblock, symbol-table root group, contiguous or chunked datasets)
# ------------------------------------------------------------------------------------------------

def _pad8(b):
    return b + b"\0" * ((-len(b)) % 8)


def _dtype_msg(dt):
    dt = np.dtype(dt)
    if dt.kind == "f":
        # class 1 (floating point), version 1; little-endian IEEE, sign bit, exponent/mantissa layout
        if dt.itemsize == 8:
            bits = bytes([0x20, 0x3F, 0x00])
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        else:
            bits = bytes([0x20, 0x1F, 0x00])
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
        return bytes([0x11]) + bits + struct.pack("<I", dt.itemsize) + props
    if dt.kind in "iu":
        bits = bytes([0x08 if dt.kind == "i" else 0x00, 0, 0])
        return bytes([0x10]) + bits + struct.pack("<I", dt.itemsize) + struct.pack("<HH", 0, dt.itemsize * 8)
    if dt.kind == "S":
        return bytes([0x13, 0x00, 0x00, 0x00]) + struct.pack("<I", dt.itemsize)
    raise HDF5Error(f"cannot write dtype {dt}")


def _space_msg(shape):
    return bytes([1, len(shape), 0, 0, 0, 0, 0, 0]) + b"".join(struct.pack("<Q", s) for s in shape)


def _message(mtype, body, flags=0):
    body = _pad8(body)
    return struct.pack("<HHB3x", mtype, len(body), flags) + body


def _object_header(msgs):
    body = b"".join(msgs)
    return struct.pack("<BBHII", 1, 0, len(msgs), 1, len(body)) + b"\0" * 4 + body


def _attribute(name, value):
    if isinstance(value, str):
        arr = np.array(value.encode(), dtype=f"S{len(value.encode()) + 1}")
        shape = ()
    else:
        arr = np.asarray(value)
        shape = arr.shape
    nm = name.encode() + b"\0"
    dt, sp = _dtype_msg(arr.dtype), (_space_msg(shape) if shape else bytes([1, 0, 0, 0, 0, 0, 0, 0]))
    body = struct.pack("<BxHHH", 1, len(nm), len(dt), len(sp)) + _pad8(nm) + _pad8(dt) + _pad8(sp) + arr.tobytes()
    return _message(0x0C, body)


def _filter_msg(filters):
    """Filter pipeline message, version 1: (id, client values) for each predefined filter."""
    body = struct.pack("<BB6x", 1, len(filters))
    for fid, vals in filters:
        body += struct.pack("<HHHH", fid, 0, 0, len(vals)) + b"".join(struct.pack("<I", v) for v in vals)
        if len(vals) % 2:
            body += b"\0" * 4
    return body


CHUNK_K = 32  # entries per chunk B-tree node: 2K (HDF5's default indexed-storage K)


def _chunk_btree(base, entries, rank, chunk, elem):
    """
    Version-1 chunk B-tree nodes for `entries` = [(offsets, size, address)] in C order, laid out
    from address `base`; every node is written at full size (2K entries).  Returns (root
    address, bytes).
    """
    keylen = 8 + 8 * (rank + 1)
    node_size = 24 + (2 * CHUNK_K + 1) * keylen + 2 * CHUNK_K * 8

    def key(size, offs):
        return struct.pack("<II", size, 0) + b"".join(struct.pack("<Q", o) for o in offs) + struct.pack("<Q", 0)

    out = bytearray()
    level = 0
    # each item: (first offsets, upper-bound offsets, size, address)
    items = [(o, tuple(a + c for a, c in zip(o, chunk)), sz, ad) for o, sz, ad in entries]
    while True:
        nodes = [items[i:i + 2 * CHUNK_K] for i in range(0, len(items), 2 * CHUNK_K)] or [[]]
        parents = []
        for k, group in enumerate(nodes):
            addr = base + len(out)
            left = UNDEF if k == 0 else addr - node_size
            right = UNDEF if k == len(nodes) - 1 else addr + node_size
            body = b"TREE" + struct.pack("<BBHQQ", 1, level, len(group), left, right)
            for first, _, sz, ad in group:
                body += key(sz if level == 0 else 0, first) + struct.pack("<Q", ad)
            body += key(0, group[-1][1] if group else (0,) * rank)
            body += b"\0" * (node_size - len(body))
            out += body
            if group:
                parents.append((group[0][0], group[-1][1], 0, addr))
        if len(nodes) == 1:
            return base + len(out) - node_size, bytes(out)
        items = parents
        level += 1


def _chunked(a, chunks, shuffle, gzip):
    """(filters, [(offsets, encoded bytes)]) for array a split into chunks of shape `chunks`."""
    a = np.ascontiguousarray(a)
    chunks = tuple(int(c) for c in chunks)
    if len(chunks) != a.ndim or any(c < 1 for c in chunks):
        raise HDF5Error(f"chunk shape {chunks} does not fit an array of rank {a.ndim}")
    filters = ([(2, [a.dtype.itemsize])] if shuffle else []) + ([(1, [int(gzip)])] if gzip is not None else [])
    out = []
    for offs in np.ndindex(*[-(-s // c) for s, c in zip(a.shape, chunks)]):
        offs = tuple(o * c for o, c in zip(offs, chunks))
        block = np.zeros(chunks, dtype=a.dtype)
        sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, chunks, a.shape))
        block[tuple(slice(0, x.stop - x.start) for x in sl)] = a[sl]
        raw = block.tobytes()
        if shuffle:
            raw = np.frombuffer(raw, dtype=np.uint8).reshape(-1, a.dtype.itemsize).T.tobytes()
        if gzip is not None:
            raw = zlib.compress(raw, int(gzip))
        out.append((offs, raw))
    return filters, out


def write_file(path, datasets, attrs=None):
    """
    Write an HDF5 file.  `datasets` maps names to arrays, stored contiguous in C order, or to
    ``(array, {"chunks": shape, "shuffle": bool, "gzip": level})`` for a chunked dataset with the
    shuffle and deflate filters (the storage of Q-POP-FerroDyn's fields).  `attrs` maps names to
    scalar numbers or strings on the root group.
    """
    names = list(datasets)
    specs = {}
    for n in names:
        v = datasets[n]
        if isinstance(v, tuple):
            a, opts = v
            specs[n] = (np.ascontiguousarray(a), dict(opts))
        else:
            specs[n] = (np.ascontiguousarray(v), None)
    heap_data = b"\0" * 8  # offset 0: the empty name
    name_off = []
    for n in names:
        name_off.append(len(heap_data))
        heap_data += _pad8(n.encode() + b"\0")
    heap_data_size = max(len(heap_data), 88)
    heap_data = heap_data + b"\0" * (heap_data_size - len(heap_data))

    # layout: superblock (96) | root object header | local heap + data | B-tree | SNOD | dataset headers | data
    sb_size = 96
    root_msgs_len = 8 + 16  # symbol-table message (type 0x11) body of 16 bytes
    root_attr_msgs = [_attribute(k, v) for k, v in (attrs or {}).items()]
    root_oh_size = 16 + root_msgs_len + sum(len(m) for m in root_attr_msgs)
    heap_addr = sb_size + root_oh_size
    heap_size = 32 + heap_data_size
    btree_addr = heap_addr + heap_size
    btree_size = 24 + 8 + 16  # header + key0 + (child, key1)
    snod_addr = btree_addr + btree_size
    leaf_k = max(4, -(-len(names) // 2))  # one symbol table node holds all 2K names
    snod_size = 8 + 40 * 2 * leaf_k
    hdr_addr = snod_addr + snod_size

    # message bodies whose size does not depend on addresses
    encoded = {}
    for n in names:
        a, opts = specs[n]
        if opts is not None:
            encoded[n] = _chunked(a, opts.get("chunks", a.shape), opts.get("shuffle", False), opts.get("gzip"))

    def layout_msg(n, addr):
        a, opts = specs[n]
        if opts is None:
            return struct.pack("<BBQQ", 3, 1, addr, a.nbytes)
        chunks = tuple(int(c) for c in opts.get("chunks", a.shape))
        return struct.pack("<BBBQ", 3, 2, a.ndim + 1, addr) + \
            b"".join(struct.pack("<I", c) for c in chunks + (a.dtype.itemsize,))

    def header_msgs(n, addr):
        a, _ = specs[n]
        msgs = [_message(0x01, _space_msg(a.shape)), _message(0x03, _dtype_msg(a.dtype))]
        if n in encoded and encoded[n][0]:
            msgs.append(_message(0x0B, _filter_msg(encoded[n][0])))
        msgs.append(_message(0x08, layout_msg(n, addr)))
        return msgs

    hdr_sizes = [16 + sum(len(m) for m in header_msgs(n, 0)) for n in names]
    cur = hdr_addr + sum(hdr_sizes)
    headers, blocks = [], []
    addr = hdr_addr
    for n, hs in zip(names, hdr_sizes):
        a, opts = specs[n]
        if opts is None:
            data_addr = cur
            blocks.append((cur, a.tobytes()))
            cur += a.nbytes
        else:
            entries = []
            for offs, raw in encoded[n][1]:
                entries.append((offs, len(raw), cur))
                blocks.append((cur, raw))
                cur += len(raw)
            chunks = tuple(int(c) for c in opts.get("chunks", a.shape))
            data_addr, tree = _chunk_btree(cur, entries, a.ndim, chunks, a.dtype.itemsize)
            blocks.append((cur, tree))
            cur += len(tree)
        h = _object_header(header_msgs(n, data_addr))
        assert len(h) == hs
        headers.append((addr, h))
        addr += hs
    eof = cur

    out = bytearray(eof)
    # superblock v0
    sb = SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", leaf_k, 16, 0)
    sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
    sb += struct.pack("<QQII", 0, sb_size, 1, 0) + struct.pack("<QQ", btree_addr, heap_addr)
    out[0:len(sb)] = sb
    # root object header: symbol table message + attributes
    st = _message(0x11, struct.pack("<QQ", btree_addr, heap_addr))
    oh = _object_header([st] + root_attr_msgs)
    out[sb_size:sb_size + len(oh)] = oh
    # local heap
    heap = b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", heap_data_size, UNDEF, heap_addr + 32)
    out[heap_addr:heap_addr + 32] = heap
    out[heap_addr + 32:heap_addr + 32 + heap_data_size] = heap_data
    # group B-tree (type 0, level 0, one child): keys are heap offsets of the last name in each child
    last = max(name_off, key=lambda o: heap_data[o:heap_data.index(b"\0", o)]) if names else 0
    bt = b"TREE" + bytes([0, 0]) + struct.pack("<HQQ", 1 if names else 0, UNDEF, UNDEF)
    bt += struct.pack("<QQQ", 0, snod_addr, last)
    out[btree_addr:btree_addr + len(bt)] = bt
    # symbol table node, names in sorted order as the format requires
    order = sorted(range(len(names)), key=lambda i: names[i])
    sn = b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(names))
    for i in order:
        sn += struct.pack("<QQII", name_off[i], headers[i][0], 0, 0) + b"\0" * 16
    out[snod_addr:snod_addr + len(sn)] = sn
    for a, h in headers:
        out[a:a + len(h)] = h
    for a, d in blocks:
        out[a:a + len(d)] = d
    with open(path, "wb") as fh:
        fh.write(bytes(out))


def write_diffraction_output(base_name, I, qx, qy, qz, step):
    """
    The reference's result files (src/python/io_utils.py:95-141): ``{base}.h5`` with ``/intensity``
    stored (nz, ny, nx), ``/q_x``, ``/q_y``, ``/q_z`` in nm^-1 and attributes ``Timestep`` and
    ``q_units``; and the ParaView sidecar ``{base}.xdmf`` (a 3DRectMesh on the q axes).
    """
    I = np.asarray(I, dtype=np.float64)
    write_file(f"{base_name}.h5", {"intensity": I.transpose(2, 1, 0), "q_x": np.asarray(qx, dtype=np.float64),
                                   "q_y": np.asarray(qy, dtype=np.float64), "q_z": np.asarray(qz, dtype=np.float64)},
               attrs={"Timestep": np.int64(step), "q_units": "nm^-1"})
    nx, ny, nz = len(qx), len(qy), len(qz)
    h5 = os.path.basename(f"{base_name}.h5")
    item = '<DataItem Dimensions="{}" NumberType="Float" Precision="8" Format="HDF">' + h5 + ':/{}</DataItem>'
    with open(f"{base_name}.xdmf", "w", encoding="utf-8") as fh:
        fh.write(f"""<?xml version="1.0" ?>
<Xdmf Version="3.0">
  <Domain>
    <Grid Name="DiffractionPattern" GridType="Uniform">
      <Topology TopologyType="3DRectMesh" Dimensions="{nz} {ny} {nx}"/>
      <Geometry GeometryType="VXVYVZ">
        {item.format(nx, "q_x")}
        {item.format(ny, "q_y")}
        {item.format(nz, "q_z")}
      </Geometry>
      <Attribute Name="Intensity" AttributeType="Scalar" Center="Node">
        {item.format(f"{nz} {ny} {nx}", "intensity")}
      </Attribute>
    </Grid>
  </Domain>
</Xdmf>
""")


def load_diffraction_output(path):
    """(I (nx, ny, nz), qx, qy, qz, attrs) from a result file (src/python/io_utils.py:186-207)."""
    r = _Reader(path)
    I = r.dataset("intensity").transpose(2, 1, 0)
    return I, r.dataset("q_x"), r.dataset("q_y"), r.dataset("q_z"), r.attrs()
