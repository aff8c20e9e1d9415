"""A small HDF5 encoder of the layout libhdf5 writes by default (TEST INFRASTRUCTURE): written
from the public HDF5 file-format specification, independently of the library's reader, so
that the reader is checked on files of the reference's own format — superblock version 0,
version-1 object headers (with continuation blocks on request), symbol-table groups (a
version-1 group B-tree over symbol nodes and a local heap; one or two levels), version-1
attribute messages, and datasets stored contiguous, compact or chunked (version-1 chunk
B-tree) with the shuffle and deflate filters.

    write(path, tree)   tree: {"name": ndarray | {"attrs": {...}, **children} , ...}

ndarray values become datasets; dict values groups; a dict's "attrs" entry holds the
attributes of that group (name -> numpy scalar or 1-D array); a dataset given as
`Data(array, layout="chunked", chunk=(...), shuffle=True, deflate=4, attrs={})` chooses its
storage."""
from __future__ import annotations

import struct
import zlib
from dataclasses import dataclass, field

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIG = b"\x89HDF\r\n\x1a\n"


@dataclass
class Data:
    array: np.ndarray
    layout: str = "contiguous"   # contiguous | compact | chunked
    chunk: tuple | None = None
    shuffle: bool = False
    deflate: int | None = None
    attrs: dict = field(default_factory=dict)
    continuation: bool = False   # put the layout and later messages in a continuation block


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * ((-len(b)) % 8)


def _dtype_msg(dt: np.dtype) -> bytes:
    dt = np.dtype(dt)
    size = dt.itemsize
    if dt.kind == "f":
        d = size == 8
        return struct.pack("<BBBBIHHBBBBI", (1 << 4) | 1, 0x20, 63 if d else 31, 0, size, 0, 8 * size,
                           52 if d else 23, 11 if d else 8, 0, 52 if d else 23, 1023 if d else 127)
    signed = dt.kind == "i"
    return struct.pack("<BBBBIHH", (1 << 4) | 0, 0x08 if signed else 0, 0, 0, size, 0, 8 * size)


def _space_msg(shape) -> bytes:
    # version 1: version, rank, flags (no maximum dims), reserved 5 bytes, dims
    b = struct.pack("<BBBB I", 1, len(shape), 0, 0, 0)
    for d in shape:
        b += struct.pack("<Q", d)
    return b


def _attr_msg(name: str, value) -> bytes:
    v = np.asarray(value)
    nm = name.encode() + b"\0"
    dt = _dtype_msg(v.dtype)
    sp = _space_msg(() if v.ndim == 0 else v.shape)
    b = struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(sp))
    return b + _pad8(nm) + _pad8(dt) + _pad8(sp) + v.astype(v.dtype.newbyteorder("<")).tobytes()


class _File:
    def __init__(self):
        self.buf = bytearray(b"\0" * 96)  # superblock, written last

    def alloc(self, data: bytes, align: int = 8) -> int:
        while len(self.buf) % align:
            self.buf += b"\0"
        a = len(self.buf)
        self.buf += data
        return a

    def reserve(self, n: int) -> int:
        return self.alloc(b"\0" * n)

    def put(self, addr: int, data: bytes):
        self.buf[addr:addr + len(data)] = data


def _v1_messages(msgs) -> bytes:
    out = b""
    for t, body in msgs:
        body = _pad8(body)
        out += struct.pack("<HHB3x", t, len(body), 0) + body
    return out


def _object_header(f: _File, msgs, split: int | None = None) -> int:
    """A version-1 object header; with `split`, messages from index `split` go into a
    continuation block."""
    if split is None:
        block = _v1_messages(msgs)
        return f.alloc(struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(block)) + block)
    first, rest = msgs[:split], msgs[split:]
    cont_body = _v1_messages(rest)
    cont_addr = f.alloc(cont_body)
    block = _v1_messages(first + [(0x0010, struct.pack("<QQ", cont_addr, len(cont_body)))])
    return f.alloc(struct.pack("<BBHII4x", 1, 0, len(msgs) + 1, 1, len(block)) + block)


def _chunk_btree(f: _File, entries, rank: int, fanout: int = 4) -> int:
    """entries: (chunk offsets, stored size, filter mask, address); leaves of at most
    `fanout` chunks, one internal level above them when there are more."""
    def node(level, items):
        # items: (key offsets, size, mask, child address); the final key bounds the last child
        b = b"TREE" + struct.pack("<BBHQQ", 1, level, len(items), UNDEF, UNDEF)
        for off, size, mask, child in items:
            b += struct.pack("<II", size, mask) + b"".join(struct.pack("<Q", o) for o in off) + struct.pack("<Q", child)
        last = items[-1][0]
        b += struct.pack("<II", 0, 0) + b"".join(struct.pack("<Q", o + (1 << 20)) for o in last)
        return f.alloc(b)
    leaves = [entries[i:i + fanout] for i in range(0, len(entries), fanout)]
    addrs = [(leaf[0][0], 0, 0, node(0, leaf)) for leaf in leaves]
    if len(addrs) == 1:
        return addrs[0][3]
    return node(1, addrs)


def _dataset(f: _File, d: Data) -> int:
    a = np.ascontiguousarray(d.array)
    a = a.astype(a.dtype.newbyteorder("<"))
    msgs = [(0x0001, _space_msg(a.shape)), (0x0003, _dtype_msg(a.dtype)),
            (0x0005, struct.pack("<BBBBI", 2, 3, 2, 0, 0))]
    es = a.dtype.itemsize
    if d.layout == "contiguous":
        addr = f.alloc(a.tobytes()) if a.size else UNDEF
        msgs.append((0x0008, struct.pack("<BBQQ", 3, 1, addr, a.nbytes)))
    elif d.layout == "compact":
        msgs.append((0x0008, struct.pack("<BBH", 3, 0, a.nbytes) + a.tobytes()))
    else:
        chunk = tuple(d.chunk)
        filters = []
        if d.shuffle:
            filters.append((2, [es]))
        if d.deflate is not None:
            filters.append((1, [d.deflate]))
        entries = []
        grid = [range(0, s, c) for s, c in zip(a.shape, chunk)]
        for off in np.array(np.meshgrid(*grid, indexing="ij")).reshape(len(chunk), -1).T:
            block = np.zeros(chunk, a.dtype)
            sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(off, chunk, a.shape))
            block[tuple(slice(0, x.stop - x.start) for x in sl)] = a[sl]
            raw = block.tobytes()
            if d.shuffle:
                raw = np.frombuffer(raw, np.uint8).reshape(-1, es).T.copy().tobytes()
            if d.deflate is not None:
                raw = zlib.compress(raw, d.deflate)
            entries.append((list(off) + [0], len(raw), 0, f.alloc(raw)))
        bt = _chunk_btree(f, entries, a.ndim)
        lay = struct.pack("<BBBQ", 3, 2, a.ndim + 1, bt) + b"".join(struct.pack("<I", c) for c in chunk + (es,))
        if filters:
            fb = struct.pack("<BB6x", 1, len(filters))
            for fid, vals in filters:
                name = _pad8(b"deflate\0" if fid == 1 else b"shuffle\0")
                fb += struct.pack("<HHHH", fid, len(name), 0, len(vals)) + name
                fb += b"".join(struct.pack("<I", v) for v in vals) + (b"\0" * 4 if len(vals) % 2 else b"")
            msgs.append((0x000B, fb))
        msgs.append((0x0008, lay))
    for k, v in d.attrs.items():
        msgs.append((0x000C, _attr_msg(k, v)))
    return _object_header(f, msgs, split=3 if d.continuation else None)


def _group(f: _File, tree: dict) -> int:
    names = [k for k in tree if k != "attrs"]
    heap_data = b"\0" * 8  # offset 0: the empty name
    offsets = {}
    for k in names:
        offsets[k] = len(heap_data)
        heap_data += _pad8(k.encode() + b"\0")
    children = {}
    for k in names:
        v = tree[k]
        if isinstance(v, dict):
            children[k] = _group(f, v)
        else:
            children[k] = _dataset(f, v if isinstance(v, Data) else Data(np.asarray(v)))
    heap_addr_data = f.alloc(heap_data)
    heap = f.alloc(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), UNDEF, heap_addr_data))
    # symbol nodes of at most 8 entries (2 x leaf K = 4), names in ascending order
    order = sorted(names)
    snods = []
    for i in range(0, max(len(order), 1), 8):
        part = order[i:i + 8]
        b = b"SNOD" + struct.pack("<BBH", 1, 0, len(part))
        for k in part:
            b += struct.pack("<QQII16x", offsets[k], children[k], 0, 0)
        snods.append((part, f.alloc(b)))

    def gnode(level, items):
        # items: (first name of the child, last name, child address); keys are heap offsets
        b = b"TREE" + struct.pack("<BBHQQ", 0, level, len(items), UNDEF, UNDEF)
        b += struct.pack("<Q", 0)
        for _, last, child in items:
            b += struct.pack("<Q", child) + struct.pack("<Q", offsets[last] if last else 0)
        return f.alloc(b)
    leaf_items = [(p[0] if p else "", p[-1] if p else "", a) for p, a in snods]
    if len(leaf_items) <= 2:
        bt = gnode(0, leaf_items)
    else:  # two levels: pairs of symbol nodes under internal entries
        lower = []
        for i in range(0, len(leaf_items), 2):
            part = leaf_items[i:i + 2]
            lower.append((part[0][0], part[-1][1], gnode(0, part)))
        bt = gnode(1, lower)
    msgs = [(0x0011, struct.pack("<QQ", bt, heap))]
    for k, v in tree.get("attrs", {}).items():
        msgs.append((0x000C, _attr_msg(k, v)))
    return _object_header(f, msgs)


def write(path, tree: dict) -> None:
    f = _File()
    root = _group(f, tree)
    eof = len(f.buf)
    sb = SIG + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, 4, 16, 0)
    sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
    sb += struct.pack("<QQII16x", 0, root, 0, 0)  # root entry, no cached scratch
    f.put(0, sb)
    with open(path, "wb") as fh:
        fh.write(bytes(f.buf))
