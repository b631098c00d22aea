"""A restatement of how kiddo's `rkyv::to_bytes(&tree)` lays out an
ImmutableKdTree archive (test infrastructure: the archive upload is checked
against archives this writes; parity unpinned against an archive written by
the Rust crate itself, which cannot be built here).

rkyv 0.8's serializer writes every field's out-of-line data first, in field
order, then the root object at the end of the buffer, aligned for its type.
For `KdTree<A, u32, SS, VecOfArenas<A, u32, K, 32>, K, 32>`
(src/kd_tree/mod.rs:211-241, src/leaf_strategy/vec_of_arenas.rs:60-69):

1. `stems` with `AsAlignedCachelineABox` (src/rkyv/adapters.rs:126-141 and
   AlignedArchiveSlice::serialize_unsized, :93-111): zero padding up to the
   next 128-byte boundary (align_writer_to, :218-236), then the stems as
   little-endian A values;
2. `leaves.leaf_extents`, a Vec<(usize, usize)>: aligned for the archived
   pair, then each (offset, len) as two archived usizes;
3. `leaves.leaf_bytes`, again AsAlignedCachelineABox: padding to 128, then
   the arena bytes;
4. the root: repr(C) fields in declaration order, each relative pointer the
   signed distance from the pointer's own position to its data, followed by
   the element count (see kiddo_b200/csrc/archive.cpp for the field table).

`pointer_width` is the byte width of rkyv's archived usize and relative
offsets (its pointer_width_16 / _32 (default) / _64 features).
"""
from __future__ import annotations

import struct

import numpy as np

CACHELINE = 128


def _align(buf: bytearray, a: int):
    buf.extend(b"\0" * ((-len(buf)) % a))


def _uint(v: int, w: int) -> bytes:
    return int(v).to_bytes(w, "little", signed=False)


def _int(v: int, w: int) -> bytes:
    return int(v).to_bytes(w, "little", signed=True)


def root_layout(w: int):
    """Field offsets of the archived root and its size (archive.cpp's table)."""
    def up(x, a):
        return (x + a - 1) // a * a
    pos = 0
    L = {"stems": 0}
    pos += 2 * w
    L["extents"] = pos
    pos += 2 * w
    L["leaf_bytes"] = pos
    pos += 2 * w
    L["leaves_size"] = pos
    pos = up(pos + w, w)
    L["resolution"] = pos
    pos += 4 * w
    L["size"] = pos
    pos = up(pos + w, 4)
    L["max_stem_level"] = pos
    pos = up(pos + 4, w)
    L["max_leaf_len"] = pos
    pos += w
    align = max(w, 4)
    L["align"] = align
    L["total"] = up(pos, align)
    return L


def write_archive(stems, leaf_bytes, extents, size, max_stem_level, max_leaf_len,
                  pointer_width=4, resolution="arithmetic", leaf_map=None, map_min=0):
    """The archive bytes of a tree layout.  `stems` is the stem array in the
    tree's dtype, `leaf_bytes` the VecOfArenas arena, `extents` [leaf_count, 2]
    (offset, len); `resolution` is "arithmetic" or "pristine" (tags 0 and 1,
    fields stems_depth = max_stem_level + 1 and leaf_count), or "mapped" (tag
    2: min_stem_leaf_idx, then leaf_idx_map as a vec of usize written after the
    arena, None as the all-ones usize, OptionNonMaxUsizeAsUsize,
    src/rkyv/adapters.rs:168-237)."""
    w = int(pointer_width)
    stems = np.ascontiguousarray(stems)
    leaf_bytes = np.ascontiguousarray(leaf_bytes, dtype=np.uint8)
    extents = np.ascontiguousarray(extents, dtype=np.uint64).reshape(-1, 2)
    buf = bytearray()
    # 1. stems: padding to a cache line, then the values
    _align(buf, CACHELINE)
    stems_pos = len(buf)
    buf.extend(stems.astype(stems.dtype.newbyteorder("<"), copy=False).tobytes())
    # 2. leaf_extents: aligned for the (usize, usize) pair
    _align(buf, w)
    ext_pos = len(buf)
    for off, ln in extents:
        buf.extend(_uint(off, w) + _uint(ln, w))
    # 3. leaf_bytes: padding to a cache line, then the arena
    _align(buf, CACHELINE)
    arena_pos = len(buf)
    buf.extend(leaf_bytes.tobytes())
    # 3b. the Mapped resolution's leaf_idx_map
    map_pos = 0
    if resolution == "mapped":
        _align(buf, w)
        map_pos = len(buf)
        none = (1 << (8 * w)) - 1
        for v in np.asarray(leaf_map, dtype=np.uint64):
            buf.extend(_uint(none if int(v) == (1 << 64) - 1 else int(v), w))
    # 4. the root, aligned for its type
    L = root_layout(w)
    _align(buf, L["align"])
    root = len(buf)
    body = bytearray(L["total"])

    def put(at, data):
        body[at:at + len(data)] = data

    put(L["stems"], _int(stems_pos - (root + L["stems"]), w) + _uint(stems.size, w))
    put(L["extents"], _int(ext_pos - (root + L["extents"]), w) + _uint(extents.shape[0], w))
    put(L["leaf_bytes"], _int(arena_pos - (root + L["leaf_bytes"]), w) +
        _uint(leaf_bytes.size, w))
    put(L["leaves_size"], _uint(size, w))
    tag = {"arithmetic": 0, "pristine": 1, "mapped": 2}[resolution]
    put(L["resolution"], bytes([tag]))
    if tag == 2:
        at = root + L["resolution"] + 2 * w
        n = 0 if leaf_map is None else len(leaf_map)
        put(L["resolution"] + w, _uint(map_min, w) + _int(map_pos - at if n else 0, w) +
            _uint(n, w))
    else:
        put(L["resolution"] + w, _uint(max_stem_level + 1, w) + _uint(extents.shape[0], w))
    put(L["size"], _uint(size, w))
    put(L["max_stem_level"], struct.pack("<i", int(max_stem_level)))
    put(L["max_leaf_len"], _uint(max_leaf_len, w))
    buf.extend(body)
    return bytes(buf)


def write_layout(lay, pointer_width=4, resolution=None):
    """write_archive over an oracle.Layout (Mapped when the layout has a leaf map)."""
    if resolution is None:
        resolution = "mapped" if getattr(lay, "leaf_map", None) is not None else "arithmetic"
    return write_archive(lay.stems, lay.leaf_bytes, lay.extents, lay.size, lay.max_stem_level,
                         lay.max_leaf_len, pointer_width, resolution,
                         getattr(lay, "leaf_map", None), getattr(lay, "map_min", 0))
