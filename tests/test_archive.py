"""Reading rkyv archives of an ImmutableKdTree in place (kgpu_archive_inspect,
host only): archives written by the oracle's restatement of kiddo's
`rkyv::to_bytes` (oracle/rkyv_archive.py) read back field for field, for each
pointer width, dtype and stem order, and damaged archives are refused with a
status, never read out of bounds."""
import numpy as np
import pytest

import kiddo_b200 as kb
import oracle
from kiddo_b200 import _capi as C
from oracle import rkyv_archive as ra


def _tree(n, dtype, dims=3, bh=0, seed=0):
    P = np.random.default_rng(seed).random((n, dims)).astype(dtype)
    return oracle.OracleTree.build(P, block_height=bh).layout()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("bh", [0, 3, 4])
@pytest.mark.parametrize("width", [2, 4, 8])
def test_archive_fields_read_back(dtype, bh, width):
    n = 300 if width == 2 else 20_000  # 16-bit offsets limit the archive to 64 KiB
    lay = _tree(n, dtype, bh=bh)
    b = ra.write_layout(lay, width)
    info = kb.GpuTree.inspect_archive(b, dtype, 3, block_height=bh, pointer_width=width)
    assert info["stem_count"] == lay.stems.size and info["leaf_count"] == lay.leaf_count
    assert info["size"] == n and info["max_stem_level"] == lay.max_stem_level
    assert info["max_leaf_len"] == lay.max_leaf_len
    assert info["leaf_bytes_len"] == lay.leaf_bytes.size
    assert info["stems_offset"] % 128 == 0 and info["leaf_bytes_offset"] % 128 == 0
    assert info["resolution"] == C.RES_ARITHMETIC
    assert info["stems_depth"] == lay.max_stem_level + 1
    raw = np.frombuffer(b, dtype=np.uint8)
    stems = raw[info["stems_offset"]:info["stems_offset"] + lay.stems.nbytes].view(dtype)
    assert np.array_equal(stems, lay.stems)
    arena = raw[info["leaf_bytes_offset"]:info["leaf_bytes_offset"] + lay.leaf_bytes.size]
    assert np.array_equal(arena, lay.leaf_bytes)
    it = {2: np.uint16, 4: np.uint32, 8: np.uint64}[width]
    ex = raw[info["extents_offset"]:info["extents_offset"] + 2 * width * lay.leaf_count].view(it)
    assert np.array_equal(ex.reshape(-1, 2).astype(np.uint64), lay.extents)


def test_archive_reads_from_a_mapped_file(tmp_path):
    lay = _tree(5000, np.float32)
    path = tmp_path / "tree.rkyv"
    path.write_bytes(ra.write_layout(lay))
    info = kb.GpuTree.inspect_archive(str(path), np.float32, 3)
    assert info["size"] == 5000 and info["stem_count"] == lay.stems.size


def test_pristine_resolution_is_read_as_arithmetic():
    lay = _tree(3000, np.float64)
    info = kb.GpuTree.inspect_archive(ra.write_layout(lay, 4, "pristine"), np.float64, 3)
    assert info["resolution"] == C.RES_PRISTINE


def _expect_refusal(b, **kw):
    with pytest.raises(kb.KiddoGpuError) as e:
        kb.GpuTree.inspect_archive(b, np.float32, 3, **kw)
    assert e.value.status in (C.KGPU_EINVAL, C.KGPU_EUNSUPPORTED)


def test_damaged_archives_are_refused():
    lay = _tree(4000, np.float32)
    good = bytearray(ra.write_layout(lay, 4))
    L = ra.root_layout(4)
    root = len(good) - L["total"]
    _expect_refusal(bytes(good[:-4]))                       # truncated: root misplaced
    _expect_refusal(bytes(good[:10]))                       # shorter than the root
    for field in ("stems", "extents", "leaf_bytes"):
        for off, cnt in ((-(1 << 30), 1), (1 << 30, 1), (0, 1 << 31)):
            bad = bytearray(good)
            at = root + L[field]
            if cnt == 1:
                bad[at:at + 4] = int(off).to_bytes(4, "little", signed=True)
            else:
                bad[at + 4:at + 8] = int(cnt).to_bytes(4, "little")
            _expect_refusal(bytes(bad))
    bad = bytearray(good)
    bad[root + L["resolution"]] = 7                         # unknown enum tag
    _expect_refusal(bytes(bad))
    bad = bytearray(good)
    bad[root + L["size"]:root + L["size"] + 4] = (4001).to_bytes(4, "little")  # sizes disagree
    _expect_refusal(bytes(bad))
    _expect_refusal(bytes(good), pointer_width=3)
    f = kb.GpuTree._archive_format(np.float32, 3, 0, 4)
    f.big_endian = 1
    info = C.ArchiveInfo()
    assert C.lib().kgpu_archive_inspect(bytes(good), len(good), f, info) == C.KGPU_EUNSUPPORTED


def test_random_damage_never_reads_out_of_bounds():
    """Random bytes of the root replaced: the reader answers with a status
    (or with fields that stay inside the buffer), never a fault."""
    lay = _tree(2000, np.float32)
    good = ra.write_layout(lay, 4)
    L = ra.root_layout(4)
    rng = np.random.default_rng(12)
    for _ in range(400):
        bad = bytearray(good)
        for _ in range(rng.integers(1, 4)):
            bad[len(bad) - L["total"] + int(rng.integers(0, L["total"]))] = int(rng.integers(0, 256))
        try:
            info = kb.GpuTree.inspect_archive(bytes(bad), np.float32, 3)
        except kb.KiddoGpuError:
            continue
        for pos, count, elem in (("stems_offset", "stem_count", 4), ("extents_offset", "leaf_count", 8),
                                 ("leaf_bytes_offset", "leaf_bytes_len", 1)):
            assert info[pos] + info[count] * elem <= len(bad)
