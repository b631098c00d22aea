// archive.cpp — reads an rkyv 0.8 archive of an ImmutableKdTree in place.
//
// kiddo serialises a tree with `rkyv::to_bytes(&tree)` and reads it back
// zero-copy with `rkyv::access::<ArchivedKdTree<..>>` (src/kd_tree/mod.rs:
// 211-241, 282-372).  The archive is one byte buffer; its root object, the
// ArchivedKdTree, sits at the end of the buffer; every array is reached
// through a relative pointer (a signed offset from the pointer's own
// position) followed by its element count.  The fields, in declaration
// order, each aligned to its archived alignment (rkyv's derived archived
// structs are repr(C)):
//
//   stems                 ArchivedBox<AlignedArchiveSlice<[A]>>   rel. offset, len
//   leaves                ArchivedVecOfArenas (vec_of_arenas.rs:60-69):
//     leaf_extents          ArchivedVec<(usize, usize)>            rel. offset, len
//     leaf_bytes            ArchivedBox<AlignedArchiveSlice<[u8]>> rel. offset, len
//     size                  usize
//   stem_leaf_resolution  enum, u8 tag (0 Arithmetic, 1 Pristine, 2 Mapped),
//                         then the variant's fields (stem_leaf_resolution.rs:28-68):
//                         Arithmetic / Pristine { stems_depth, leaf_count },
//                         Mapped { min_stem_leaf_idx, leaf_idx_map: vec of usize,
//                         all-ones = None (rkyv/adapters.rs:168-237) }
//   size                  usize
//   max_stem_level        i32
//   max_leaf_len          usize
//
// where usize and the relative offsets are `pointer_width` bytes wide (rkyv's
// pointer_width_16/32/64 features; 32 is rkyv's default) and little-endian.
// The stems and the leaf arena are written 128-byte aligned inside the
// buffer (AsAlignedCachelineABox, src/rkyv/adapters.rs:114-165).
//
// Every offset and length is checked against the buffer before anything is
// read through it, so a buffer that is not such an archive gives KGPU_EINVAL,
// never an out-of-bounds read.  The stems and the arena are then uploaded
// straight from the caller's buffer (for example a read-only mmap of the
// archive file); only the extents are converted on the host.
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/kiddo_gpu.h"
#include "kgpu_internal.h"

namespace kgpu {
namespace {

struct Reader {
  const uint8_t* p;
  uint64_t len;
  uint32_t w;  // pointer width in bytes

  // little-endian unsigned of `n` bytes at `pos` (pos + n <= len checked by the caller)
  uint64_t u(uint64_t pos, uint32_t n) const {
    uint64_t v = 0;
    for (uint32_t i = 0; i < n; ++i) v |= uint64_t(p[pos + i]) << (8 * i);
    return v;
  }
  int64_t s(uint64_t pos, uint32_t n) const {
    const uint64_t v = u(pos, n);
    const uint32_t bits = 8 * n;
    return bits == 64 ? int64_t(v) : int64_t(v << (64 - bits)) >> (64 - bits);
  }
};

uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Byte layout of the archived root for a pointer width: field offsets and
// the struct's size.
struct RootLayout {
  uint64_t stems, extents, leaf_bytes, leaves_size, resolution, size, max_stem_level,
      max_leaf_len, total, align;
};

RootLayout root_layout(uint32_t w) {
  RootLayout L{};
  uint64_t pos = 0;
  const uint64_t a32 = 4;
  L.stems = pos;  // rel. pointer + len
  pos += 2 * w;
  // ArchivedVecOfArenas: vec (2w), box (2w), usize (w); align w
  L.extents = pos;
  pos += 2 * w;
  L.leaf_bytes = pos;
  pos += 2 * w;
  L.leaves_size = pos;
  pos += w;
  pos = align_up(pos, w);  // the nested struct's size is a multiple of its alignment
  // the resolution enum: a u8 tag, then a variant of up to three usize-wide
  // fields (Mapped: min_stem_leaf_idx, then a vec of 2w); alignment w
  pos = align_up(pos, w);
  L.resolution = pos;
  pos += 4 * w;
  L.size = pos;
  pos += w;
  pos = align_up(pos, a32);
  L.max_stem_level = pos;
  pos += 4;
  pos = align_up(pos, w);
  L.max_leaf_len = pos;
  pos += w;
  L.align = w > a32 ? w : a32;
  L.total = align_up(pos, L.align);
  return L;
}

// Target position and element count of the relative pointer at `at`, checked
// to lie inside the buffer with `elem` bytes per element and `align`-byte
// alignment.
int rel_slice(const Reader& r, uint64_t at, uint64_t elem, uint64_t align, const char* what,
              uint64_t* pos, uint64_t* count) {
  const int64_t off = r.s(at, r.w);
  const uint64_t n = r.u(at + r.w, r.w);
  *count = n;
  if (n == 0) {
    *pos = 0;
    return KGPU_OK;
  }
  const int64_t target = int64_t(at) + off;
  if (target < 0 || uint64_t(target) > r.len)
    return set_error(KGPU_EINVAL, std::string("archive: ") + what + " points outside the buffer");
  if (elem && n > (r.len - uint64_t(target)) / elem)
    return set_error(KGPU_EINVAL, std::string("archive: ") + what + " runs past the buffer");
  if (uint64_t(target) % align)
    return set_error(KGPU_EINVAL, std::string("archive: ") + what + " is misaligned");
  *pos = uint64_t(target);
  return KGPU_OK;
}

}  // namespace
}  // namespace kgpu

using namespace kgpu;

extern "C" {

int32_t kgpu_archive_inspect(const void* bytes, uint64_t len, const kgpu_archive_format* fmt,
                             kgpu_archive_info* info) {
  if (!bytes || !fmt || !info) return set_error(KGPU_EINVAL, "NULL argument");
  std::memset(info, 0, sizeof(*info));
  if (fmt->abi_version != KGPU_ABI_VERSION) return set_error(KGPU_EINVAL, "abi_version mismatch");
  if (fmt->dtype != KGPU_F32 && fmt->dtype != KGPU_F64)
    return set_error(KGPU_EINVAL, "dtype must be KGPU_F32 or KGPU_F64");
  if (fmt->dims < 1 || fmt->dims > uint32_t(kMaxDims))
    return set_error(KGPU_EUNSUPPORTED, "dims must be 1..4");
  if (fmt->pointer_width != 2 && fmt->pointer_width != 4 && fmt->pointer_width != 8)
    return set_error(KGPU_EINVAL, "pointer_width must be 2, 4 or 8 bytes");
  if (fmt->big_endian) return set_error(KGPU_EUNSUPPORTED, "big-endian archives are not read");
  const Reader r{static_cast<const uint8_t*>(bytes), len, fmt->pointer_width};
  const RootLayout L = root_layout(r.w);
  if (len < L.total) return set_error(KGPU_EINVAL, "archive shorter than its root object");
  const uint64_t root = len - L.total;  // rkyv places the root at the end
  if (root % L.align) return set_error(KGPU_EINVAL, "archive root is misaligned");
  // positions are checked for alignment relative to the buffer start, as
  // rkyv lays them out; the buffer itself may sit anywhere (reads are bytewise)
  const uint64_t sa = fmt->dtype == KGPU_F64 ? 8 : 4;
  uint64_t pos, n;
  int st;
  if ((st = rel_slice(r, root + L.stems, sa, sa, "stems", &pos, &n)) != KGPU_OK) return st;
  info->stems_offset = pos;
  info->stem_count = n;
  if ((st = rel_slice(r, root + L.extents, 2 * r.w, r.w, "leaf_extents", &pos, &n)) != KGPU_OK)
    return st;
  info->extents_offset = pos;
  info->leaf_count = n;
  if ((st = rel_slice(r, root + L.leaf_bytes, 1, 1, "leaf_bytes", &pos, &n)) != KGPU_OK) return st;
  info->leaf_bytes_offset = pos;
  info->leaf_bytes_len = n;
  const uint64_t tag = r.u(root + L.resolution, 1);
  if (tag > 2) return set_error(KGPU_EINVAL, "archive: unknown stem/leaf resolution tag");
  info->resolution = tag == 0 ? KGPU_RES_ARITHMETIC : tag == 1 ? KGPU_RES_PRISTINE
                                                               : KGPU_RES_MAPPED;
  if (tag < 2) {
    info->stems_depth = r.u(root + L.resolution + r.w, r.w);
    info->resolution_leaf_count = r.u(root + L.resolution + 2 * r.w, r.w);
  } else {
    // Mapped { min_stem_leaf_idx: usize, leaf_idx_map: Vec<usize with the
    // all-ones sentinel for None> }
    info->min_stem_leaf_idx = r.u(root + L.resolution + r.w, r.w);
    if ((st = rel_slice(r, root + L.resolution + 2 * r.w, r.w, r.w, "leaf_idx_map", &pos, &n)) !=
        KGPU_OK)
      return st;
    info->map_offset = pos;
    info->map_len = n;
  }
  info->size = r.u(root + L.size, r.w);
  info->leaves_size = r.u(root + L.leaves_size, r.w);
  info->max_stem_level = int32_t(r.s(root + L.max_stem_level, 4));
  info->max_leaf_len = r.u(root + L.max_leaf_len, r.w);
  info->root_offset = root;
  if (info->leaves_size != info->size)
    return set_error(KGPU_EINVAL, "archive: the leaves' size and the tree's size differ");
  if (tag < 2 && info->resolution_leaf_count != info->leaf_count)
    return set_error(KGPU_EINVAL, "archive: resolution leaf_count != number of leaf extents");
  return KGPU_OK;
}

int32_t kgpu_tree_create_from_archive(const void* bytes, uint64_t len,
                                      const kgpu_archive_format* fmt, void* stream,
                                      kgpu_tree** out) {
  if (!out) return set_error(KGPU_EINVAL, "NULL argument");
  *out = nullptr;
  kgpu_archive_info info;
  int st = kgpu_archive_inspect(bytes, len, fmt, &info);
  if (st != KGPU_OK) return st;
  const Reader r{static_cast<const uint8_t*>(bytes), len, fmt->pointer_width};
  const bool mapped = info.resolution == KGPU_RES_MAPPED;
  std::vector<uint64_t> map;
  if (mapped) {
    try {
      map.resize(info.map_len);
    } catch (const std::bad_alloc&) {
      return set_error(KGPU_ENOMEM, "host allocation failed");
    }
    const uint64_t none = r.w == 8 ? ~uint64_t(0) : (uint64_t(1) << (8 * r.w)) - 1;
    for (uint64_t i = 0; i < info.map_len; ++i) {
      const uint64_t v = r.u(info.map_offset + i * r.w, r.w);
      map[i] = v == none ? ~uint64_t(0) : v;
    }
  }
  std::vector<uint64_t> ex;
  try {
    ex.resize(2 * info.leaf_count);
  } catch (const std::bad_alloc&) {
    return set_error(KGPU_ENOMEM, "host allocation failed");
  }
  for (uint64_t l = 0; l < info.leaf_count; ++l) {
    ex[2 * l] = r.u(info.extents_offset + 2 * l * r.w, r.w);
    ex[2 * l + 1] = r.u(info.extents_offset + (2 * l + 1) * r.w, r.w);
  }
  kgpu_tree_desc d;
  std::memset(&d, 0, sizeof(d));
  d.abi_version = KGPU_ABI_VERSION;
  d.dtype = fmt->dtype;
  d.dims = fmt->dims;
  d.item_size = 4;
  d.bucket_size = 32;
  d.stem_strategy = fmt->stem_strategy;
  d.block_height = fmt->block_height;
  d.resolution = mapped ? KGPU_RES_MAPPED : KGPU_RES_ARITHMETIC;  // Pristine: arithmetic
  const uint8_t* base = static_cast<const uint8_t*>(bytes);
  d.stems = info.stem_count ? base + info.stems_offset : nullptr;
  d.stem_count = info.stem_count;
  d.leaf_bytes = info.leaf_bytes_len ? base + info.leaf_bytes_offset : nullptr;
  d.leaf_bytes_len = info.leaf_bytes_len;
  d.leaf_extents = ex.empty() ? nullptr : ex.data();
  d.leaf_count = info.leaf_count;
  d.max_stem_level = info.max_stem_level;
  d.size = info.size;
  d.max_leaf_len = info.max_leaf_len;
  // kgpu_tree_create checks the layout itself (extents inside the arena,
  // leaf count against the stem depth or every walk against the leaf map,
  // sizes) before it touches the device
  if (mapped) {
    const kgpu_leaf_map lm{map.empty() ? nullptr : map.data(), map.size(),
                           info.min_stem_leaf_idx};
    return kgpu_tree_create_mapped(&d, &lm, stream, out);
  }
  return kgpu_tree_create(&d, stream, out);
}

}  // extern "C"
