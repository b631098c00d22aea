/*
 * kiddo_gpu.h — C ABI of the B200 batched query engine for kiddo's
 * ImmutableKdTree (KdTree<A, u32, Eytzinger, VecOfArenas<A,u32,K,32>, K, 32>).
 *
 * The engine takes the reference builder's own layout — the Eytzinger stem
 * array, the VecOfArenas leaf arena bytes and the (offset, len) leaf extents —
 * uploads it to HBM (3-D leaves re-encoded as one row per point, the same
 * points in the same order; the reference's bytes read back unchanged) and
 * answers whole batches of queries with CUDA kernels for sm_100a.  Results
 * are bit-identical to the reference's scalar `.execute()` path on the same
 * tree and queries.
 *
 * Conventions
 *  - Every entry point returns a kgpu_status; nothing aborts or throws across
 *    the ABI.  kgpu_last_error() gives a message for the calling thread.
 *  - Host arrays passed in are borrowed for the duration of the call only.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *    With KGPU_FLAG_HOST_BUFFERS clear, query inputs and outputs are device
 *    pointers and the call is asynchronous on `stream`.  With the flag set
 *    they are host pointers (pinned or pageable); the library stages them
 *    through HBM on `stream` and returns after the results are back.
 *  - Trees are immutable after creation; a tree handle may be queried from
 *    several host threads on different streams at once.
 *
 * Reference surface replaced (paths relative to the kiddo repository root):
 *   KdTree::query(&q) -> QueryBuilder ... .execute()   src/kd_tree/query/builder.rs:2318-2331, :1693
 *   the per-family execute impls                         src/kd_tree/query/builder.rs:4444-5419
 *   KdTreeAccessor (layout read access)                  src/traits/kd_tree.rs:15-46
 */
#ifndef KIDDO_GPU_H
#define KIDDO_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KGPU_ABI_VERSION 1u

typedef enum kgpu_status {
  KGPU_OK = 0,
  KGPU_EINVAL = 1,        /* invalid argument (bad handle, size, box <= 0, k == 0 ...) */
  KGPU_EUNSUPPORTED = 2,  /* layout or option this engine does not handle */
  KGPU_ENOMEM = 3,        /* device or host allocation failed */
  KGPU_ECUDA = 4,         /* a CUDA runtime call failed */
  KGPU_ETIMEDOUT = 5,     /* a bounded device wait gave up */
  KGPU_EOVERFLOW = 6,     /* result capacity or a size limit exceeded */
  KGPU_ENOTREADY = 7
} kgpu_status;

typedef enum kgpu_dtype { KGPU_F32 = 0, KGPU_F64 = 1 } kgpu_dtype;

typedef enum kgpu_stem_strategy {
  KGPU_STEM_EYTZINGER = 0, /* src/stem_strategy/eytzinger/mod.rs */
  KGPU_STEM_DONNELLY = 1   /* src/stem_strategy/donnelly/core.rs, Donnelly<3> and Donnelly<4> */
} kgpu_stem_strategy;

typedef enum kgpu_resolution {
  KGPU_RES_ARITHMETIC = 0, /* OwnedStemLeafResolution::Arithmetic, stem_leaf_resolution.rs:28-68 */
  KGPU_RES_MAPPED = 1,
  KGPU_RES_PRISTINE = 2
} kgpu_resolution;

typedef enum kgpu_metric {
  KGPU_SQUARED_EUCLIDEAN = 0, /* src/dist/squared_euclidean/mod.rs:21-40 */
  KGPU_MANHATTAN = 1,         /* src/dist/manhattan/mod.rs:21-48 */
  KGPU_CHEBYSHEV = 2,         /* src/dist/chebyshev/mod.rs:19-59; not with periodic boxes */
  KGPU_MINKOWSKI3 = 3,        /* Minkowski<3>, src/dist/minkowski/mod.rs:19-58; not periodic */
  KGPU_MINKOWSKI4 = 4         /* Minkowski<4>; not periodic */
} kgpu_metric;

typedef enum kgpu_family {
  KGPU_NEAREST_ONE = 0,        /* .nearest_one::<D>()                 builder.rs:4444 */
  KGPU_APPROX_NEAREST_ONE = 1, /* .nearest_one::<D>().approx()        builder.rs:4502 */
  KGPU_NEAREST_N = 2,          /* .nearest_n::<D>(k)                  builder.rs:4629/:4706 */
  KGPU_NEAREST_N_WITHIN = 3,   /* .nearest_n::<D>(k).within(r)        builder.rs:4783/:4874 */
  KGPU_WITHIN = 4,             /* .within::<D>(r)                     builder.rs:4965 */
  KGPU_WITHIN_UNSORTED = 5,    /* .within::<D>(r).unsorted()          builder.rs:5048 */
  KGPU_BEST_N_WITHIN = 6       /* .best_n_within::<D>(r, n)           builder.rs:5419 */
} kgpu_family;

/* Query flags */
#define KGPU_FLAG_HOST_BUFFERS 0x1u  /* queries/outputs are host pointers */
#define KGPU_FLAG_SPATIAL_ORDER 0x2u /* process queries grouped by leaf (same results); */
                                     /* default for >= 65,536 queries on >= 4,096 leaves */
#define KGPU_FLAG_NO_SPATIAL_ORDER 0x10u /* process queries in the order given */
#define KGPU_FLAG_ENGINE_WARP 0x4u   /* force one warp per query (same results) */
#define KGPU_FLAG_ENGINE_THREAD 0x8u /* force one thread per query (same results) */
#define KGPU_FLAG_ENGINE_COOP 0x20u  /* one walk per thread, each leaf scanned by the whole
                                        warp (same results; nearest_n sorted, k <= 32) */

/* Layout of one ImmutableKdTree as the reference stores it
 * (src/kd_tree/mod.rs:221-241, src/leaf_strategy/vec_of_arenas.rs:60-69). */
typedef struct kgpu_tree_desc {
  uint32_t abi_version;      /* KGPU_ABI_VERSION */
  int32_t dtype;             /* kgpu_dtype of the axis type A */
  uint32_t dims;             /* K, 1..4 */
  uint32_t item_size;        /* sizeof(T); 4 (u32) */
  uint32_t bucket_size;      /* B; 32 */
  int32_t stem_strategy;     /* kgpu_stem_strategy */
  uint32_t block_height;     /* Donnelly BH; 0 for Eytzinger */
  int32_t resolution;        /* kgpu_resolution */
  const void* stems;         /* stem_count values of type A, Eytzinger order, +inf = no split */
  uint64_t stem_count;
  const uint8_t* leaf_bytes; /* VecOfArenas arena: tiles 32/8/4/2/1, K columns then items */
  uint64_t leaf_bytes_len;
  const uint64_t* leaf_extents; /* leaf_count pairs (byte offset, len) */
  uint64_t leaf_count;
  int32_t max_stem_level;    /* KdTree::max_stem_level, -1 for a stemless tree */
  uint32_t reserved0;
  uint64_t size;             /* number of points */
  uint64_t max_leaf_len;
} kgpu_tree_desc;

/* A FlatVec tree (src/leaf_strategy/flat_vec.rs:20-26). */
typedef struct kgpu_flatvec_desc {
  uint32_t abi_version;      /* KGPU_ABI_VERSION */
  int32_t dtype;             /* kgpu_dtype of the axis type A */
  uint32_t dims;             /* K, 1..4 */
  int32_t stem_strategy;     /* kgpu_stem_strategy */
  uint32_t block_height;     /* Donnelly BH; 0 for Eytzinger */
  int32_t max_stem_level;    /* KdTree::max_stem_level, -1 for a stemless tree */
  const void* stems;         /* stem_count values of type A */
  uint64_t stem_count;
  const void* columns[4];    /* leaf_points: `dims` arrays of `size` values of A */
  const uint32_t* items;     /* leaf_items: `size` values */
  const uint32_t* extents;   /* leaf_extents: leaf_count (start, end) pairs, in points */
  uint64_t leaf_count;
  uint64_t size;             /* number of points */
} kgpu_flatvec_desc;

/* A VecOfArrays tree (src/leaf_strategy/vec_of_arrays.rs:51-97): one LeafNode
 * per leaf, `bucket` (B) slots each, its first `size` slots live. */
typedef struct kgpu_vecofarrays_desc {
  uint32_t abi_version;      /* KGPU_ABI_VERSION */
  int32_t dtype;             /* kgpu_dtype of the axis type A */
  uint32_t dims;             /* K, 1..4 */
  int32_t stem_strategy;     /* kgpu_stem_strategy */
  uint32_t block_height;     /* Donnelly BH; 0 for Eytzinger */
  int32_t max_stem_level;    /* KdTree::max_stem_level, -1 for a stemless tree */
  const void* stems;         /* stem_count values of type A */
  uint64_t stem_count;
  uint32_t bucket;           /* B, 1..65536 */
  uint32_t reserved0;
  const void* content_points; /* leaf_count * dims * bucket values of A: leaf l's
                                 content_points[d][i] at (l * dims + d) * bucket + i */
  const uint32_t* content_items; /* leaf_count * bucket values: leaf l's slot i at l * bucket + i */
  const uint64_t* sizes;     /* leaf_count live-entry counts, each <= bucket */
  uint64_t leaf_count;
} kgpu_vecofarrays_desc;

typedef struct kgpu_query_desc {
  uint32_t abi_version;   /* KGPU_ABI_VERSION */
  int32_t family;         /* kgpu_family */
  int32_t metric;         /* kgpu_metric */
  uint32_t max_qty;       /* k for nearest_n*, n for best_n_within: 1..1,048,576 on 2-D
                             and 3-D trees (lists above 256, Donnelly lists above 32 and
                             periodic lists above 32 in the output rows); 1..256 on 1-D
                             and 4-D trees (periodic: 1..32) */
  double radius;          /* metric units (squared distance for SquaredEuclidean); cast to A */
  int32_t exclusive;      /* .exclusive_boundaries(): strict `< radius` */
  int32_t sorted;         /* 1 = default sorted output, 0 = .unsorted() */
  const void* periodic_box; /* host pointer to K values of A (each > 0), or NULL: Cartesian */
  uint32_t flags;         /* KGPU_FLAG_* */
  uint32_t tuning;        /* launch knobs, same results (0 = defaults): KGPU_TUNE_REFILL(n),
                             KGPU_TUNE_CHUNK_LOG2(c) */
} kgpu_query_desc;

/* kgpu_query_desc::tuning: the lane-refilled kernels refill a warp's idle
 * lanes once n of them (1..32; default 24) are idle, and hand queries to a
 * warp 2^c at a time (c in 5..10; default 64 queries). */
#define KGPU_TUNE_REFILL(n) ((uint32_t)(n) & 0x3fu)
#define KGPU_TUNE_CHUNK_LOG2(c) (((uint32_t)(c) & 0xfu) << 8)

typedef struct kgpu_layout kgpu_layout; /* host-side tree layout built by this library */
typedef struct kgpu_tree kgpu_tree;     /* device-resident tree */

/* ---- errors ------------------------------------------------------------ */
const char* kgpu_last_error(void);
const char* kgpu_status_string(int32_t status);
uint32_t kgpu_abi_version(void);

/* ---- host construction -------------------------------------------------
 * Builds the ImmutableKdTree layout with the reference's soft-bucket bulk
 * construction (src/kd_tree/construction.rs:413-539, 868-968, 1089-1175;
 * VecOfArenas::append_leaf src/leaf_strategy/vec_of_arenas.rs:292-323).
 * Replaces KdTree::new_from_slice (items NULL: item = source index,
 * construction.rs:278-303) and KdTree::new_from_entries (construction.rs:403-409).
 * `points` is n rows of `dims` values of `dtype`.  Points inside a leaf are
 * stored in ascending source index. */
int32_t kgpu_layout_build(int32_t dtype, uint32_t dims, const void* points,
                          const uint32_t* items, uint64_t n, int32_t nthreads,
                          kgpu_layout** out);
/* The same construction over another stem order (replaces KdTree<A, u32, SS, ...>
 * ::new_from_slice / new_from_entries for SS = Eytzinger or Donnelly<BH>,
 * src/lib.rs:235, construction.rs:431-469): stem_strategy KGPU_STEM_EYTZINGER
 * (block_height ignored) or KGPU_STEM_DONNELLY with block_height 3 or 4, the
 * heights the reference uses (Donnelly<3> for f64, Donnelly<4> for f32 trees). */
int32_t kgpu_layout_build_stems(int32_t dtype, uint32_t dims, const void* points,
                                const uint32_t* items, uint64_t n, int32_t stem_strategy,
                                uint32_t block_height, int32_t nthreads, kgpu_layout** out);
/* Fills `desc` with pointers into the layout's own storage (valid until free). */
int32_t kgpu_layout_describe(const kgpu_layout* layout, kgpu_tree_desc* desc);
int32_t kgpu_layout_free(kgpu_layout* layout);

/* ---- device trees --------------------------------------------------------
 * Upload a layout (one the reference built, or kgpu_layout_build's) to the
 * current CUDA device.  Stems are copied unchanged; extents are re-encoded as
 * 32-bit (offset / 8, len) pairs; 3-D leaves are re-encoded as rows (f32: 16
 * bytes per point at the same offsets, which must then be multiples of 16, as
 * the reference's are; f64: 32 bytes per point at offsets of their own).
 * kgpu_tree_read_layout returns the layout's original bytes. */
int32_t kgpu_tree_create(const kgpu_tree_desc* desc, void* stream, kgpu_tree** out);
/* Uploads a VecOfArrays tree (KdTree<A, u32, SS, VecOfArrays<A, u32, K, B>, K, B>,
 * src/leaf_strategy/vec_of_arrays.rs:51-97, append_leaf :249-275): its stems and
 * each leaf's live slots, in slot order.  Construction hands every leaf
 * strategy the same leaf chunks in the same order, so the leaves are re-encoded
 * on the host as VecOfArenas tiles and uploaded as kgpu_tree_create does. */
int32_t kgpu_tree_create_vecofarrays(const kgpu_vecofarrays_desc* desc, void* stream,
                                     kgpu_tree** out);
/* ---- Mapped stem/leaf resolution (MutableKdTree) -------------------------
 * OwnedStemLeafResolution::Mapped (src/kd_tree/stem_leaf_resolution.rs:53-66,
 * 77-120): a terminal stem maps straight to a leaf, so leaves may sit at any
 * depth.  kiddo's MutableKdTree (KdTree<A, u32, Eytzinger, VecOfArrays<..>>,
 * src/lib.rs:274-275) uses it from bulk construction on (hard buckets,
 * construction.rs:413-539, 695-864, 972-1009) and keeps it through leaf
 * splits (:19-130).  Queries walk such trees with the reference's scalar
 * backtracking (orchestrator/mod.rs:214-345, 607-669), either stem order;
 * 2-D and 3-D trees.  The map is checked at upload: every walk from the root
 * must end at a mapped terminal stem. */
typedef struct kgpu_leaf_map {
  const uint64_t* leaf_idx_map; /* `len` entries: leaf index of stem min_stem_leaf_idx + i,
                                   or UINT64_MAX for None (not terminal) */
  uint64_t len;
  uint64_t min_stem_leaf_idx;
} kgpu_leaf_map;
/* kgpu_tree_create for desc->resolution == KGPU_RES_MAPPED. */
int32_t kgpu_tree_create_mapped(const kgpu_tree_desc* desc, const kgpu_leaf_map* map,
                                void* stream, kgpu_tree** out);
/* kgpu_tree_create_vecofarrays with a Mapped resolution: a MutableKdTree's
 * own leaves and map. */
int32_t kgpu_tree_create_vecofarrays_mapped(const kgpu_vecofarrays_desc* desc,
                                            const kgpu_leaf_map* map, void* stream,
                                            kgpu_tree** out);

/* ---- upload from an rkyv archive -----------------------------------------
 * Replaces `rkyv::access::<ArchivedKdTree<A, u32, SS, VecOfArenas<..>, K, 32>>`
 * followed by the per-query `.execute()` on the archived tree
 * (src/kd_tree/mod.rs:282-372, src/rkyv/adapters.rs:114-237,
 * src/rkyv/query.rs): the archive's stems and leaf arena are uploaded straight
 * from `bytes` (for example a read-only mmap of the archive file; registering
 * that mapping with cudaHostRegister lets the copies run at bus speed), with
 * no deserialisation.  The archive carries no type information, so `fmt`
 * names the tree's type parameters and rkyv's format features. */
typedef struct kgpu_archive_format {
  uint32_t abi_version;   /* KGPU_ABI_VERSION */
  int32_t dtype;          /* kgpu_dtype of A */
  uint32_t dims;          /* K, 1..4 */
  int32_t stem_strategy;  /* kgpu_stem_strategy of SS */
  uint32_t block_height;  /* Donnelly BH; 0 for Eytzinger */
  uint32_t pointer_width; /* bytes of rkyv's archived usize and relative offsets: 2, 4
                             (rkyv's default, pointer_width_32) or 8 */
  uint32_t big_endian;    /* 0 (rkyv's default little_endian); big-endian is refused */
  uint32_t reserved0;
} kgpu_archive_format;

/* What kgpu_archive_inspect reads off an archive (offsets are byte positions
 * in the buffer). */
typedef struct kgpu_archive_info {
  uint64_t root_offset;
  uint64_t stems_offset, stem_count;
  uint64_t extents_offset, leaf_count;
  uint64_t leaf_bytes_offset, leaf_bytes_len;
  int32_t resolution;     /* a kgpu_resolution value: Arithmetic, Pristine or Mapped */
  int32_t max_stem_level;
  uint64_t stems_depth, resolution_leaf_count; /* Arithmetic / Pristine fields */
  uint64_t size, leaves_size, max_leaf_len;
  uint64_t map_offset, map_len, min_stem_leaf_idx; /* Mapped fields (leaf_idx_map) */
} kgpu_archive_info;

/* Checks an archive's structure (every relative pointer and length inside the
 * buffer) and reports its fields; touches no device. */
int32_t kgpu_archive_inspect(const void* bytes, uint64_t len, const kgpu_archive_format* fmt,
                             kgpu_archive_info* info);
/* kgpu_tree_create over an archive in place (kgpu_tree_create_mapped for a
 * Mapped resolution, whose leaf_idx_map entries equal to the all-ones usize
 * are None, src/rkyv/adapters.rs:168-237); Pristine resolves arithmetically.
 * `bytes` is only read during the call. */
int32_t kgpu_tree_create_from_archive(const void* bytes, uint64_t len,
                                      const kgpu_archive_format* fmt, void* stream,
                                      kgpu_tree** out);

/* Uploads a tree whose leaves use the FlatVec strategy (KdTree<A, u32, SS,
 * FlatVec<A, u32, K, 32>, K, 32>, src/leaf_strategy/flat_vec.rs:20-26): its
 * stems as in kgpu_tree_desc, its K point columns, items and (start, end)
 * leaf extents.  The leaves are re-encoded on the host in the VecOfArenas
 * tiles (same points, same order per leaf) and uploaded as kgpu_tree_create
 * does, so every query family runs on it unchanged. */
int32_t kgpu_tree_create_flatvec(const kgpu_flatvec_desc* desc, void* stream, kgpu_tree** out);
int32_t kgpu_tree_destroy(kgpu_tree* tree);
/* Builds the ImmutableKdTree of `n` points on the current device: `points` (n rows
 * of `dims` values of `dtype`) and `items` (NULL: item = source index) are DEVICE
 * pointers.  The resulting layout is byte-identical to kgpu_layout_build's (the
 * reference's soft construction, src/kd_tree/construction.rs:413-539, 868-968,
 * 1089-1175), built level by level on the GPU.  Synchronizes `stream` before
 * returning.  At most 2^31 - 1 points. */
int32_t kgpu_tree_build(int32_t dtype, uint32_t dims, const void* points, const uint32_t* items,
                        uint64_t n, void* stream, kgpu_tree** out);
/* Copies a device tree's layout to host arrays: stems (stem_count values), the
 * leaf arena (leaf_bytes_len bytes) and the extents as (byte offset, len) u64
 * pairs, leaf_count of them (sizes from kgpu_tree_info).  Any pointer may be NULL. */
int32_t kgpu_tree_read_layout(const kgpu_tree* tree, void* stems, uint8_t* leaf_bytes,
                              uint64_t* extents, void* stream);
/* info[0..7] = dtype, dims, size, leaf_count, max_stem_level, stem_count,
 *              leaf_bytes_len, device bytes held */
int32_t kgpu_tree_info(const kgpu_tree* tree, int64_t* info);

/* ---- iteration order and stored points -------------------------------------
 * The tree's entries in the reference's iteration order (KdTreeIter,
 * src/kd_tree/iter.rs:54-90; KdTree::iter, src/kd_tree/mod.rs:481): leaf 0 to
 * leaf_count - 1, each leaf's entries in stored order.  An entry's position
 * in that sequence is its rank.  Device pointers; the tree's device must be
 * current.
 * kgpu_tree_iter writes out_items[size] and out_points[size * dims] (values
 * of the tree's dtype) in rank order; either may be NULL.
 * kgpu_tree_project backs QueryBuilder::with_points
 * (src/kd_tree/query/builder.rs:1982-1987, 2175-2305): for each of n result
 * items it writes the entry's rank to out_ranks[n] and its stored point to
 * out_points[n * dims] (either may be NULL); an item not in the tree, such as
 * the 0xFFFFFFFF of an unused result slot, gives rank 0xFFFFFFFF and a zero
 * point.  An item must name one entry: KGPU_EUNSUPPORTED when two entries of
 * the tree share an item, or for trees of 2^32 - 1 entries or more.  The
 * first call for a tree builds its table (the points in rank order and the
 * items sorted: dims values of the dtype + 8 bytes per entry, held until
 * kgpu_tree_destroy) and synchronizes `stream`. */
int32_t kgpu_tree_iter(kgpu_tree* tree, uint32_t* out_items, void* out_points, void* stream);
int32_t kgpu_tree_project(kgpu_tree* tree, const uint32_t* items, uint64_t n, uint32_t* out_ranks,
                          void* out_points, void* stream);

/* ---- fixed-size families --------------------------------------------------
 * KGPU_NEAREST_ONE, KGPU_APPROX_NEAREST_ONE: out_dists/out_items hold nq
 * entries.  KGPU_NEAREST_N, KGPU_NEAREST_N_WITHIN, KGPU_BEST_N_WITHIN: they
 * hold nq * max_qty entries, row-major; out_counts[nq] (may be NULL) receives
 * the number of valid entries per query; unused slots hold +inf and
 * 0xFFFFFFFF.  A periodic box is accepted for the nearest families
 * (src/kd_tree/query/periodic.rs:156-214, :682-791).
 * Output order: nearest_n sorted by (distance, traversal arrival);
 * .unsorted() keeps arrival order while fewer than k were found (ThresholdVec
 * into_vec, results/result_collection.rs:136-215); best_n_within ascending
 * (item, arrival). */
int32_t kgpu_query(kgpu_tree* tree, const kgpu_query_desc* desc, const void* queries,
                   uint64_t nq, void* out_dists, uint32_t* out_items, uint32_t* out_counts,
                   void* stream);

/* ---- radius families (KGPU_WITHIN, KGPU_WITHIN_UNSORTED) ---------------
 * Two phases with caller-owned memory:
 *  1. kgpu_query_radius_count writes offsets[0..nq] (exclusive prefix of the
 *     per-query hit counts; offsets[nq] = total).
 *  2. kgpu_query_radius_fill writes total hits into out_dists/out_items at
 *     those offsets: sorted = stable by distance over traversal order
 *     (Vec::sort, results/result_collection.rs:1313-1316); unsorted =
 *     traversal order (within_unsorted.rs:133-157).
 * Both accept a periodic box. */
int32_t kgpu_query_radius_count(kgpu_tree* tree, const kgpu_query_desc* desc,
                                const void* queries, uint64_t nq, uint64_t* offsets,
                                void* stream);
int32_t kgpu_query_radius_fill(kgpu_tree* tree, const kgpu_query_desc* desc,
                               const void* queries, uint64_t nq, const uint64_t* offsets,
                               void* out_dists, uint32_t* out_items, void* stream);

/* ---- radius count without allocation -------------------------------------
 * No counterpart in the reference: an addition of this engine for callers that
 * cannot allocate device memory while they query (a process whose HBM is
 * reserved up front by its own pool, a latency-critical loop that must not
 * allocate, a host framework that owns every device buffer).
 * Same result as kgpu_query_radius_count, with device pointers only
 * (KGPU_FLAG_HOST_BUFFERS is rejected with KGPU_EINVAL).  It calls no
 * cudaMalloc, cudaMallocAsync, cudaFree or allocating library routine: the
 * prefix-sum scratch is a fixed 64 KiB array in device memory that every GPU
 * loading the library holds until exit.  Limit: nq <= 16,777,216 queries
 * (KGPU_EOVERFLOW beyond).  The tree's device must be current.  The first
 * call on each device looks up the array's device address
 * (cudaGetSymbolAddress), and so does the first call after cudaDeviceReset
 * has made the device's context anew; make that first call before any
 * stream capture.
 * All calls share the one array, so calls that overlap on the GPU (on
 * different streams or from different threads) race and must be serialised
 * by the caller. */
int32_t kgpu_query_radius_count_noalloc(kgpu_tree* tree, const kgpu_query_desc* desc,
                                        const void* queries, uint64_t nq, uint64_t* offsets,
                                        void* stream);

/* ---- traversal statistics ----------------------------------------------
 * Runs the query's traversal (for the radius families: the counting pass)
 * with counters and writes the totals over the batch to stats[0..2]:
 * stem visits, leaf visits, points scanned — the quantities of
 * src/test_utils/exact_query_stats.rs:23-60.  Outputs are discarded.
 * Synchronous; for sizing and for the algorithmic-bytes roofline model. */
int32_t kgpu_query_stats(kgpu_tree* tree, const kgpu_query_desc* desc, const void* queries,
                         uint64_t nq, uint64_t* stats, void* stream);

/* ---- batches over many trees --------------------------------------------
 * A forest groups uploaded trees of one dtype, dimensionality and stem order
 * (Eytzinger, or Donnelly of one block height; the trees must outlive it).  Forest queries take device pointers only: queries
 * [nq, dims], tree_of[nq] (index into the forest; a query naming no tree gets
 * empty results) and optionally radii[nq] (one radius per query, type A;
 * NULL = desc->radius).  One persistent launch answers the whole batch, its
 * warps pulling queries from a device work counter.  Output layouts are those
 * of the single-tree calls.  Replaces running the reference's per-tree
 * `.execute()` (or one GPU launch per tree) over a catalogue of trees. */
typedef struct kgpu_forest kgpu_forest;
int32_t kgpu_forest_create(kgpu_tree* const* trees, uint32_t n_trees, void* stream,
                           kgpu_forest** out);
int32_t kgpu_forest_destroy(kgpu_forest* forest);
int32_t kgpu_forest_query(kgpu_forest* forest, const kgpu_query_desc* desc, const void* queries,
                          const uint32_t* tree_of, const void* radii, uint64_t nq,
                          void* out_dists, uint32_t* out_items, uint32_t* out_counts,
                          void* stream);
int32_t kgpu_forest_query_radius_count(kgpu_forest* forest, const kgpu_query_desc* desc,
                                       const void* queries, const uint32_t* tree_of,
                                       const void* radii, uint64_t nq, uint64_t* offsets,
                                       void* stream);
/* Fills at most `capacity` hits (the caller sizes the output, for example from
 * a previous batch) and never reads the total back to the host, so the call
 * can be captured in a CUDA graph.  If a query's hits do not fit, *status
 * (device int32, zeroed by the caller; may be NULL) becomes KGPU_EOVERFLOW
 * and the caller retries with offsets[nq] as the capacity. */
int32_t kgpu_forest_query_radius_fill(kgpu_forest* forest, const kgpu_query_desc* desc,
                                      const void* queries, const uint32_t* tree_of,
                                      const void* radii, uint64_t nq, const uint64_t* offsets,
                                      uint64_t capacity, void* out_dists, uint32_t* out_items,
                                      int32_t* status, void* stream);

/* ---- Chamfer / ICP neighbour loss and its adjoint ------------------------
 * No counterpart in the reference (an addition built on the nearest_n path).
 * f32, 3-D, device pointers.  With the neighbours of each source point from a
 * nearest_n query (SquaredEuclidean) on the target tree:
 *   L = sum_i sum_{j < counts[i]} phi(d_ij),  phi(d) = d * exp(-d / (2 sigma^2)).
 * kgpu_chamfer_loss reduces phi over dists[n_src * k] in a fixed order into
 * *loss (device float); per_src (optional) receives each source's term.
 * kgpu_chamfer_backward writes grad_scale * dL/dsrc [n_src, 3] and
 * grad_scale * dL/dtgt [n_tgt, 3] (either may be NULL).  items[n_src * k] are
 * the neighbours' items = row numbers into tgt (new_from_slice); for batches
 * of cloud pairs, tree_of[i] names the pair of source i and tgt_base[pair]
 * the first row of that pair's targets in tgt.  Deterministic: fixed-order
 * sums and an integer counting sort, no floating-point atomics. */
int32_t kgpu_chamfer_loss(const float* dists, const uint32_t* counts, uint64_t n_src, uint32_t k,
                          double sigma, float* per_src, float* loss, void* stream);
int32_t kgpu_chamfer_backward(const float* src, uint64_t n_src, const float* tgt, uint64_t n_tgt,
                              const uint32_t* items, const uint32_t* counts, uint32_t k,
                              const uint32_t* tree_of, const uint64_t* tgt_base, double sigma,
                              float grad_scale, float* grad_src, float* grad_tgt, void* stream);

/* ---- CUDA graphs --------------------------------------------------------
 * Capture a sequence of device-pointer calls on `stream` (not the legacy
 * default stream) and replay it.  Capturable: kgpu_query, kgpu_query_radius_count,
 * the forest calls; not capturable: calls with KGPU_FLAG_HOST_BUFFERS and
 * kgpu_query_radius_fill (both read back to the host). */
typedef struct kgpu_graph kgpu_graph;
int32_t kgpu_graph_begin(void* stream);
int32_t kgpu_graph_end(void* stream, kgpu_graph** out);
int32_t kgpu_graph_launch(kgpu_graph* graph, void* stream);
int32_t kgpu_graph_destroy(kgpu_graph* graph);

/* ---- accounting --------------------------------------------------------
 * Number of CUDA kernels this library has launched in the process so far
 * (all threads).  Lets a caller count the launches inside a timed region. */
uint64_t kgpu_launch_count(void);

/* ---- scratch memory ----------------------------------------------------
 * No counterpart in the reference (its queries allocate on the host heap).
 * The entry points take their scratch (staging buffers, scan tiles, sort
 * buffers) from a stream-ordered memory pool of the library's own, one per
 * device, which keeps freed scratch cached between calls; the device's default
 * pool and other users of cudaMallocAsync are not touched.
 * kgpu_scratch_stats: out[0] bytes in use, out[1] the high-water mark of bytes
 * in use, out[2] bytes the pool holds from the driver, on `device` (zeros if
 * the library has not used that device).  kgpu_scratch_trim waits for the
 * device, returns every cached byte not in use to the driver and resets the
 * high-water mark to the bytes in use. */
int32_t kgpu_scratch_stats(int32_t device, uint64_t out[3]);
int32_t kgpu_scratch_trim(int32_t device);

#ifdef __cplusplus
}
#endif
#endif /* KIDDO_GPU_H */
