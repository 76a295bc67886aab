/*
 * quarry_b200.h -- C ABI of the B200 spatial-query engine.
 *
 * This is the boundary a foreign-function layer binds (ctypes, cffi, cgo, JNI).  Every entry
 * point takes plain device pointers, element counts, a caller-provided device workspace and
 * a CUDA stream passed as void* (NULL = legacy default stream), and returns a status code
 * (QK_OK = 0).  Nothing here allocates device memory: callers size buffers with the *_bytes
 * queries.  Launches are asynchronous on the given stream unless a comment says "syncs".
 * No entry point keeps global state, so independent trees may be used from several host
 * threads and streams at once.
 *
 * Data layouts follow quarry's API types (reference file:line):
 *   triangle  9 floats  a.xyz b.xyz c.xyz                  src/core/geometry.h:91-101
 *   point     3 floats                                     src/core/point_cloud.h:9-17
 *   gaussian 10 floats  mean.xyz quat.xyzw scale.xyz       src/core/gaussian.h:12-20
 *   ray       8 floats  origin.xyz dir.xyz tMin tMax       src/core/geometry.h:84-89
 *   node     32 bytes   mn.xyz mx.xyz left right           src/gpu/gpu_node.h:9-14
 *   wide    128 bytes   4 x {mn.xyz mx.xyz child pad}      src/gpu/gpu_node.h:46-57
 *   ray result    uint64 (hit << 32) | bits(t)             src/gpu/gpu_bvh.h:91-97
 *   query result  {uint32 dist2 bits, int32 id}, id -1 = none   src/gpu/gpu_bvh.h:250-253
 *   radius CSR    int32 offsets[n+1], uint64 keys (bits(d2) << 32 | id), each segment
 *                 ascending                                 src/gpu/gpu_bvh.h:296-301
 */
#ifndef QUARRY_B200_H
#define QUARRY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define QK_OK 0
#define QK_ERR_INVALID 1     /* bad argument; see qk_last_error() */
#define QK_ERR_CUDA 2        /* a CUDA call failed */
#define QK_ERR_WORKSPACE 3   /* workspace smaller than the matching *_bytes query */
#define QK_ERR_OVERFLOW 4    /* a traversal stack or a fixed table overflowed */
#define QK_ERR_DEPTH 5       /* tree deeper than the traversal stacks support: every traversal
                                entry point returns it, launching nothing, when tree->depth is
                                outside [0, 63] (trees from qk_build never are) */

/* ---- primitive kinds and builders ---- */
#define QK_TRI 0
#define QK_POINT 1
#define QK_GAUSS 2
#define QK_BUILD_LBVH 0
#define QK_BUILD_SAH 1
#define QK_BUILD_SAH4 2  /* leaf-size-4 binned SAH (the lever quarry names in docs/design.md:203,
                            207; no quarry counterpart): splits stop at ranges of at most 4
                            primitives, which are split by count (left half first) down to single
                            primitives, so the arrays keep the one-primitive-per-leaf format and
                            every entry point takes the tree; QK_TUNE_LEAF4 and
                            qk_wide_build_leaf4 then treat each such range as one leaf */

/* ---- query flags ---- */
#define QK_ORDER_MORTON 1u       /* QueryOrder::Morton / RayOrder::Morton (origin keys) */
#define QK_ORDER_DIRECTION 2u    /* RayOrder::MortonDirection (direction keys) */
#define QK_WIDE 4u               /* traverse the 4-wide nodes */
#define QK_ORDER_COHERENT 8u     /* engine order (no quarry counterpart): a counting sort on
                                    a Morton key of at most 15 bits over origin and direction
                                    (rays) or position (queries); same results as input order;
                                    batches under 64 keep input order */
/* tuning flags (same results, different schedules; chosen by the autotuner) */
#define QK_TUNE_DYNAMIC 256u     /* persistent warps fetching new rays as lanes finish */
#define QK_TUNE_HIGH_OCC 512u    /* register cap for 5 resident blocks of 256 per SM */
#define QK_TUNE_SHORT_STACK 2048u /* binary rays: top 8 stack entries per thread in shared memory */
#define QK_TUNE_LEAF4 4096u      /* binary nodes: child subtrees of 2..4 primitives are tested
                                    as leaves (skips their inner boxes) */
#define QK_TUNE_STASH 8192u     /* single-pass radius (binary nodes, one thread per query;
                                    batched plans on 4-wide nodes too; ignored with
                                    QK_TUNE_SPLIT): the count pass keeps every key it finds -- a
                                    query's first 16 in its stash, the rest in chained 32-key
                                    chunks of a pool of 128 keys per query in the workspace --
                                    and the fill pass copies them, traversing again only the
                                    queries the pool could not hold (pass the same workspace
                                    and flags to qk_radius_count and qk_radius_fill; a batched
                                    radius plan takes it as a plan flag) */
#define QK_TUNE_SPLIT 1024u      /* closest / kNN / radius on binary nodes: one warp per query,
                                    lanes on disjoint subtrees sharing the pruning bound */
#define QK_TUNE_SPLIT8 32768u    /* the same with 8 lanes per query (few queries fill more of the
                                    GPU); kNN takes at least the next group size >= k (k > 8:
                                    a warp) */
#define QK_TUNE_SPLIT4 65536u    /* the same with 4 lanes per query (kNN: at least k lanes) */
#define QK_TUNE_TAIL 16384u      /* closest / kNN on point clouds, binary nodes (thread or warp
                                    per query): a query still traversing after a step budget is
                                    answered by a brute-force scan over all points that every
                                    such query shares, merged per query; the call then reads the
                                    number of such queries back (syncs) and adds it to stats[3]
                                    (the workspace grows by 33.5 MB + 4 bytes per query; ignored
                                    for other kinds) */

/*
 * Device arrays of one tree.  The caller allocates every array (sizes from qk_tree_bytes)
 * and qk_build / qk_refit fill them.  Mirrors GpuBVH (src/gpu/gpu_bvh.h:26-77):
 *   nodes     2n-1 canonical 32-byte nodes (internal 0..n-2, leaf of slot s at n-1+s)
 *   items     n primitives in leaf order (the API's d_tris)
 *   prim_ids  n scene indices, prim_ids[slot]
 *   parent    2n-1 parent links, -1 at the root
 *   depth     2n-1 node depths (root 0)
 *   bnodes    n-1 traversal nodes of 64 bytes (both child boxes inline)
 *   leaves    n leaf payloads of 16*qk_leaf_vec4(kind) bytes
 *   slot_of   n: inverse of prim_ids (scene index -> slot), written by the build
 *   flags     n-1 ints of scratch for the bottom-up box pass
 *   wide      4-wide nodes (capacity n-1), filled by qk_wide_build; wide_id n-1 ints
 */
typedef struct qk_tree {
    int32_t kind;
    int32_t n;
    int32_t depth;       /* maximum node depth (set by qk_build) */
    int32_t wide_count;  /* set by qk_wide_build, 0 when absent */
    void* nodes;
    void* items;
    int32_t* prim_ids;
    int32_t* parent;
    int32_t* depth_arr;
    void* bnodes;
    void* leaves;
    int32_t* slot_of;
    int32_t* flags;
    void* wide;
    int32_t* wide_id;
    int32_t wide_leaf;   /* form of the 4-wide nodes, set by the wide builds: 1 from
                            qk_wide_build (every slot's pad is 0, as quarry writes it), 4 from
                            qk_wide_build_leaf4 (a leaf slot's pad holds its primitive count);
                            0 before either */
    int32_t reserved;
} qk_tree;

/* Byte sizes of the arrays of a tree with n primitives (same order as qk_tree). */
typedef struct qk_tree_sizes {
    size_t nodes, items, prim_ids, parent, depth_arr, bnodes, leaves, slot_of, flags, wide,
        wide_id;
} qk_tree_sizes;

/* ---- errors and device info ---- */
const char* qk_status_string(int status);
/* detail of the most recent failure on the calling host thread ("" if none) */
const char* qk_last_error(void);
/* gpuDescribe (src/gpu/gpu_bvh.h:100): writes "name sm_XY (N SM, G GiB)"; 0 when no device */
int qk_describe(char* buf, int len);

/* ---- sizes ---- */
int qk_stride_floats(int kind);  /* 9, 3, 10 */
int qk_leaf_vec4(int kind);      /* 3, 1, 3 */
int qk_tree_bytes(int kind, int n, qk_tree_sizes* out);
size_t qk_build_workspace_bytes(int kind, int n, int builder);
size_t qk_query_workspace_bytes(int count, unsigned flags);
size_t qk_radius_workspace_bytes(int count, unsigned flags);

/*
 * Build (buildBVHGPU / buildBVHSahGPU and the point / Gaussian variants,
 * src/gpu/gpu_bvh.h:103-118).  items: n primitives in scene order (device).  Syncs on the
 * stream to read the tree depth back into tree->depth.  sah_bins: SAH bin count (4..64),
 * ignored by LBVH.  n >= 2.
 */
int qk_build(qk_tree* tree, int builder, int sah_bins, const void* items, void* workspace,
             size_t workspace_bytes, void* stream);

/* Full refit (refitBVHGPU without dirty list, src/gpu/gpu_bvh.h:141): items in scene order,
 * same count; topology frozen; 4-wide nodes re-emitted when present. */
int qk_refit(qk_tree* tree, const void* items, void* workspace, size_t workspace_bytes,
             void* stream);

/* Partial refit (refitBVHGPU with dirty list, src/gpu/gpu_bvh.h:145-146): dirty_ids are scene
 * indices (device, count entries, each < n), dirty_items the new primitives for them (device,
 * same order).  Only the ancestors of the dirty leaves are merged. */
int qk_refit_dirty(qk_tree* tree, const int32_t* dirty_ids, const void* dirty_items, int count,
                   void* workspace, size_t workspace_bytes, void* stream);

/*
 * Topology edit (updateBVHGPU / updatePointBVHGPU / updateGaussianBVHGPU,
 * src/gpu/gpu_bvh.h:182-213; GpuTopoEdit semantics).  The new scene is the old one's
 * survivors in their order (old scene indices `deleted` removed), new primitives at the new
 * indices `inserted`, and `appended` more at its end; `moved` lists new indices whose geometry
 * changed.  All index arrays are device int32 arrays; deleted and inserted ascending and
 * unique; extra_items holds the n_inserted + appended new primitives (the inserted ones in
 * ascending index order, then the appended ones) and moved_items the n_moved moved ones.
 *
 * Only the small subtrees the edit touches are rebuilt (SAH over each); the rest is relinked
 * and renumbered.  new_tree: arrays for n_new = n_old - n_deleted + n_inserted + appended
 * primitives, of the same kind, none shared with old_tree; its wide layer is not built.
 * Query results on it equal those of a fresh build of the new scene.  Syncs.  When the plan
 * declines (the edit touches too much of the tree, a subtree would outgrow the forest
 * builder, or the root would change) info->rebuild is set, new_tree is left unwritten and the
 * caller rebuilds from the whole new scene.  cut_size: largest subtree a touched leaf may
 * rebuild (2..1024; 0 = n_old / (8 x edited primitives) clamped to 8..256, so the rebuilt
 * subtrees hold about an eighth of the tree).
 */
typedef struct qk_topo_edit {
    const int32_t* deleted;
    int n_deleted;
    const int32_t* inserted;
    int n_inserted;
    int appended;
    const int32_t* moved;
    int n_moved;
    const void* extra_items;
    const void* moved_items;
} qk_topo_edit;

typedef struct qk_topo_info {
    int rebuild;         /* 1: the plan declined; new_tree untouched */
    int cuts;            /* subtrees rebuilt */
    int old_leaves;      /* leaves under them before the edit */
    int new_leaves;      /* ... after it */
    int max_cut;         /* largest rebuilt subtree after the edit */
    int spliced;         /* internal nodes removed because one side became empty */
    int depth;           /* depth of the new tree */
    int reason;          /* why the plan declined: 1 the root is a subtree to rebuild, 2 the
                            root loses a side, 3 a subtree exceeds 1024 leaves, 4 more than a
                            quarter of the leaves, 5 depth */
} qk_topo_info;

size_t qk_update_workspace_bytes(int kind, int n_old, int n_new, int n_extra);
int qk_update_topology(const qk_tree* old_tree, qk_tree* new_tree, const qk_topo_edit* edit,
                       int cut_size, int sah_bins, qk_topo_info* info, void* workspace,
                       size_t workspace_bytes, void* stream);

/* 4-wide collapse (buildWideNodesGPU, src/gpu/gpu_bvh.h:229).  Syncs to read the count into
 * tree->wide_count.  With tree->wide == NULL the call only computes wide_id and the count, so
 * the caller can allocate wide_count * 128 bytes and call again to emit the nodes. */
int qk_wide_build(qk_tree* tree, void* workspace, size_t workspace_bytes, void* stream);

/* 4-wide nodes with leaf-size-4 slots (no quarry counterpart; the 4-wide half of the lever in
 * quarry's docs/design.md:203, 207): as qk_wide_build, but a child or grandchild subtree of 2..4
 * primitives on contiguous leaf slots (every such range of a QK_BUILD_SAH4 tree) takes one slot
 * as a leaf range -- child = -(first slot + 1), pad = its primitive count; single leaves have
 * pad = 1 -- so fewer wide nodes cover the tree and no node level below a range is fetched.
 * Same two-call pattern; sets tree->wide_leaf = 4.  Every QK_WIDE traversal of the tree reads
 * the form tree->wide_leaf records, with the same results as any other layout; refits re-emit
 * the form. */
int qk_wide_build_leaf4(qk_tree* tree, void* workspace, size_t workspace_bytes, void* stream);

/*
 * First-hit rays (raycastGPU, src/gpu/gpu_bvh.h:233-234).  rays: count rays (device);
 * out: count uint64 results.  flags: QK_ORDER_* and QK_WIDE.  stats (nullable, device, 4
 * uint64, accumulated): node tests, triangle tests, stack overflows, 0.
 */
int qk_raycast(const qk_tree* tree, const void* rays, int count, uint64_t* out, unsigned flags,
               uint64_t* stats, void* workspace, size_t workspace_bytes, void* stream);

/* First-hit rays from host memory (the whole raycastGPU round trip, src/gpu/gpu_bvh.h:217-237):
 * rays are uploaded, traced and read back in `chunks` pieces: the uploads on upload_stream,
 * the traversals alternating between trace_stream0 and trace_stream1 (a traversal can start
 * while the one before drains), the read-backs on readback_stream, so the upload of one
 * piece overlaps the traversal of the one before and the read-back of the one before that.
 * host_rays / host_out should be pinned (page-locked) for the copies to be asynchronous;
 * dev_rays (count rays) and dev_out (count results) are device buffers.  dev_out may be
 * NULL when host_out is mapped page-locked memory: the traversals then store the results
 * straight into host_out and no read-back copies run (readback_stream still waits for every
 * traversal).  The workspace holds two chunk workspaces.  Results equal qk_raycast's.  Every read-back waits for its
 * traversal and follows the earlier read-backs, and every traversal waits for its upload,
 * so synchronising readback_stream covers all the work before host_out is read.  The
 * streams may coincide (the pieces then run one after another). */
size_t qk_raycast_host_workspace_bytes(int count, int chunks);
int qk_raycast_host(const qk_tree* tree, const void* host_rays, int count, uint64_t* host_out,
                    void* dev_rays, uint64_t* dev_out, int chunks, unsigned flags, void* workspace,
                    size_t workspace_bytes, void* upload_stream, void* trace_stream0,
                    void* trace_stream1, void* readback_stream);

/* First-hit rays read from and written to page-locked host memory by the traversal kernel
 * itself (zero-copy; the rest of the raycastGPU round trip, src/gpu/gpu_bvh.h:217-237): each
 * ray crosses the host link once, as the thread that traces it loads it, and each result
 * once, as it is stored, so transfers and traversal overlap inside one launch.  host_rays
 * and host_out must be page-locked memory mapped into the device's address space (pinned
 * allocations under unified addressing are); anything else returns QK_ERR_INVALID before
 * any launch.  Flags and workspace as qk_raycast; an order flag makes the key pass read the
 * rays over the link too.  Results equal qk_raycast's once the stream is synchronised. */
int qk_raycast_mapped(const qk_tree* tree, const void* host_rays, int count, uint64_t* host_out,
                      unsigned flags, void* workspace, size_t workspace_bytes, void* stream);

/* Closest primitive per query point (closestPointGPU / closestVertexGPU /
 * closestGaussianGPU, src/gpu/gpu_bvh.h:283-330).  points: count x 3 floats; out: count
 * query results. */
int qk_closest(const qk_tree* tree, const float* points, int count, void* out, unsigned flags,
               uint64_t* stats, void* workspace, size_t workspace_bytes, void* stream);

/* k nearest (kNearestGPU and variants, src/gpu/gpu_bvh.h:289-333): 1 <= k <= 32,
 * stride >= k results per query, ascending by (dist2, id), missing slots id -1, dist2 0. */
int qk_knn(const qk_tree* tree, const float* points, int count, int k, int stride, void* out,
           unsigned flags, uint64_t* stats, void* workspace, size_t workspace_bytes,
           void* stream);

/*
 * Radius query as CSR (radiusQueryGPU and variants, src/gpu/gpu_bvh.h:307-336), in two
 * calls.  qk_radius_count writes counts and offsets[count+1] (offsets[count] = total) and
 * copies the total to *total_host (syncs).  The caller then allocates keys[total] and calls
 * qk_radius_fill with the same points, radius and flags, which writes every segment sorted
 * by (dist2, id).  radius >= 0.
 */
int qk_radius_count(const qk_tree* tree, const float* points, int count, float radius,
                    int32_t* offsets, int64_t* total_host, unsigned flags, uint64_t* stats,
                    void* workspace, size_t workspace_bytes, void* stream);
int qk_radius_fill(const qk_tree* tree, const float* points, int count, float radius,
                   const int32_t* offsets, uint64_t* keys, unsigned flags, void* workspace,
                   size_t workspace_bytes, void* stream);

/*
 * Structural check (validateBVHGPU and variants, src/gpu/gpu_bvh.h:347-349).  items: the
 * scene-order primitives the tree should hold (device).  errors: 8 device ints, zeroed by
 * the call, then [0] bad children or box, [1] bad leaf box, [2] bad reference count, [3] bad
 * leaf id, [4] bad primitive map, [5] bad depth, [6] 4-wide node mismatch.
 */
int qk_validate(const qk_tree* tree, const void* items, int32_t* errors, void* workspace,
                size_t workspace_bytes, void* stream);
size_t qk_validate_workspace_bytes(int n);

/* ---- differentiable queries (no counterpart in quarry, which has no backward pass) ---- */

/* First-hit rays that also report the hit primitive: ids[count] = scene index (-1 on a
 * miss); among primitives at the same t the smallest index.  The t results equal
 * qk_raycast's bit for bit. */
int qk_raycast_ids(const qk_tree* tree, const void* rays, int count, uint64_t* out, int32_t* ids,
                   unsigned flags, void* workspace, size_t workspace_bytes, void* stream);

size_t qk_grad_workspace_bytes(int count, int channels);

/* Adjoint of d_i = |p_i - closest point of the selected primitive| (distance, not squared)
 * for the selected primitive of qk_closest's results, recomputed in FP64.  grad_dist: count
 * weights dL/dd_i (NULL = all ones).  Writes grad_points (count x 3) and grad_items (n x
 * stride, scene order; summed over queries in query order, deterministic).  d = 0 (inside an
 * ellipsoid, on a triangle) contributes 0. */
int qk_distance_grad(const qk_tree* tree, const void* items, const float* points,
                     const void* results, const float* grad_dist, int count, float* grad_points,
                     float* grad_items, void* workspace, size_t workspace_bytes, void* stream);

/* Adjoint of the first-hit t of the rays with respect to the hit triangles (grad_tris, n x 9,
 * scene order, deterministic sums) and, when grad_rays is not NULL, the rays' origins and
 * directions (count x 6).  ids from qk_raycast_ids; grad_t: dL/dt_i (NULL = all ones). */
int qk_ray_t_grad(const qk_tree* tree, const void* items, const void* rays, const int32_t* ids,
                  const float* grad_t, int count, float* grad_tris, float* grad_rays,
                  void* workspace, size_t workspace_bytes, void* stream);

/* Vertex form of qk_ray_t_grad and qk_distance_grad (triangle trees), for meshes given as
 * shared vertices and corner indices: indices holds the n x 3 vertex ids of the tree's
 * triangles in scene order.  The per-query FP64 terms are summed straight into grad_verts
 * (nverts x 3) in FP64 and rounded to FP32 once, in a fixed order (deterministic), so a vertex
 * whose terms cancel keeps its precision; the per-triangle path rounds each triangle's sum
 * first.  grad_rays / grad_points as in the per-triangle calls. */
size_t qk_grad_vertices_workspace_bytes(int count);
int qk_ray_t_grad_vertices(const qk_tree* tree, const void* items, const void* rays,
                           const int32_t* ids, const float* grad_t, int count,
                           const int32_t* indices, int nverts, float* grad_verts,
                           float* grad_rays, void* workspace, size_t workspace_bytes,
                           void* stream);
int qk_distance_grad_vertices(const qk_tree* tree, const void* items, const float* points,
                              const void* results, const float* grad_dist, int count,
                              const int32_t* indices, int nverts, float* grad_points,
                              float* grad_verts, void* workspace, size_t workspace_bytes,
                              void* stream);

/* Deterministic segmented sum: out[k, c] = sum over i in increasing order with keys[i] == k of
 * values[i, c] (FP64 accumulation); keys < 0 are skipped.  1 <= channels <= 10. */
int qk_segment_sum(const int32_t* keys, const float* values, int count, int channels, int segments,
                   float* out, void* workspace, size_t workspace_bytes, void* stream);

/* Allocation-free first-hit rays (no counterpart in quarry).  For callers that cannot
 * allocate device memory when they trace (a host that reserves all device memory up front and
 * forbids later allocations, or code without an allocator): same results as qk_raycast with
 * the same flags, but the Morton-order scratch lives in a fixed array inside this library
 * (4.5 MB per GPU that loads it, held until exit), so no workspace is passed.  At most
 * 262,144 rays per call; larger counts return QK_ERR_INVALID.  The array's address belongs to
 * the current CUDA context, so every call looks it up (a host-side query that allocates
 * nothing); the first call on a device may load the library's device code, so make it before
 * any stream capture.  Calls share the array: calls that overlap on the GPU race. */
int qk_raycast_noalloc(const qk_tree* tree, const void* rays, int count, uint64_t* out,
                       unsigned flags, void* stream);

/* Stable LSD radix sort of 32-bit keys with 32-bit values over the low `bits` bits.  All
 * four buffers hold n entries; the sorted result ends in keys_out / vals_out. */
size_t qk_sort_workspace_bytes(int n);
int qk_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                  uint32_t* vals_out, int n, int bits, void* workspace, size_t workspace_bytes,
                  void* stream);

/*
 * ---- Batched scenes (new; quarry has no batched API) ----
 * A batch holds `scenes` trees of ONE primitive kind whose inputs are concatenated in one
 * device array (scene s starts at item counts[0] + ... + counts[s-1]).  Every tree lives in
 * a caller-allocated arena and is an ordinary qk_tree (qk_batch_tree), so every single-tree
 * call above works on it too.  Under the batched schedule each phase of the build and of a
 * query is ONE launch over all scenes; queries run persistent warps that take 32-query chunks
 * of any scene from a shared counter (work stealing).  qk_batch_build and qk_batch_query
 * with schedule QK_SCHEDULE_BATCHED only enqueue kernels and memsets, so a whole build +
 * query sequence can be captured in one CUDA graph; qk_batch_create, qk_batch_sync,
 * qk_batch_plan_create and qk_batch_plan_status synchronize.  QK_SCHEDULE_LOOP runs the same
 * work as a per-scene loop over the single-tree calls (qk_build, qk_raycast, ...), with their
 * per-scene synchronizations: the comparison schedule.  Results are bit-identical between
 * the two schedules and to the single-tree calls.
 */
typedef struct qk_batch qk_batch;            /* opaque host object */
typedef struct qk_batch_plan qk_batch_plan;  /* opaque host object */

#define QK_SCHEDULE_BATCHED 0u
#define QK_SCHEDULE_LOOP 1u

#define QK_OP_RAY 0
#define QK_OP_CLOSEST 1
#define QK_OP_KNN 2
#define QK_OP_RADIUS 3

/* Launch shape of the persistent query kernels (chosen by the autotuner). */
typedef struct qk_batch_tune {
    int32_t block;          /* threads per block: 64, 128 or 256 */
    int32_t blocks_per_sm;  /* persistent grid = SMs x blocks_per_sm (1..16) */
    int32_t short_stack;    /* stack entries per thread held in shared memory (0..32) */
    int32_t chunks_per_fetch; /* 32-query chunks a warp takes per counter fetch (1..64) */
    int32_t split;          /* 1: closest / kNN / radius with one warp per query (binary
                               nodes; see QK_TUNE_SPLIT); 0: one thread per query */
} qk_batch_tune;

/* flags: QK_WIDE reserves and builds the 4-wide nodes of every scene. */
size_t qk_batch_arena_bytes(int kind, const int32_t* counts, int scenes, unsigned flags);
int qk_batch_create(qk_batch** out, int kind, const int32_t* counts, int scenes,
                    const void* items, void* arena, size_t arena_bytes, unsigned flags,
                    void* stream);
/* Builds every scene's LBVH (and 4-wide nodes when created with QK_WIDE). */
int qk_batch_build(qk_batch* batch, unsigned schedule, void* stream);
/* Builds every scene with the binned SAH builder (sah_bins 4..64), scene after scene: the
 * SAH level loop reads counts back, so this call synchronizes and cannot be captured.  The
 * trees stay in the arena and serve every batched query like the LBVH ones. */
int qk_batch_build_sah(qk_batch* batch, int sah_bins, void* stream);
/* Waits for the stream, reads every scene's depth / wide-node count back into its tree and
 * reports QK_ERR_DEPTH when a scene is too deep for the traversal stack. */
int qk_batch_sync(qk_batch* batch, void* stream);
int qk_batch_tree(const qk_batch* batch, int scene, qk_tree* out);
int qk_batch_scenes(const qk_batch* batch);
void qk_batch_destroy(qk_batch* batch);

/* A query plan: per-scene query counts of one operation (concatenated by scene in the
 * inputs and outputs) and, for QK_OP_RADIUS, the per-scene radius (host floats).
 * flags: QK_ORDER_MORTON (scene-major Morton order of the inputs, within each scene's
 * bounds), QK_WIDE (traverse the 4-wide nodes) and, for QK_OP_RADIUS, QK_TUNE_STASH (the
 * single-pass radius; the plan then holds its stash and a key pool of 512 keys per query on
 * average, about 4.3 KB per query). */
size_t qk_batch_plan_bytes(const qk_batch* batch, int op, const int32_t* counts,
                           unsigned flags);
int qk_batch_plan_create(qk_batch_plan** out, const qk_batch* batch, int op,
                         const int32_t* counts, const float* params, void* mem, size_t bytes,
                         unsigned flags, void* stream);
typedef struct qk_batch_io {
    const void* input;  /* rays (8 floats) or points (3 floats), device, concatenated by scene */
    void* out;          /* RAY: uint64 per ray (qk_raycast layout); CLOSEST: 8 B per point;
                           KNN: k x 8 B per point; RADIUS: uint64 keys, `capacity` entries */
    int32_t* offsets;   /* RADIUS: CSR offsets into out, queries + scenes + 1 entries; batched
                           schedule: one global CSR in the first queries + 1; loop schedule:
                           scene s's own CSR (from 0) at offsets[q_begin(s) + s], its keys at
                           out + (sum of earlier scenes' totals) */
    int64_t capacity;   /* RADIUS: keys that fit in out */
    int32_t k;          /* KNN: 1..32 */
    int32_t pad;
} qk_batch_io;
int qk_batch_query(qk_batch_plan* plan, const qk_batch_io* io, const qk_batch_tune* tune,
                   unsigned schedule, void* stream);
/* Waits for the stream; radius_total: keys of the last radius query (-1 otherwise);
 * overflows: traversals stopped by a stack or iteration limit.  QK_ERR_WORKSPACE when the
 * radius keys exceeded the capacity (nothing was written past it). */
int qk_batch_plan_status(qk_batch_plan* plan, int64_t* radius_total, int64_t* overflows,
                         void* stream);
void qk_batch_plan_destroy(qk_batch_plan* plan);

#ifdef __cplusplus
}
#endif

#endif
