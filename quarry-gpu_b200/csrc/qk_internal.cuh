// qk_internal.cuh -- shared host/device plumbing of the engine: workspace carving, error
// reporting, ordered-float atomics, and the launchers the C ABI (qk_capi.cu) calls.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/quarry_b200.h"
#include "qk_device.cuh"

namespace qk {

constexpr int kBlock = 256;
constexpr int kStack = 64;       // binary traversal stack (LBVH depth <= 63, SAH depth capped)
constexpr int kStackWide = 128;  // 4-wide traversal stack (up to 3 far entries per level)
constexpr int kMaxKnn = 32;
constexpr int kSortTile = 4096;  // keys per radix-sort tile (256 threads x 16)
constexpr int kScanBlock = 1024; // elements per scan block (256 threads x 4)

inline int blocks_for(long long n, int per = kBlock) {
    return static_cast<int>((n + per - 1) / per);
}

// Thread-local error detail behind qk_last_error().
void set_error(const char* fmt, ...);
int fail(int status, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);

// Per-stage device timing behind the C++ API's timing structs (GpuBuildTimings,
// GpuRefitTimings, GpuTopoUpdateTimings).  A host thread installs a StageClock for the
// duration of one call; the builders, refits and topology edits then record an event on their
// stream at each stage boundary (stage_mark), and the SAH builder adds its per-level binning,
// split and partition times.  With no clock installed (every C-ABI call) nothing is recorded.
enum StageMark {
    kMarkStart,     // call begins
    kMarkMorton,    // LBVH: centroid bounds + Morton codes done
    kMarkSort,      // LBVH: radix sort done
    kMarkPlan,      // topology edit: cut plan chosen (host synchronisation)
    kMarkRelayout,  // topology edit: kept nodes renumbered, kept leaves and new items staged
    kMarkTopo,      // links done (LBVH emit, SAH levels + lower tiers, edit forests)
    kMarkScatter,   // leaves written (SAH leaf scatter; refit leaf gather / dirty marking)
    kMarkBoxes,     // bottom-up boxes (or the refit merge) done
    kMarkEnd,       // depths read back / wide nodes re-emitted: call done
    kMarkCount
};
struct StageClock {
    cudaEvent_t ev[kMarkCount] = {};
    bool hit[kMarkCount] = {};
    cudaEvent_t lv[4] = {};  // SAH global-tier level: start, binned, split, partitioned
    double sah_bin = 0.0, sah_split = 0.0, sah_part = 0.0;
};
// the calling host thread's installed clock (nullptr when none)
StageClock*& stage_clock();
inline void stage_mark(int m, cudaStream_t s) {
    StageClock* c = stage_clock();
    if (c != nullptr && cudaEventRecord(c->ev[m], s) == cudaSuccess) c->hit[m] = true;
}

// Carves aligned sub-buffers out of one workspace.  With base == nullptr it only measures.
struct Carve {
    char* base = nullptr;
    size_t used = 0;
    template <typename T>
    T* take(size_t count, size_t align = 256) {
        used = (used + align - 1) / align * align;
        T* p = base ? reinterpret_cast<T*>(base + used) : nullptr;
        used += count * sizeof(T);
        return p;
    }
};

// Arrival counter of the bottom-up passes: one acquire-release add at device scope.  The
// release half publishes the arriving thread's earlier writes (its child's box) before the
// count changes; the acquire half makes the other arrivals' writes visible to the thread that
// goes on to merge the node.  Replaces a full fence on each side of a relaxed atomicAdd.
__device__ __forceinline__ int arrive_add(int* counter, int v) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;"
                 : "=r"(old)
                 : "l"(counter), "r"(v)
                 : "memory");
    return old;
}

// IEEE-754 bits mapped to a monotone unsigned order, for atomicMin / atomicMax on floats.
__device__ __forceinline__ unsigned ord_f(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unord_f(unsigned u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Per-call header at the start of every workspace: centroid / query bounds as ordered uints,
// the maximum depth, a counter and the overflow / error words.
struct Header {
    unsigned lo[3];
    unsigned hi[3];
    int max_depth;
    int counter;
    int overflow;
    int error;
    int list_count[2];
    int pad[4];
};

// ---- sort / scan (qk_sort.cu) ----
size_t sort_ws_bytes(int n);
cudaError_t sort_pairs(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout,
                       int n, int bits, void* ws, cudaStream_t s);
size_t scan_ws_bytes(int n);
// exclusive scan of n ints; writes the total to out[n] when write_total is set
cudaError_t scan_exclusive(const int* in, int* out, int n, bool write_total, void* ws,
                           cudaStream_t s);

// ---- build / refit / wide / validate (qk_build.cu) ----
size_t build_ws_bytes(int kind, int n, int builder);
// the bottom-up pass's range scratch inside a build workspace
int2* build_ranges(void* ws, int kind, int n, int builder);
int build_tree(qk_tree* t, int builder, int bins, const void* items, void* ws, size_t ws_bytes,
               cudaStream_t s);
// SAH topology (qk_sah.cu): fills links, parents, order-derived leaves; boxes come after
size_t sah_ws_bytes(int n);
int build_sah(qk_tree* t, int bins, int leaf_size, const void* items, void* ws, cudaStream_t s);
// Forest of independent ranges for the SAH builder's lower tiers (qk_sah.cu): task i =
// {begin, end, node, depth} over positions of `order` (indices into cen / plo / phi), its
// internal nodes below `node` numbered from id_base[i]; node < 0 skips the task.  Leaf of
// position p is n-1+p of t; tmp: partition scratch like `order`.  Ranges of 2..1024
// primitives, at most max_count: those of up to 256 take one warp each, larger ones a block.
int sah_forest(const int4* tasks, int ntask, int max_count, const int* id_base, int* order,
               int* tmp, const float4* cen, const float4* plo, const float4* phi, qk_tree* t,
               int bins, int* err, cudaStream_t s);
// boxes, traversal nodes and depths of a tree whose links and leaves are set (syncs)
int finish_tree_boxes(qk_tree* t, Header* h, int2* ranges, cudaStream_t s);
// topology edits (qk_topo.cu)
size_t update_ws_bytes(int kind, int n_old, int n_new, int n_extra);
int update_topology(const qk_tree* old_t, qk_tree* new_t, const qk_topo_edit* edit, int cut_size,
                    int bins, qk_topo_info* info, void* ws, cudaStream_t s);
int refit_tree(qk_tree* t, const void* items, cudaStream_t s);
int refit_tree_dirty(qk_tree* t, const int* ids, const void* items, int count, void* ws,
                     cudaStream_t s);
int wide_build(qk_tree* t, int leaf, void* ws, size_t ws_bytes, cudaStream_t s);
int wide_emit_all(qk_tree* t, cudaStream_t s);
size_t validate_ws_bytes(int n);
int validate_tree(const qk_tree* t, const void* items, int* errors, void* ws, cudaStream_t s);

// ---- traversal (qk_query.cu) ----
size_t order_ws_bytes(int count);
// closest / kNN workspace: the order buffers plus, with QK_TUNE_TAIL, the heavy-query tail's
size_t point_query_ws_bytes(int count, unsigned flags);
int ray_query(const qk_tree* t, const void* rays, int count, uint64_t* out, int* ids,
              unsigned flags, uint64_t* stats, void* ws, cudaStream_t s);
int closest_query(const qk_tree* t, const float* pts, int count, void* out, unsigned flags,
                  uint64_t* stats, void* ws, cudaStream_t s);
int knn_query(const qk_tree* t, const float* pts, int count, int k, int stride, void* out,
              unsigned flags, uint64_t* stats, void* ws, cudaStream_t s);
size_t radius_ws_bytes(int count, unsigned flags);
int radius_count(const qk_tree* t, const float* pts, int count, float r, int* offsets,
                 long long* total, unsigned flags, uint64_t* stats, void* ws, cudaStream_t s);
int radius_fill(const qk_tree* t, const float* pts, int count, float r, const int* offsets,
                uint64_t* keys, unsigned flags, void* ws, cudaStream_t s);
// sorts every CSR segment [offsets[q], offsets[q+1]) of keys ascending; medium / large hold
// count ints each; cap >= 0 skips the sort when offsets[count] > cap
int radius_sort_segments(const int* offsets, int count, uint64_t* keys, int* medium, int* large,
                         Header* h, long long cap, cudaStream_t s);

// ---- adjoints (qk_grad.cu) ----
size_t grad_ws_bytes(int count, int channels);
int closest_distance_grad(int kind, int n, const void* items, const float* pts, const void* res,
                          const float* gw, int count, float* gpts, float* gitems, void* ws,
                          cudaStream_t s);
int ray_t_grad(int n, const void* tris, const void* rays, const int* ids, const float* gw,
               int count, float* gtris, float* grays, void* ws, cudaStream_t s);
int segment_sum(const int* keys, const float* vals, int count, int channels, int nseg, float* out,
                void* ws, cudaStream_t s);
size_t grad_vertices_ws_bytes(int count);
int ray_t_grad_vertices(int n, const void* tris, const void* rays, const int* ids, const float* gw,
                        int count, const int* indices, int nverts, float* gverts, float* grays,
                        void* ws, cudaStream_t s);
int distance_grad_vertices(int n, const void* tris, const float* pts, const void* res,
                           const float* gw, int count, const int* indices, int nverts,
                           float* gpts, float* gverts, void* ws, cudaStream_t s);

}  // namespace qk
