// qk_capi.cu -- extern "C" entry points (include/quarry_b200.h): argument checks, workspace
// size checks and dispatch to the launchers.  Errors are reported as status codes with a
// thread-local message; nothing here allocates device memory or keeps global state.
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "qk_internal.cuh"

namespace qk {

namespace {
thread_local char g_error[512] = "";
}

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

int fail(int status, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
    return status;
}

int cuda_status(cudaError_t e, const char* what) {
    std::snprintf(g_error, sizeof(g_error), "CUDA %s: %s", what, cudaGetErrorString(e));
    return QK_ERR_CUDA;
}

StageClock*& stage_clock() {
    static thread_local StageClock* clock = nullptr;
    return clock;
}

}  // namespace qk

using namespace qk;

namespace {

int check_tree(const qk_tree* t, bool need_bnodes = true) {
    if (!t) return fail(QK_ERR_INVALID, "tree is NULL");
    if (t->kind < 0 || t->kind > 2) return fail(QK_ERR_INVALID, "unknown primitive kind %d", t->kind);
    if (t->n < 2) return fail(QK_ERR_INVALID, "at least 2 primitives are required (n=%d)", t->n);
    if (!t->nodes || !t->items || !t->prim_ids || !t->parent || !t->depth_arr || !t->leaves ||
        !t->slot_of || !t->flags || (need_bnodes && !t->bnodes))
        return fail(QK_ERR_INVALID, "tree has a NULL device array");
    return QK_OK;
}

int check_ws(void* ws, size_t have, size_t need) {
    if (need > 0 && (ws == nullptr || have < need))
        return fail(QK_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu required",
                    have, need);
    return QK_OK;
}

// Every traversal entry point: the tree's recorded depth must fit the traversal stacks (a
// tree from qk_build / qk_update_topology always does; one assembled by the caller may not),
// so nothing is launched on a tree the stacks cannot hold.
int check_wide(const qk_tree* t, unsigned flags) {
    if (t->depth < 0 || t->depth >= kStack)
        return fail(QK_ERR_DEPTH, "tree depth %d exceeds the traversal stack (%d levels)",
                    t->depth, kStack - 1);
    if ((flags & QK_WIDE) && (t->wide == nullptr || t->wide_count <= 0))
        return fail(QK_ERR_INVALID, "wide nodes not built");
    if (__builtin_popcount(flags & (QK_ORDER_MORTON | QK_ORDER_DIRECTION | QK_ORDER_COHERENT)) > 1)
        return fail(QK_ERR_INVALID,
                    "choose one of QK_ORDER_MORTON, QK_ORDER_DIRECTION and QK_ORDER_COHERENT");
    return QK_OK;
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace

extern "C" {

const char* qk_status_string(int status) {
    switch (status) {
        case QK_OK: return "ok";
        case QK_ERR_INVALID: return "invalid argument";
        case QK_ERR_CUDA: return "CUDA error";
        case QK_ERR_WORKSPACE: return "workspace too small";
        case QK_ERR_OVERFLOW: return "traversal stack overflow";
        case QK_ERR_DEPTH: return "tree too deep";
        default: return "unknown status";
    }
}

const char* qk_last_error(void) { return g_error; }

int qk_describe(char* buf, int len) {
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
        if (buf && len > 0) buf[0] = '\0';
        cudaGetLastError();
        return 0;
    }
    cudaDeviceProp prop{};
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return 0;
    if (buf && len > 0) {
        std::snprintf(buf, static_cast<size_t>(len), "%s sm_%d%d (%d SM, %.1f GiB)", prop.name,
                      prop.major, prop.minor, prop.multiProcessorCount,
                      static_cast<double>(prop.totalGlobalMem) / (1024.0 * 1024.0 * 1024.0));
    }
    return 1;
}

int qk_stride_floats(int kind) { return kind == 0 ? 9 : kind == 1 ? 3 : kind == 2 ? 10 : 0; }
int qk_leaf_vec4(int kind) { return kind == 0 ? 3 : kind == 1 ? 1 : kind == 2 ? 3 : 0; }

int qk_tree_bytes(int kind, int n, qk_tree_sizes* out) {
    if (!out) return fail(QK_ERR_INVALID, "sizes pointer is NULL");
    if (kind < 0 || kind > 2) return fail(QK_ERR_INVALID, "unknown primitive kind %d", kind);
    if (n < 2) return fail(QK_ERR_INVALID, "at least 2 primitives are required (n=%d)", n);
    const size_t nn = static_cast<size_t>(n);
    out->nodes = (2 * nn - 1) * sizeof(Node);
    out->items = nn * qk_stride_floats(kind) * sizeof(float);
    out->prim_ids = nn * sizeof(int32_t);
    out->parent = (2 * nn - 1) * sizeof(int32_t);
    out->depth_arr = (2 * nn - 1) * sizeof(int32_t);
    out->bnodes = (nn - 1) * sizeof(BNode);
    out->leaves = nn * qk_leaf_vec4(kind) * 16;
    out->slot_of = nn * sizeof(int32_t);
    out->flags = (nn - 1) * sizeof(int32_t);
    out->wide = (nn - 1) * sizeof(WideNode);
    out->wide_id = (nn - 1) * sizeof(int32_t);
    return QK_OK;
}

size_t qk_build_workspace_bytes(int kind, int n, int builder) {
    if (n < 2) return 0;
    return build_ws_bytes(kind, n, builder);
}

size_t qk_query_workspace_bytes(int count, unsigned flags) {
    return count > 0 ? point_query_ws_bytes(count, flags) : 0;
}

size_t qk_radius_workspace_bytes(int count, unsigned flags) {
    return count > 0 ? radius_ws_bytes(count, flags) : 0;
}

int qk_build(qk_tree* tree, int builder, int sah_bins, const void* items, void* workspace,
             size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (!items) return fail(QK_ERR_INVALID, "items is NULL");
    if (builder != QK_BUILD_LBVH && builder != QK_BUILD_SAH && builder != QK_BUILD_SAH4)
        return fail(QK_ERR_INVALID, "builder must be QK_BUILD_LBVH, QK_BUILD_SAH or QK_BUILD_SAH4");
    if (builder != QK_BUILD_LBVH && (sah_bins < 4 || sah_bins > 64))
        return fail(QK_ERR_INVALID, "sah_bins must be in [4, 64]");
    st = check_ws(workspace, workspace_bytes, build_ws_bytes(tree->kind, tree->n, builder));
    if (st) return st;
    return build_tree(tree, builder, sah_bins, items, workspace, workspace_bytes, as_stream(stream));
}

int qk_refit(qk_tree* tree, const void* items, void* workspace, size_t workspace_bytes,
             void* stream) {
    (void)workspace;
    (void)workspace_bytes;
    int st = check_tree(tree);
    if (st) return st;
    if (!items) return fail(QK_ERR_INVALID, "items is NULL");
    return refit_tree(tree, items, as_stream(stream));
}

int qk_refit_dirty(qk_tree* tree, const int32_t* dirty_ids, const void* dirty_items, int count,
                   void* workspace, size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (count < 0) return fail(QK_ERR_INVALID, "negative dirty count");
    if (count == 0) return QK_OK;
    if (!dirty_ids || !dirty_items) return fail(QK_ERR_INVALID, "dirty arrays are NULL");
    st = check_ws(workspace, workspace_bytes, build_ws_bytes(tree->kind, tree->n, 0));
    if (st) return st;
    if (count > tree->n) return fail(QK_ERR_INVALID, "more dirty entries than primitives");
    return refit_tree_dirty(tree, dirty_ids, dirty_items, count, workspace, as_stream(stream));
}

size_t qk_update_workspace_bytes(int kind, int n_old, int n_new, int n_extra) {
    if (kind < 0 || kind > 2 || n_old < 2 || n_new < 2 || n_extra < 0) return 0;
    return update_ws_bytes(kind, n_old, n_new, n_extra);
}

int qk_update_topology(const qk_tree* old_tree, qk_tree* new_tree, const qk_topo_edit* edit,
                       int cut_size, int sah_bins, qk_topo_info* info, void* workspace,
                       size_t workspace_bytes, void* stream) {
    int st = check_tree(old_tree);
    if (st) return st;
    if ((st = check_tree(new_tree))) return st;
    if (!edit || !info) return fail(QK_ERR_INVALID, "edit or info is NULL");
    if (new_tree->kind != old_tree->kind)
        return fail(QK_ERR_INVALID, "new tree kind %d differs from %d", new_tree->kind, old_tree->kind);
    if (new_tree->nodes == old_tree->nodes || new_tree->items == old_tree->items ||
        new_tree->leaves == old_tree->leaves || new_tree->bnodes == old_tree->bnodes ||
        new_tree->prim_ids == old_tree->prim_ids || new_tree->parent == old_tree->parent)
        return fail(QK_ERR_INVALID, "new tree shares arrays with the old tree");
    if (edit->n_deleted < 0 || edit->n_inserted < 0 || edit->appended < 0 || edit->n_moved < 0)
        return fail(QK_ERR_INVALID, "negative edit counts");
    const long long n_new = static_cast<long long>(old_tree->n) - edit->n_deleted +
                            edit->n_inserted + edit->appended;
    if (n_new != new_tree->n)
        return fail(QK_ERR_INVALID, "the edit leaves %lld primitives, the new tree has %d", n_new,
                    new_tree->n);
    const int n_extra = edit->n_inserted + edit->appended;
    if ((edit->n_deleted && !edit->deleted) || (edit->n_inserted && !edit->inserted) ||
        (edit->n_moved && (!edit->moved || !edit->moved_items)) || (n_extra && !edit->extra_items))
        return fail(QK_ERR_INVALID, "edit array is NULL");
    if (sah_bins < 4 || sah_bins > 64) return fail(QK_ERR_INVALID, "sah_bins must be in [4, 64]");
    st = check_ws(workspace, workspace_bytes,
                  update_ws_bytes(old_tree->kind, old_tree->n, new_tree->n, n_extra));
    if (st) return st;
    return update_topology(old_tree, new_tree, edit, cut_size, sah_bins, info, workspace,
                           as_stream(stream));
}

int qk_wide_build(qk_tree* tree, void* workspace, size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (!tree->wide_id) return fail(QK_ERR_INVALID, "wide_id is NULL");
    st = check_ws(workspace, workspace_bytes, build_ws_bytes(tree->kind, tree->n, 0));
    if (st) return st;
    return wide_build(tree, 1, workspace, workspace_bytes, as_stream(stream));
}

int qk_wide_build_leaf4(qk_tree* tree, void* workspace, size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (!tree->wide_id) return fail(QK_ERR_INVALID, "wide_id is NULL");
    st = check_ws(workspace, workspace_bytes, build_ws_bytes(tree->kind, tree->n, 0));
    if (st) return st;
    return wide_build(tree, 4, workspace, workspace_bytes, as_stream(stream));
}

int qk_raycast(const qk_tree* tree, const void* rays, int count, uint64_t* out, unsigned flags,
               uint64_t* stats, void* workspace, size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (tree->kind != QK_TRI) return fail(QK_ERR_INVALID, "raycast needs a triangle tree");
    if (count < 0) return fail(QK_ERR_INVALID, "negative ray count");
    if (count > 0 && (!rays || !out)) return fail(QK_ERR_INVALID, "rays or out is NULL");
    if ((st = check_wide(tree, flags))) return st;
    if ((st = check_ws(workspace, workspace_bytes, order_ws_bytes(count)))) return st;
    return ray_query(tree, rays, count, out, nullptr, flags, stats, workspace, as_stream(stream));
}

int qk_raycast_ids(const qk_tree* tree, const void* rays, int count, uint64_t* out, int32_t* ids,
                   unsigned flags, void* workspace, size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (tree->kind != QK_TRI) return fail(QK_ERR_INVALID, "raycast needs a triangle tree");
    if (count < 0) return fail(QK_ERR_INVALID, "negative ray count");
    if (count > 0 && (!rays || !out || !ids)) return fail(QK_ERR_INVALID, "rays, out or ids is NULL");
    if ((st = check_wide(tree, flags))) return st;
    if ((st = check_ws(workspace, workspace_bytes, order_ws_bytes(count)))) return st;
    return ray_query(tree, rays, count, out, ids, flags, nullptr, workspace, as_stream(stream));
}

namespace {
// device alias of page-locked, mapped host memory, or nullptr
void* mapped_alias(const void* host) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, host) != cudaSuccess) {
        cudaGetLastError();  // clear the (non-sticky) error the query left
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}
}  // namespace

int qk_raycast_mapped(const qk_tree* tree, const void* host_rays, int count, uint64_t* host_out,
                      unsigned flags, void* workspace, size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (tree->kind != QK_TRI) return fail(QK_ERR_INVALID, "raycast needs a triangle tree");
    if (count < 0) return fail(QK_ERR_INVALID, "negative ray count");
    if (count == 0) return QK_OK;
    if (!host_rays || !host_out) return fail(QK_ERR_INVALID, "rays or out is NULL");
    void* rays_d = mapped_alias(host_rays);
    void* out_d = mapped_alias(host_out);
    if (!rays_d || !out_d)
        return fail(QK_ERR_INVALID, "host_rays and host_out must be page-locked, mapped host memory");
    if ((reinterpret_cast<uintptr_t>(rays_d) & 15u) || (reinterpret_cast<uintptr_t>(out_d) & 7u))
        return fail(QK_ERR_INVALID, "rays must be 16-byte and results 8-byte aligned");
    if ((st = check_wide(tree, flags))) return st;
    if ((st = check_ws(workspace, workspace_bytes, order_ws_bytes(count)))) return st;
    return ray_query(tree, rays_d, count, static_cast<uint64_t*>(out_d), nullptr, flags, nullptr,
                     workspace, as_stream(stream));
}

size_t qk_raycast_host_workspace_bytes(int count, int chunks) {
    if (count <= 0) return 0;
    if (chunks < 1) chunks = 1;
    const int per = (count + chunks - 1) / chunks;
    return 2 * ((order_ws_bytes(per) + 255) / 256 * 256);
}

int qk_raycast_host(const qk_tree* tree, const void* host_rays, int count, uint64_t* host_out,
                    void* dev_rays, uint64_t* dev_out, int chunks, unsigned flags, void* workspace,
                    size_t workspace_bytes, void* upload_stream, void* trace_stream0,
                    void* trace_stream1, void* readback_stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (tree->kind != QK_TRI) return fail(QK_ERR_INVALID, "raycast needs a triangle tree");
    if (count < 0) return fail(QK_ERR_INVALID, "negative ray count");
    if (count == 0) return QK_OK;
    if (!host_rays || !host_out || !dev_rays)
        return fail(QK_ERR_INVALID, "a ray or result buffer is NULL");
    // without dev_out the traversals store the results straight into mapped host_out
    uint64_t* direct = nullptr;
    if (!dev_out) {
        direct = static_cast<uint64_t*>(mapped_alias(host_out));
        if (!direct || (reinterpret_cast<uintptr_t>(direct) & 7u))
            return fail(QK_ERR_INVALID,
                        "dev_out is NULL but host_out is not 8-byte aligned, mapped page-locked memory");
    }
    if ((st = check_wide(tree, flags))) return st;
    if (chunks < 1) chunks = 1;
    if (chunks > count) chunks = count;
    if ((st = check_ws(workspace, workspace_bytes, qk_raycast_host_workspace_bytes(count, chunks))))
        return st;
    const int per = (count + chunks - 1) / chunks;
    const size_t half = (order_ws_bytes(per) + 255) / 256 * 256;
    cudaStream_t up = as_stream(upload_stream), rb = as_stream(readback_stream);
    cudaStream_t tr[2] = {as_stream(trace_stream0), as_stream(trace_stream1)};
    // The uploads follow one another on the host-to-device copy engine and the read-backs on
    // the device-to-host engine; chunk c is traced on trace stream c % 2 with workspace half
    // c % 2, so a traversal can start while the previous one drains its last rays.  Chunk c's
    // traversal waits for its upload, its read-back for its traversal.  A wait takes the
    // event's latest record at the time of the call, so one event per edge serves every chunk.
    cudaEvent_t uploaded = nullptr, traced = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&uploaded, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&traced, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (uploaded) cudaEventDestroy(uploaded);
        return cuda_status(e, "pipeline events");
    }
    for (int c = 0; c < chunks && st == QK_OK; ++c) {
        const int b = c * per;
        const int m = b + per <= count ? per : count - b;
        if (m <= 0) break;
        cudaStream_t ts = tr[c & 1];
        void* ws = static_cast<char*>(workspace) + (c & 1) * half;
        const char* hr = static_cast<const char*>(host_rays) + static_cast<size_t>(b) * 32;
        char* dr = static_cast<char*>(dev_rays) + static_cast<size_t>(b) * 32;
        e = cudaMemcpyAsync(dr, hr, static_cast<size_t>(m) * 32, cudaMemcpyHostToDevice, up);
        if (e == cudaSuccess) e = cudaEventRecord(uploaded, up);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(ts, uploaded, 0);
        if (e != cudaSuccess) {
            st = cuda_status(e, "ray upload");
            break;
        }
        st = ray_query(tree, dr, m, (direct ? direct : dev_out) + b, nullptr, flags, nullptr, ws,
                       ts);
        if (st) break;
        e = cudaEventRecord(traced, ts);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(rb, traced, 0);
        if (e == cudaSuccess && !direct)
            e = cudaMemcpyAsync(host_out + b, dev_out + b, static_cast<size_t>(m) * 8,
                                cudaMemcpyDeviceToHost, rb);
        if (e != cudaSuccess) st = cuda_status(e, "result read-back");
    }
    // destroying an event that pending waits still reference is allowed: its resources are
    // released once the work completes
    cudaEventDestroy(uploaded);
    cudaEventDestroy(traced);
    return st;
}

size_t qk_grad_workspace_bytes(int count, int channels) {
    return count > 0 ? grad_ws_bytes(count, channels < 10 ? 10 : channels) : 256;
}

int qk_distance_grad(const qk_tree* tree, const void* items, const float* points,
                     const void* results, const float* grad_dist, int count, float* grad_points,
                     float* grad_items, void* workspace, size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (count < 0) return fail(QK_ERR_INVALID, "negative query count");
    if (!items || !grad_items || (count > 0 && (!points || !results || !grad_points)))
        return fail(QK_ERR_INVALID, "NULL array");
    if ((st = check_ws(workspace, workspace_bytes, grad_ws_bytes(count, qk_stride_floats(tree->kind)))))
        return st;
    return closest_distance_grad(tree->kind, tree->n, items, points, results, grad_dist, count,
                                 grad_points, grad_items, workspace, as_stream(stream));
}

int qk_ray_t_grad(const qk_tree* tree, const void* items, const void* rays, const int32_t* ids,
                  const float* grad_t, int count, float* grad_tris, float* grad_rays,
                  void* workspace, size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (tree->kind != QK_TRI) return fail(QK_ERR_INVALID, "ray gradients need a triangle tree");
    if (count < 0) return fail(QK_ERR_INVALID, "negative ray count");
    if (!items || !grad_tris || (count > 0 && (!rays || !ids))) return fail(QK_ERR_INVALID, "NULL array");
    if ((st = check_ws(workspace, workspace_bytes, grad_ws_bytes(count, 9)))) return st;
    return ray_t_grad(tree->n, items, rays, ids, grad_t, count, grad_tris, grad_rays, workspace,
                      as_stream(stream));
}

size_t qk_grad_vertices_workspace_bytes(int count) {
    return count >= 0 ? grad_vertices_ws_bytes(count) : 0;
}

int qk_ray_t_grad_vertices(const qk_tree* tree, const void* items, const void* rays,
                           const int32_t* ids, const float* grad_t, int count,
                           const int32_t* indices, int nverts, float* grad_verts,
                           float* grad_rays, void* workspace, size_t workspace_bytes,
                           void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (tree->kind != QK_TRI) return fail(QK_ERR_INVALID, "ray gradients need a triangle tree");
    if (count < 0 || nverts < 1) return fail(QK_ERR_INVALID, "negative ray count or no vertices");
    if (!items || !indices || !grad_verts || (count > 0 && (!rays || !ids)))
        return fail(QK_ERR_INVALID, "NULL array");
    if ((st = check_ws(workspace, workspace_bytes, grad_vertices_ws_bytes(count)))) return st;
    return ray_t_grad_vertices(tree->n, items, rays, ids, grad_t, count, indices, nverts,
                               grad_verts, grad_rays, workspace, as_stream(stream));
}

int qk_distance_grad_vertices(const qk_tree* tree, const void* items, const float* points,
                              const void* results, const float* grad_dist, int count,
                              const int32_t* indices, int nverts, float* grad_points,
                              float* grad_verts, void* workspace, size_t workspace_bytes,
                              void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (tree->kind != QK_TRI) return fail(QK_ERR_INVALID, "vertex gradients need a triangle tree");
    if (count < 0 || nverts < 1) return fail(QK_ERR_INVALID, "negative query count or no vertices");
    if (!items || !indices || !grad_verts || (count > 0 && (!points || !results || !grad_points)))
        return fail(QK_ERR_INVALID, "NULL array");
    if ((st = check_ws(workspace, workspace_bytes, grad_vertices_ws_bytes(count)))) return st;
    return distance_grad_vertices(tree->n, items, points, results, grad_dist, count, indices,
                                  nverts, grad_points, grad_verts, workspace, as_stream(stream));
}

int qk_segment_sum(const int32_t* keys, const float* values, int count, int channels, int segments,
                   float* out, void* workspace, size_t workspace_bytes, void* stream) {
    if (count < 0 || segments < 0 || channels < 1 || channels > 10)
        return fail(QK_ERR_INVALID, "bad count, segments or channels (1..10)");
    if (segments > 0 && !out) return fail(QK_ERR_INVALID, "out is NULL");
    if (count > 0 && (!keys || !values)) return fail(QK_ERR_INVALID, "NULL array");
    int st = check_ws(workspace, workspace_bytes, grad_ws_bytes(count, 0));
    if (st) return st;
    return segment_sum(keys, values, count, channels, segments, out, workspace, as_stream(stream));
}

int qk_closest(const qk_tree* tree, const float* points, int count, void* out, unsigned flags,
               uint64_t* stats, void* workspace, size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (count < 0) return fail(QK_ERR_INVALID, "negative query count");
    if (count > 0 && (!points || !out)) return fail(QK_ERR_INVALID, "points or out is NULL");
    if (flags & QK_ORDER_DIRECTION) return fail(QK_ERR_INVALID, "direction order is for rays");
    if ((st = check_wide(tree, flags))) return st;
    if ((st = check_ws(workspace, workspace_bytes, point_query_ws_bytes(count, flags)))) return st;
    return closest_query(tree, points, count, out, flags, stats, workspace, as_stream(stream));
}

int qk_knn(const qk_tree* tree, const float* points, int count, int k, int stride, void* out,
           unsigned flags, uint64_t* stats, void* workspace, size_t workspace_bytes,
           void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (k < 1 || k > kMaxKnn) return fail(QK_ERR_INVALID, "k must be in [1, 32]");
    if (stride < k) return fail(QK_ERR_INVALID, "stride must be >= k");
    if (count < 0) return fail(QK_ERR_INVALID, "negative query count");
    if (count > 0 && (!points || !out)) return fail(QK_ERR_INVALID, "points or out is NULL");
    if (flags & QK_ORDER_DIRECTION) return fail(QK_ERR_INVALID, "direction order is for rays");
    if ((st = check_wide(tree, flags))) return st;
    if ((st = check_ws(workspace, workspace_bytes, point_query_ws_bytes(count, flags)))) return st;
    return knn_query(tree, points, count, k, stride, out, flags, stats, workspace,
                     as_stream(stream));
}

int qk_radius_count(const qk_tree* tree, const float* points, int count, float radius,
                    int32_t* offsets, int64_t* total_host, unsigned flags, uint64_t* stats,
                    void* workspace, size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (!(radius >= 0.0f)) return fail(QK_ERR_INVALID, "radius must be >= 0");
    if (count < 0) return fail(QK_ERR_INVALID, "negative query count");
    if (!offsets || !total_host) return fail(QK_ERR_INVALID, "offsets or total is NULL");
    if (count > 0 && !points) return fail(QK_ERR_INVALID, "points is NULL");
    if (flags & QK_ORDER_DIRECTION) return fail(QK_ERR_INVALID, "direction order is for rays");
    if ((st = check_wide(tree, flags))) return st;
    if ((st = check_ws(workspace, workspace_bytes, radius_ws_bytes(count, flags)))) return st;
    long long total = 0;
    st = radius_count(tree, points, count, radius, offsets, &total, flags, stats, workspace,
                      as_stream(stream));
    *total_host = total;
    return st;
}

int qk_radius_fill(const qk_tree* tree, const float* points, int count, float radius,
                   const int32_t* offsets, uint64_t* keys, unsigned flags, void* workspace,
                   size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (!(radius >= 0.0f)) return fail(QK_ERR_INVALID, "radius must be >= 0");
    if (count < 0) return fail(QK_ERR_INVALID, "negative query count");
    if (count > 0 && (!points || !offsets)) return fail(QK_ERR_INVALID, "points or offsets is NULL");
    if (flags & QK_ORDER_DIRECTION) return fail(QK_ERR_INVALID, "direction order is for rays");
    if ((st = check_wide(tree, flags))) return st;
    if ((st = check_ws(workspace, workspace_bytes, radius_ws_bytes(count, flags)))) return st;
    return radius_fill(tree, points, count, radius, offsets, keys, flags, workspace,
                       as_stream(stream));
}

size_t qk_validate_workspace_bytes(int n) { return n >= 2 ? validate_ws_bytes(n) : 0; }

int qk_validate(const qk_tree* tree, const void* items, int32_t* errors, void* workspace,
                size_t workspace_bytes, void* stream) {
    int st = check_tree(tree);
    if (st) return st;
    if (!items || !errors) return fail(QK_ERR_INVALID, "items or errors is NULL");
    if ((st = check_ws(workspace, workspace_bytes, validate_ws_bytes(tree->n)))) return st;
    return validate_tree(tree, items, errors, workspace, as_stream(stream));
}

size_t qk_sort_workspace_bytes(int n) { return n > 0 ? sort_ws_bytes(n) : 0; }

int qk_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                  uint32_t* vals_out, int n, int bits, void* workspace, size_t workspace_bytes,
                  void* stream) {
    if (n < 0 || bits < 1 || bits > 32) return fail(QK_ERR_INVALID, "bad n or bits");
    if (n == 0) return QK_OK;
    if (!keys_in || !vals_in || !keys_out || !vals_out) return fail(QK_ERR_INVALID, "NULL buffer");
    int st = check_ws(workspace, workspace_bytes, sort_ws_bytes(n));
    if (st) return st;
    const cudaError_t e = sort_pairs(keys_in, vals_in, keys_out, vals_out, n, bits, workspace,
                                     as_stream(stream));
    return e == cudaSuccess ? QK_OK : cuda_status(e, "sort");
}

}  // extern "C"
