// qk_noalloc.cu -- a first-hit ray query that allocates nothing.
//
// Some callers cannot allocate device memory at the moment they trace rays: a host
// application that reserves all device memory up front and forbids allocations afterwards
// (frame loops, plugin hosts with a fixed budget), or code that holds no allocator at all.
// For them qk_raycast_noalloc runs the Morton-ordered ray query of qk_raycast with its
// scratch (sort keys, permutation, radix histograms) in a fixed array that lives in this
// library's device memory, so the caller passes only the tree, the rays and the output.
//
// The array is a file-scope __device__ variable: every GPU that loads the library holds
// kNoAllocScratchBytes of it until the process exits.  Host code cannot use the variable's
// name as a device address, so each call looks the address up with cudaGetSymbolAddress,
// with the caller's device current.  The address belongs to the current CUDA context (it
// changes after cudaDeviceReset, and differs under another driver context on the same
// device), so it is not kept between calls; the lookup is a host-side query that allocates
// nothing.  The first call on a device may load the library's device code, so make it
// before any stream capture.  All calls share the one array: calls whose work overlaps on
// the GPU (different streams, no ordering between them) race on it.  Each call rewrites
// every scratch word it reads before reading it, so nothing has to start at zero.
#include "qk_internal.cuh"

namespace qk {

namespace {

// Largest ray count: 262,144 rays use about 4.3 MB of scratch.
constexpr int kNoAllocMaxRays = 1 << 18;
constexpr size_t kNoAllocScratchBytes = 4608 * 1024;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The scratch address in the current context (looked up on every call, see above).
int scratch_for_current_context(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, "noalloc: current device");
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "noalloc: scratch address");
    *out = p;
    return QK_OK;
}

}  // namespace

}  // namespace qk

extern "C" int qk_raycast_noalloc(const qk_tree* tree, const void* rays, int count,
                                  uint64_t* out, unsigned flags, void* stream) {
    using namespace qk;
    if (!tree) return fail(QK_ERR_INVALID, "tree is NULL");
    if (tree->kind != QK_TRI) return fail(QK_ERR_INVALID, "raycast needs a triangle tree");
    if (tree->n < 2 || !tree->nodes || !tree->leaves || !tree->bnodes)
        return fail(QK_ERR_INVALID, "tree is not built");
    if (count < 0) return fail(QK_ERR_INVALID, "negative ray count");
    if (count > kNoAllocMaxRays)
        return fail(QK_ERR_INVALID,
                    "qk_raycast_noalloc handles at most %d rays per call (got %d); split the "
                    "batch or use qk_raycast with a caller workspace",
                    kNoAllocMaxRays, count);
    if (count > 0 && (!rays || !out)) return fail(QK_ERR_INVALID, "rays or out is NULL");
    if (tree->depth < 0 || tree->depth >= kStack)
        return fail(QK_ERR_DEPTH, "tree depth %d exceeds the traversal stack (%d levels)",
                    tree->depth, kStack - 1);
    if ((flags & QK_WIDE) && (tree->wide == nullptr || tree->wide_count <= 0))
        return fail(QK_ERR_INVALID, "wide nodes not built");
    if (__builtin_popcount(flags & (QK_ORDER_MORTON | QK_ORDER_DIRECTION | QK_ORDER_COHERENT)) > 1)
        return fail(QK_ERR_INVALID,
                    "choose one of QK_ORDER_MORTON, QK_ORDER_DIRECTION and QK_ORDER_COHERENT");
    if (count == 0) return QK_OK;
    if (order_ws_bytes(count) > kNoAllocScratchBytes)
        return fail(QK_ERR_WORKSPACE, "noalloc scratch too small for %d rays", count);
    void* scratch = nullptr;
    const int st = scratch_for_current_context(&scratch);
    if (st != QK_OK) return st;
    return ray_query(tree, rays, count, out, nullptr, flags, nullptr, scratch,
                     static_cast<cudaStream_t>(stream));
}
