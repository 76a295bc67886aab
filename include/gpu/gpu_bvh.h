// gpu/gpu_bvh.h -- host C++ API of the B200 engine, declaration for declaration the API of
// quarry's src/gpu/gpu_bvh.h:20-352 (same types, functions, default arguments and error
// behaviour), so code written against quarry compiles and links unchanged.  No CUDA types
// appear here; device pointers are void*.  Every call is synchronous on return and reports
// CUDA failures as std::runtime_error (bad topology edits as std::invalid_argument).
//
// Internally every function forwards to the C ABI of include/quarry_b200.h.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "core/fingerprint.h"
#include "core/gaussian.h"
#include "core/geometry.h"
#include "core/point_cloud.h"
#include "core/scene.h"

// A cached device block (gpu_bvh.h:21-24).
struct GpuDevBlock {
    void* p = nullptr;
    size_t bytes = 0;
};

// One tree.  Public fields as in quarry: node array (2n-1 nodes of 32 bytes, internal
// 0..n-2, leaves n-1+slot), primitives in leaf order, leaf slot -> scene index, counts and
// depth, and the optional 4-wide node layer.  `impl` owns the rest of the device state.
struct GpuBVH {
    void* d_nodes = nullptr;
    void* d_tris = nullptr;
    void* d_primIds = nullptr;
    int primCount = 0;
    int nodeCount = 0;
    int depth = 0;
    void* d_wideNodes = nullptr;
    int wideCount = 0;
    bool sah = false;
    void* impl = nullptr;
};

struct GpuBuildTimings {
    double mortonMs = 0.0;
    double sortMs = 0.0;
    double treeMs = 0.0;
    double scatterMs = 0.0;
    double refitMs = 0.0;
    double sahBinMs = 0.0;
    double sahSplitMs = 0.0;
    double sahPartMs = 0.0;
    double totalMs = 0.0;
};

struct GpuRayBuffer {
    void* d_rays = nullptr;     // Ray[]
    void* d_results = nullptr;  // uint64 (hit << 32 | bits(t)) per ray
    int count = 0;
    void* d_sortScratch = nullptr;  // internal: query workspace
};

bool gpuDescribe(std::string* why);

GpuBVH buildBVHGPU(const Scene& scene, GpuBuildTimings* timings = nullptr);
GpuBVH buildBVHSahGPU(const Scene& scene, GpuBuildTimings* timings = nullptr);
GpuBVH buildPointBVHSahGPU(const PointCloud& cloud, GpuBuildTimings* timings = nullptr);
GpuBVH buildGaussianBVHSahGPU(const GaussianCloud& cloud, GpuBuildTimings* timings = nullptr);
// Engine addition (no quarry counterpart; the leaf-size-4 lever of quarry's docs/design.md):
// binned SAH whose split search stops at ranges of at most 4 primitives (QK_BUILD_SAH4);
// buildWideNodesGPU then gives such a tree 4-wide nodes with leaf-range slots.  Same
// results as every other build.
GpuBVH buildBVHSah4GPU(const Scene& scene, GpuBuildTimings* timings = nullptr);
GpuBVH buildPointBVHSah4GPU(const PointCloud& cloud, GpuBuildTimings* timings = nullptr);
GpuBVH buildGaussianBVHSah4GPU(const GaussianCloud& cloud, GpuBuildTimings* timings = nullptr);
GpuBVH buildPointBVHGPU(const PointCloud& cloud, GpuBuildTimings* timings = nullptr);
GpuBVH buildGaussianBVHGPU(const GaussianCloud& cloud, GpuBuildTimings* timings = nullptr);

// Loads the engine's kernels before a timed build.
void warmupBuildGPU();

struct GpuRefitTimings {
    double uploadMs = 0.0;
    double gatherMs = 0.0;
    double treeMs = 0.0;
    double markMs = 0.0;
    double mergeMs = 0.0;
    double wideMs = 0.0;
    double totalMs = 0.0;
    int updated = 0;
};

// Topology-frozen refit: same primitive count, primitive i still the same element.
double refitBVHGPU(GpuBVH& bvh, const Scene& scene, GpuRefitTimings* timings = nullptr);
double refitBVHGPU(GpuBVH& bvh, const Scene& scene, const std::vector<int>& dirty,
                   GpuRefitTimings* timings = nullptr);
double refitPointBVHGPU(GpuBVH& bvh, const PointCloud& cloud, GpuRefitTimings* timings = nullptr);
double refitPointBVHGPU(GpuBVH& bvh, const PointCloud& cloud, const std::vector<int>& dirty,
                        GpuRefitTimings* timings = nullptr);
double refitGaussianBVHGPU(GpuBVH& bvh, const GaussianCloud& cloud,
                           GpuRefitTimings* timings = nullptr);
double refitGaussianBVHGPU(GpuBVH& bvh, const GaussianCloud& cloud,
                           const std::vector<int>& dirty, GpuRefitTimings* timings = nullptr);

// Topology edit script (gpu_bvh.h:182-187): newScene = survivors of the old scene minus
// `deleted` (old indices, ascending), with new primitives at the new indices `inserted`
// (ascending, < newScene.size() - appended) and `appended` more at the end; `moved` lists
// new indices whose geometry changed.
struct GpuTopoEdit {
    std::vector<int> deleted;
    std::vector<int> moved;
    std::vector<int> inserted;
    int appended = 0;
};

struct GpuTopoUpdateTimings {
    double uploadMs = 0.0;
    double planMs = 0.0;
    double surgeryMs = 0.0;
    double relayoutMs = 0.0;
    double mergeMs = 0.0;
    double wideMs = 0.0;
    double totalMs = 0.0;
    int deleted = 0;
    int moved = 0;
    int inserted = 0;
    int appended = 0;
    int surgeryRoots = 0;
    int rebuiltLeaves = 0;
    int newDepth = 0;
    bool fullRebuild = false;
    double refitMs = 0.0;
};

// Results equal a fresh build over the new scene bit for bit.  Move-only edits take the
// partial refit; edits that change the primitive set rebuild with the tree's builder.
double updateBVHGPU(GpuBVH& bvh, const Scene& scene, const GpuTopoEdit& edit,
                    GpuTopoUpdateTimings* timings = nullptr);
double updatePointBVHGPU(GpuBVH& bvh, const PointCloud& cloud, const GpuTopoEdit& edit,
                         GpuTopoUpdateTimings* timings = nullptr);
double updateGaussianBVHGPU(GpuBVH& bvh, const GaussianCloud& cloud, const GpuTopoEdit& edit,
                            GpuTopoUpdateTimings* timings = nullptr);

void destroyBVHGPU(GpuBVH& bvh);

GpuRayBuffer uploadRaysGPU(const std::vector<Ray>& rays);
void destroyRayBufferGPU(GpuRayBuffer& buf);

// Coherent (engine addition): counting sort on a Morton key of origin and direction
enum class RayOrder { Input, Morton, MortonDirection, Coherent };

// 4-wide collapse; call again after a refit (the reference contract).  Returns ms.
double buildWideNodesGPU(GpuBVH& bvh);

// First hits; returns the device time in ms (CUDA events, no copies).
double raycastGPU(const GpuBVH& bvh, GpuRayBuffer& buf, bool collectStats = false,
                  RayOrder order = RayOrder::Input, bool wide = false);

RayStats summarizeGPU(const GpuRayBuffer& buf, std::vector<uint64_t>* perRay = nullptr);

struct GpuTraversalStats {
    uint64_t nodeTests = 0;
    uint64_t triTests = 0;
    uint64_t stackOverflows = 0;
    double sortMs = 0.0;
};
GpuTraversalStats lastTraversalStatsGPU();

struct GpuClosestResult {
    uint32_t dist2Bits = 0;
    int32_t triangle = -1;
};

struct GpuPointBuffer {
    void* d_points = nullptr;
    void* d_results = nullptr;
    int count = 0;
    int stride = 1;
    AABB bounds;
    void* d_sortScratch = nullptr;
};

struct GpuQueryStats {
    uint64_t nodeTests = 0;
    uint64_t triTests = 0;
    uint64_t stackOverflows = 0;
    double sortMs = 0.0;
};

// Coherent (engine addition): counting sort on a Morton key of the position
enum class QueryOrder { Input, Morton, Coherent };

GpuPointBuffer uploadPointsGPU(const std::vector<Vec3>& points, int resultsPerPoint = 1);
void destroyPointBufferGPU(GpuPointBuffer& buf);

double closestPointGPU(const GpuBVH& bvh, GpuPointBuffer& buf, bool collectStats = false,
                       QueryOrder order = QueryOrder::Input, bool wide = false);
double kNearestGPU(const GpuBVH& bvh, GpuPointBuffer& buf, int k, bool collectStats = false,
                   QueryOrder order = QueryOrder::Input, bool wide = false);

// CSR radius results: segment i = [offsets[i], offsets[i+1]), ascending by (dist2, index).
struct GpuRadiusBuffer {
    void* d_offsets = nullptr;  // int[count + 1]
    void* d_keys = nullptr;     // uint64 (bits(dist2) << 32) | index
    int count = 0;
    int total = 0;
};

void destroyRadiusBufferGPU(GpuRadiusBuffer& buf);

double radiusQueryGPU(const GpuBVH& bvh, GpuPointBuffer& buf, float radius, GpuRadiusBuffer& out,
                      bool collectStats = false, QueryOrder order = QueryOrder::Input,
                      bool wide = false);

std::vector<std::vector<ClosestHit>> readRadiusResultsGPU(const GpuRadiusBuffer& buf);

double closestVertexGPU(const GpuBVH& bvh, GpuPointBuffer& buf, bool collectStats = false,
                        QueryOrder order = QueryOrder::Input, bool wide = false);
double kNearestVertexGPU(const GpuBVH& bvh, GpuPointBuffer& buf, int k,
                         bool collectStats = false, QueryOrder order = QueryOrder::Input,
                         bool wide = false);
double radiusQueryVertexGPU(const GpuBVH& bvh, GpuPointBuffer& buf, float radius,
                            GpuRadiusBuffer& out, bool collectStats = false,
                            QueryOrder order = QueryOrder::Input, bool wide = false);

double closestGaussianGPU(const GpuBVH& bvh, GpuPointBuffer& buf, bool collectStats = false,
                          QueryOrder order = QueryOrder::Input, bool wide = false);
double kNearestGaussianGPU(const GpuBVH& bvh, GpuPointBuffer& buf, int k,
                           bool collectStats = false, QueryOrder order = QueryOrder::Input,
                           bool wide = false);
double radiusQueryGaussianGPU(const GpuBVH& bvh, GpuPointBuffer& buf, float radius,
                              GpuRadiusBuffer& out, bool collectStats = false,
                              QueryOrder order = QueryOrder::Input, bool wide = false);

std::vector<GpuClosestResult> readQueryResultsGPU(const GpuPointBuffer& buf);

GpuQueryStats lastQueryStatsGPU();
void warmupQueryGPU();

// Structural invariants; "" means pass.
std::string validateBVHGPU(const GpuBVH& bvh, const Scene& scene);
std::string validatePointBVHGPU(const GpuBVH& bvh, const PointCloud& cloud);
std::string validateGaussianBVHGPU(const GpuBVH& bvh, const GaussianCloud& cloud);

// 64-bit FNV-1a over the node array bytes: the determinism gate.
uint64_t treeHashGPU(const GpuBVH& bvh);

// Additive (no quarry counterpart): the tree's device arrays as the C ABI sees them
// (include/quarry_b200.h), for callers that query it with their own device buffers and
// stream -- the zero-copy path of the Python module.  Valid while `bvh` lives and is not
// rebuilt; wide nodes appear once buildWideNodesGPU has run.
const struct qk_tree* gpuTreeView(const GpuBVH& bvh);
