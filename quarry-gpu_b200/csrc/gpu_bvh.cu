// gpu_bvh.cu -- the C++ API of include/gpu/gpu_bvh.h implemented over the C ABI
// (include/quarry_b200.h).  This layer owns device allocations (cudaMalloc / cudaFree),
// moves data between host and device, times calls with CUDA events on the legacy default
// stream and turns status codes into exceptions, exactly where quarry's own host code does
// (src/gpu/lbvh.cu, raycast.cu, query.cu).  All kernels run through qk_* entry points.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "gpu/gpu_bvh.h"
#include "qk_internal.cuh"
#include "quarry_b200.h"
#include "scenes.h"

namespace {

void cudaOk(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("CUDA ") + what + ": " + cudaGetErrorString(e));
    }
}

void qkOk(int status, const char* what) {
    if (status != QK_OK) {
        throw std::runtime_error(std::string(what) + ": " + qk_status_string(status) + " (" +
                                 qk_last_error() + ")");
    }
}

void* devAlloc(size_t bytes, const char* what) {
    void* p = nullptr;
    cudaOk(cudaMalloc(&p, std::max<size_t>(bytes, 16)), what);
    return p;
}

void devFree(void*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// Events on the legacy default stream, as the reference times its calls.
struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    Timer() {
        cudaOk(cudaEventCreate(&a), "event");
        cudaOk(cudaEventCreate(&b), "event");
        cudaOk(cudaEventRecord(a, nullptr), "event record");
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    double stop() {
        cudaOk(cudaEventRecord(b, nullptr), "event record");
        cudaOk(cudaEventSynchronize(b), "event sync");
        float ms = 0.0f;
        cudaOk(cudaEventElapsedTime(&ms, a, b), "elapsed");
        return static_cast<double>(ms);
    }
};

// Installs a qk::StageClock on this host thread for one engine call, so the builders, refits
// and topology edits record an event at each stage boundary; ms(a, b) reads a stage's device
// time (0 when a mark was not reached).  The role of quarry's StageClock
// (src/gpu/lbvh.cu:173-190).
struct StageScope {
    qk::StageClock c;
    StageScope() {
        for (cudaEvent_t& e : c.ev) cudaOk(cudaEventCreate(&e), "event");
        for (cudaEvent_t& e : c.lv) cudaOk(cudaEventCreate(&e), "event");
        qk::stage_clock() = &c;
    }
    ~StageScope() {
        qk::stage_clock() = nullptr;
        for (cudaEvent_t& e : c.ev) cudaEventDestroy(e);
        for (cudaEvent_t& e : c.lv) cudaEventDestroy(e);
    }
    StageScope(const StageScope&) = delete;
    StageScope& operator=(const StageScope&) = delete;
    double ms(int a, int b) const {
        if (!c.hit[a] || !c.hit[b]) return 0.0;
        cudaOk(cudaEventSynchronize(c.ev[b]), "event sync");
        float v = 0.0f;
        cudaOk(cudaEventElapsedTime(&v, c.ev[a], c.ev[b]), "elapsed");
        return static_cast<double>(v);
    }
};

constexpr int kTreeArrays = 10;

// Device state behind GpuBVH::impl.  Topology edits write the new tree into the spare array
// set and swap, so steady updates allocate nothing.
struct Impl {
    qk_tree t{};
    void* arrays[kTreeArrays] = {};
    int cap = 0;                     // primitives the arrays hold
    void* spare[kTreeArrays] = {};
    int spareCap = 0;
    void* ws = nullptr;
    size_t wsBytes = 0;
    void* stage = nullptr;  // scene-order upload buffer (refit, validate)
    size_t stageBytes = 0;
    void* upd = nullptr;    // topology-edit workspace and edit script
    size_t updBytes = 0;
    int builder = QK_BUILD_LBVH;
    int bins = 32;
    int baseDepth = 0;      // depth after the last full build (topology-edit depth budget)
};

void allocTreeArrays(int kind, int cap, void* arrays[kTreeArrays]) {
    qk_tree_sizes sz{};
    qkOk(qk_tree_bytes(kind, cap, &sz), "tree sizes");
    const size_t sizes[kTreeArrays] = {sz.nodes, sz.bnodes, sz.items, sz.prim_ids, sz.parent,
                                       sz.depth_arr, sz.leaves, sz.slot_of, sz.flags, sz.wide_id};
    for (int i = 0; i < kTreeArrays; ++i) arrays[i] = devAlloc(sizes[i], "tree arrays");
}

void bindTree(qk_tree& t, int kind, int n, void* const arrays[kTreeArrays]) {
    t.kind = kind;
    t.n = n;
    t.nodes = arrays[0];
    t.bnodes = arrays[1];
    t.items = arrays[2];
    t.prim_ids = static_cast<int32_t*>(arrays[3]);
    t.parent = static_cast<int32_t*>(arrays[4]);
    t.depth_arr = static_cast<int32_t*>(arrays[5]);
    t.leaves = arrays[6];
    t.slot_of = static_cast<int32_t*>(arrays[7]);
    t.flags = static_cast<int32_t*>(arrays[8]);
    t.wide_id = static_cast<int32_t*>(arrays[9]);
}

Impl* implOf(const GpuBVH& bvh) {
    if (!bvh.impl) throw std::runtime_error("GpuBVH is not built");
    return static_cast<Impl*>(bvh.impl);
}

void* stageOf(Impl* im, size_t bytes) {
    if (im->stageBytes < bytes) {
        devFree(im->stage);
        im->stage = devAlloc(bytes, "stage");
        im->stageBytes = bytes;
    }
    return im->stage;
}

void syncPublic(GpuBVH& bvh, Impl* im) {
    bvh.d_nodes = im->t.nodes;
    bvh.d_tris = im->t.items;
    bvh.d_primIds = im->t.prim_ids;
    bvh.primCount = im->t.n;
    bvh.nodeCount = 2 * im->t.n - 1;
    bvh.depth = im->t.depth;
    bvh.d_wideNodes = im->t.wide;
    bvh.wideCount = im->t.wide_count;
}

void freeImpl(Impl* im) {
    if (!im) return;
    for (void*& p : im->arrays) devFree(p);
    for (void*& p : im->spare) devFree(p);
    devFree(im->ws);
    devFree(im->stage);
    devFree(im->upd);
    if (im->t.wide) {
        void* w = im->t.wide;
        cudaFree(w);
    }
    delete im;
}

GpuBVH buildImpl(int kind, const void* host, size_t itemBytes, int n, int builder,
                 GpuBuildTimings* timings) {
    if (n < 2) throw std::runtime_error("build: at least 2 primitives required");
    auto* im = new Impl;
    GpuBVH bvh;
    try {
        allocTreeArrays(kind, n, im->arrays);
        im->cap = n;
        qk_tree& t = im->t;
        bindTree(t, kind, n, im->arrays);
        t.wide = nullptr;
        cudaOk(cudaMemset(t.flags, 0, sizeof(int32_t) * static_cast<size_t>(n - 1)), "flags");
        im->builder = builder;
        im->wsBytes = qk_build_workspace_bytes(kind, n, builder);
        im->ws = devAlloc(im->wsBytes, "build workspace");
        void* src = stageOf(im, itemBytes * static_cast<size_t>(n));
        cudaOk(cudaMemcpy(src, host, itemBytes * static_cast<size_t>(n), cudaMemcpyHostToDevice),
               "H2D prims");
        StageScope clock;
        Timer timer;
        qkOk(qk_build(&t, builder, im->bins, src, im->ws, im->wsBytes, nullptr), "build");
        const double ms = timer.stop();
        if (timings) {
            // stage times as quarry reports them (src/gpu/lbvh.cu:2027-2034, 2105-2115)
            using namespace qk;
            GpuBuildTimings& bt = *timings;
            bt = GpuBuildTimings{};
            if (builder == QK_BUILD_SAH || builder == QK_BUILD_SAH4) {
                // topology (levels + lower tiers) and depths; the leaf scatter; the boxes
                bt.treeMs = clock.ms(kMarkStart, kMarkTopo) + clock.ms(kMarkBoxes, kMarkEnd);
                bt.scatterMs = clock.ms(kMarkTopo, kMarkScatter);
                bt.refitMs = clock.ms(kMarkScatter, kMarkBoxes);
                bt.sahBinMs = clock.c.sah_bin;
                bt.sahSplitMs = clock.c.sah_split;
                bt.sahPartMs = clock.c.sah_part;
            } else {
                // the emit kernel writes the leaves (the scatter) and the internal nodes in
                // one pass, so its time is in treeMs and scatterMs stays 0
                bt.mortonMs = clock.ms(kMarkStart, kMarkMorton);
                bt.sortMs = clock.ms(kMarkMorton, kMarkSort);
                bt.treeMs = clock.ms(kMarkSort, kMarkTopo) + clock.ms(kMarkBoxes, kMarkEnd);
                bt.refitMs = clock.ms(kMarkTopo, kMarkBoxes);
            }
            bt.totalMs = clock.ms(kMarkStart, kMarkEnd);
            if (bt.totalMs <= 0.0) bt.totalMs = ms;
        }
        bvh.sah = builder != QK_BUILD_LBVH;
        im->baseDepth = t.depth;
        bvh.impl = im;
        syncPublic(bvh, im);
    } catch (...) {
        freeImpl(im);
        throw;
    }
    return bvh;
}

template <typename Item>
double refitImpl(GpuBVH& bvh, const std::vector<Item>& items, const std::vector<int>* dirty,
                 GpuRefitTimings* timings) {
    Impl* im = implOf(bvh);
    const int n = im->t.n;
    if (static_cast<int>(items.size()) != n) {
        throw std::runtime_error("refitBVHGPU: primitive count changed, rebuild instead");
    }
    GpuRefitTimings local;
    GpuRefitTimings* tm = timings ? timings : &local;
    *tm = GpuRefitTimings{};
    Timer timer;
    StageScope clock;
    double uploadMs = 0.0;
    if (dirty) {
        // unique, in range; the engine writes each dirty leaf once
        std::vector<int> ids = *dirty;
        for (int id : ids) {
            if (id < 0 || id >= n) throw std::runtime_error("refitBVHGPU: dirty index out of range");
        }
        std::sort(ids.begin(), ids.end());
        ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
        const int count = static_cast<int>(ids.size());
        if (count > 0) {
            std::vector<Item> moved(static_cast<size_t>(count));
            for (int i = 0; i < count; ++i) moved[static_cast<size_t>(i)] = items[static_cast<size_t>(ids[static_cast<size_t>(i)])];
            char* st = static_cast<char*>(stageOf(im, sizeof(int) * count + 256 + sizeof(Item) * count));
            int* dIds = reinterpret_cast<int*>(st);
            void* dItems = st + ((sizeof(int) * count + 255) / 256) * 256;
            Timer up;
            cudaOk(cudaMemcpy(dIds, ids.data(), sizeof(int) * count, cudaMemcpyHostToDevice), "H2D ids");
            cudaOk(cudaMemcpy(dItems, moved.data(), sizeof(Item) * count, cudaMemcpyHostToDevice), "H2D prims");
            uploadMs = up.stop();
            qkOk(qk_refit_dirty(&im->t, dIds, dItems, count, im->ws, im->wsBytes, nullptr), "refit");
        }
        tm->updated = count;
    } else {
        void* src = stageOf(im, sizeof(Item) * static_cast<size_t>(n));
        Timer up;
        cudaOk(cudaMemcpy(src, items.data(), sizeof(Item) * static_cast<size_t>(n),
                          cudaMemcpyHostToDevice),
               "H2D prims");
        uploadMs = up.stop();
        qkOk(qk_refit(&im->t, src, im->ws, im->wsBytes, nullptr), "refit");
        tm->updated = n;
    }
    const double ms = timer.stop();
    // stage times as quarry reports them (src/gpu/gpu_bvh.h:129-138): the full refit gathers
    // the leaves then merges; the dirty refit rewrites the dirty leaves and marks their
    // ancestors in one kernel (markMs), then merges them
    {
        using namespace qk;
        tm->uploadMs = uploadMs;
        const double first = clock.ms(kMarkStart, kMarkScatter);
        tm->mergeMs = clock.ms(kMarkScatter, kMarkBoxes);
        if (dirty) {
            tm->markMs = first;
            tm->treeMs = first + tm->mergeMs;
        } else {
            tm->gatherMs = first;
            tm->treeMs = tm->mergeMs;
        }
        tm->wideMs = clock.ms(kMarkBoxes, kMarkEnd);
        tm->totalMs = ms;
    }
    syncPublic(bvh, im);
    return ms;
}

void checkEdit(int nOld, const GpuTopoEdit& edit, size_t newSize) {
    if (nOld < 2) throw std::invalid_argument("updateBVHGPU: BVH not built");
    if (edit.appended < 0) throw std::invalid_argument("updateBVHGPU: appended must be >= 0");
    for (size_t i = 0; i < edit.deleted.size(); ++i) {
        const int id = edit.deleted[i];
        if (id < 0 || id >= nOld) throw std::invalid_argument("updateBVHGPU: deleted out of range");
        if (i > 0 && id <= edit.deleted[i - 1])
            throw std::invalid_argument("updateBVHGPU: deleted must be ascending and unique");
    }
    const long long nNew = static_cast<long long>(nOld) - static_cast<long long>(edit.deleted.size()) +
                           static_cast<long long>(edit.inserted.size()) + edit.appended;
    if (nNew < 2) throw std::invalid_argument("updateBVHGPU: at least 2 primitives required");
    if (static_cast<long long>(newSize) != nNew)
        throw std::invalid_argument("updateBVHGPU: scene size does not match the edit");
    const long long tailBeg = nNew - edit.appended;
    for (size_t i = 0; i < edit.inserted.size(); ++i) {
        const int id = edit.inserted[i];
        if (id < 0 || id >= tailBeg)
            throw std::invalid_argument("updateBVHGPU: inserted index out of range");
        if (i > 0 && id <= edit.inserted[i - 1])
            throw std::invalid_argument("updateBVHGPU: inserted must be ascending and unique");
    }
    for (int id : edit.moved) {
        if (id < 0 || id >= nNew) throw std::invalid_argument("updateBVHGPU: moved index out of range");
    }
}

// Depth a topology edit may add over the last full build before the tree is rebuilt to
// rebalance it (quarry's kTopoDepthSlack, src/gpu/lbvh.cu:2543-2545).
constexpr int kTopoDepthSlack = 6;

size_t alignUp(size_t b) { return (b + 255) / 256 * 256; }

template <typename Item>
double updateImpl(GpuBVH& bvh, int kind, const std::vector<Item>& items, const GpuTopoEdit& edit,
                  GpuTopoUpdateTimings* timings) {
    if (!bvh.impl) throw std::invalid_argument("updateBVHGPU: BVH not built");
    Impl* im = implOf(bvh);
    checkEdit(im->t.n, edit, items.size());
    GpuTopoUpdateTimings local;
    GpuTopoUpdateTimings* t = timings ? timings : &local;
    *t = GpuTopoUpdateTimings{};
    t->deleted = static_cast<int>(edit.deleted.size());
    t->inserted = static_cast<int>(edit.inserted.size());
    t->appended = edit.appended;
    t->moved = static_cast<int>(edit.moved.size());
    if (edit.deleted.empty() && edit.inserted.empty() && edit.appended == 0) {
        GpuRefitTimings rt;
        t->refitMs = refitImpl<Item>(bvh, items, &edit.moved, &rt);
        t->moved = rt.updated;
        t->totalMs = t->refitMs;
        t->newDepth = bvh.depth;
        return t->totalMs;
    }
    const bool wide = im->t.wide != nullptr;
    const int nOld = im->t.n;
    const int nNew = static_cast<int>(items.size());
    const int nIns = static_cast<int>(edit.inserted.size());
    const int nDel = static_cast<int>(edit.deleted.size());
    const int nMov = static_cast<int>(edit.moved.size());
    const int extra = nIns + edit.appended;
    Timer timer;

    // rebuild with the tree's own builder (results equal a fresh build by construction) and
    // restore the 4-wide layer when the tree had one
    auto rebuildAll = [&]() -> double {
        const int builder = im->builder;
        GpuBVH fresh = buildImpl(kind, items.data(), sizeof(Item), nNew, builder, nullptr);
        destroyBVHGPU(bvh);
        bvh = fresh;
        im = implOf(bvh);
        double wideMs = 0.0;
        if (wide) wideMs = buildWideNodesGPU(bvh);
        t->totalMs = timer.stop();
        t->wideMs = wideMs;
        t->surgeryMs = t->totalMs - wideMs;
        t->surgeryRoots = 1;
        t->rebuiltLeaves = bvh.primCount;
        t->newDepth = bvh.depth;
        t->fullRebuild = true;
        return t->totalMs;
    };
    // more than half of the primitives change: a rebuild costs about as much
    if (nDel + extra > nOld / 2) return rebuildAll();

    // the edit script and only the primitives it brings, in one upload
    const size_t oDel = 0, oIns = alignUp(sizeof(int) * nDel);
    const size_t oMov = oIns + alignUp(sizeof(int) * nIns);
    const size_t oExtra = oMov + alignUp(sizeof(int) * nMov);
    const size_t oMoved = oExtra + alignUp(sizeof(Item) * extra);
    const size_t scriptBytes = oMoved + alignUp(sizeof(Item) * nMov);
    std::vector<char> script(scriptBytes);
    if (nDel) std::memcpy(script.data() + oDel, edit.deleted.data(), sizeof(int) * nDel);
    if (nIns) std::memcpy(script.data() + oIns, edit.inserted.data(), sizeof(int) * nIns);
    if (nMov) std::memcpy(script.data() + oMov, edit.moved.data(), sizeof(int) * nMov);
    Item* ex = reinterpret_cast<Item*>(script.data() + oExtra);
    for (int k = 0; k < nIns; ++k) ex[k] = items[static_cast<size_t>(edit.inserted[k])];
    for (int k = 0; k < edit.appended; ++k)
        ex[nIns + k] = items[static_cast<size_t>(nNew - edit.appended + k)];
    Item* mv = reinterpret_cast<Item*>(script.data() + oMoved);
    for (int k = 0; k < nMov; ++k) mv[k] = items[static_cast<size_t>(edit.moved[k])];
    const size_t wsBytes = alignUp(qk_update_workspace_bytes(kind, nOld, nNew, extra));
    if (im->updBytes < wsBytes + scriptBytes) {
        // headroom for the next edits (scenes that grow a little per edit reuse it)
        devFree(im->upd);
        im->updBytes = alignUp(qk_update_workspace_bytes(kind, nOld + nOld / 8, nNew + nNew / 8,
                                                         extra + extra / 8 + 64)) +
                       scriptBytes + scriptBytes / 8;
        im->upd = devAlloc(im->updBytes, "topology workspace");
    }
    char* dScript = static_cast<char*>(im->upd) + wsBytes;
    cudaOk(cudaMemcpy(dScript, script.data(), scriptBytes, cudaMemcpyHostToDevice), "H2D edit");
    Timer surgery;

    if (im->spareCap < nNew) {
        for (void*& p : im->spare) devFree(p);
        im->spareCap = nNew + nNew / 8 + 16;
        allocTreeArrays(kind, im->spareCap, im->spare);
    }
    qk_tree nt{};
    bindTree(nt, kind, nNew, im->spare);
    qk_topo_edit ed{};
    ed.deleted = reinterpret_cast<const int32_t*>(dScript + oDel);
    ed.n_deleted = nDel;
    ed.inserted = reinterpret_cast<const int32_t*>(dScript + oIns);
    ed.n_inserted = nIns;
    ed.appended = edit.appended;
    ed.moved = reinterpret_cast<const int32_t*>(dScript + oMov);
    ed.n_moved = nMov;
    ed.extra_items = dScript + oExtra;
    ed.moved_items = dScript + oMoved;
    qk_topo_info info{};
    double planMs = 0.0, relayoutMs = 0.0, forestMs = 0.0, mergeMs = 0.0;
    {
        StageScope clock;
        qkOk(qk_update_topology(&im->t, &nt, &ed, 0, im->bins, &info, im->upd, wsBytes, nullptr),
             "topology update");
        using namespace qk;
        planMs = clock.ms(kMarkStart, kMarkPlan);
        relayoutMs = clock.ms(kMarkPlan, kMarkRelayout);
        forestMs = clock.ms(kMarkRelayout, kMarkTopo);
        mergeMs = clock.ms(kMarkTopo, kMarkEnd);
    }
    if (info.rebuild || nt.depth > im->baseDepth + kTopoDepthSlack) return rebuildAll();
    // the whole device call; its stages: cut plan, renumbering + leaf staging, the forest
    // builds of the touched subtrees, and the box merge of the new tree (with depths)
    const double deviceMs = surgery.stop();
    t->planMs = planMs;
    t->relayoutMs = relayoutMs;
    t->mergeMs = mergeMs;
    t->surgeryMs = forestMs > 0.0 ? forestMs : deviceMs;

    nt.wide = im->t.wide;  // reused by the wide rebuild below (or freed with the tree)
    nt.wide_count = 0;
    im->t = nt;
    for (int i = 0; i < kTreeArrays; ++i) std::swap(im->arrays[i], im->spare[i]);
    std::swap(im->cap, im->spareCap);
    if (qk_build_workspace_bytes(kind, nNew, im->builder) > im->wsBytes) {
        devFree(im->ws);
        im->wsBytes = qk_build_workspace_bytes(kind, nNew + nNew / 8, im->builder);
        im->ws = devAlloc(im->wsBytes, "build workspace");
    }
    syncPublic(bvh, im);
    double wideMs = 0.0;
    if (wide) wideMs = buildWideNodesGPU(bvh);
    t->totalMs = timer.stop();
    t->wideMs = wideMs;
    t->uploadMs = std::max(0.0, t->totalMs - deviceMs - wideMs);
    t->surgeryRoots = info.cuts;
    t->rebuiltLeaves = info.new_leaves;
    t->newDepth = bvh.depth;
    t->fullRebuild = false;
    return t->totalMs;
}

thread_local GpuTraversalStats gRayStats;
thread_local GpuQueryStats gQueryStats;

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// Query workspace with 4 stats words at its end.
struct QueryWs {
    void* ws;
    size_t bytes;
    uint64_t* stats;
};

QueryWs queryWs(void* scratch, int count) {
    const size_t b = align256(qk_query_workspace_bytes(count, QK_ORDER_MORTON));
    return {scratch, b, reinterpret_cast<uint64_t*>(static_cast<char*>(scratch) + b)};
}

unsigned flagsOf(QueryOrder order, bool wide) {
    return (order == QueryOrder::Morton ? QK_ORDER_MORTON : 0u) |
           (order == QueryOrder::Coherent ? QK_ORDER_COHERENT : 0u) | (wide ? QK_WIDE : 0u);
}

void requireWide(const GpuBVH& bvh, bool wide, const char* who) {
    if (wide && implOf(bvh)->t.wide == nullptr) {
        throw std::runtime_error(std::string(who) + ": wide nodes not built");
    }
}

template <typename F>
double timedQuery(const GpuBVH& bvh, GpuPointBuffer& buf, bool collectStats, F&& call) {
    gQueryStats = GpuQueryStats{};
    if (buf.count <= 0 || bvh.nodeCount <= 0) return 0.0;
    const QueryWs w = queryWs(buf.d_sortScratch, buf.count);
    if (collectStats) cudaOk(cudaMemset(w.stats, 0, 32), "stats");
    Timer timer;
    qkOk(call(w, collectStats ? w.stats : nullptr), "query");
    const double ms = timer.stop();
    if (collectStats) {
        uint64_t s[4];
        cudaOk(cudaMemcpy(s, w.stats, sizeof(s), cudaMemcpyDeviceToHost), "stats");
        gQueryStats.nodeTests = s[0];
        gQueryStats.triTests = s[1];
        gQueryStats.stackOverflows = s[2];
    }
    return ms;
}

double closestAny(const GpuBVH& bvh, GpuPointBuffer& buf, bool collectStats, QueryOrder order,
                  bool wide) {
    requireWide(bvh, wide, "closestPointGPU");
    Impl* im = implOf(bvh);
    return timedQuery(bvh, buf, collectStats, [&](const QueryWs& w, uint64_t* st) {
        return qk_closest(&im->t, static_cast<const float*>(buf.d_points), buf.count,
                          buf.d_results, flagsOf(order, wide), st, w.ws, w.bytes, nullptr);
    });
}

double knnAny(const GpuBVH& bvh, GpuPointBuffer& buf, int k, bool collectStats, QueryOrder order,
              bool wide) {
    requireWide(bvh, wide, "kNearestGPU");
    if (k < 1 || k > 32) throw std::runtime_error("kNearestGPU: k must be in [1, 32]");
    if (buf.stride < k)
        throw std::runtime_error("kNearestGPU: result buffer was uploaded with a smaller stride");
    Impl* im = implOf(bvh);
    return timedQuery(bvh, buf, collectStats, [&](const QueryWs& w, uint64_t* st) {
        return qk_knn(&im->t, static_cast<const float*>(buf.d_points), buf.count, k, buf.stride,
                      buf.d_results, flagsOf(order, wide), st, w.ws, w.bytes, nullptr);
    });
}

double radiusAny(const GpuBVH& bvh, GpuPointBuffer& buf, float radius, GpuRadiusBuffer& out,
                 bool collectStats, QueryOrder order, bool wide) {
    out = GpuRadiusBuffer{};
    gQueryStats = GpuQueryStats{};
    if (buf.count <= 0 || bvh.nodeCount <= 0) return 0.0;
    requireWide(bvh, wide, "radiusQueryGPU");
    Impl* im = implOf(bvh);
    const unsigned flags = flagsOf(order, wide);
    const size_t wsBytes = qk_radius_workspace_bytes(buf.count, flags);
    void* ws = devAlloc(wsBytes + 256, "radius workspace");
    uint64_t* stats = reinterpret_cast<uint64_t*>(static_cast<char*>(ws) + align256(wsBytes));
    int32_t* offsets = static_cast<int32_t*>(devAlloc(sizeof(int32_t) * (buf.count + 1), "radius offsets"));
    uint64_t* keys = nullptr;
    double ms = 0.0;
    try {
        if (collectStats) cudaOk(cudaMemset(stats, 0, 32), "stats");
        Timer timer;
        int64_t total = 0;
        qkOk(qk_radius_count(&im->t, static_cast<const float*>(buf.d_points), buf.count, radius,
                             offsets, &total, flags, collectStats ? stats : nullptr, ws, wsBytes,
                             nullptr),
             "radius count");
        if (total > 0x7fffffffLL) throw std::runtime_error("radiusQueryGPU: more than 2^31 results");
        keys = static_cast<uint64_t*>(devAlloc(sizeof(uint64_t) * static_cast<size_t>(std::max<int64_t>(total, 1)), "radius keys"));
        qkOk(qk_radius_fill(&im->t, static_cast<const float*>(buf.d_points), buf.count, radius,
                            offsets, keys, flags, ws, wsBytes, nullptr),
             "radius fill");
        ms = timer.stop();
        out.total = static_cast<int>(total);
        if (collectStats) {
            uint64_t s[4];
            cudaOk(cudaMemcpy(s, stats, sizeof(s), cudaMemcpyDeviceToHost), "stats");
            gQueryStats.nodeTests = s[0];
            gQueryStats.triTests = s[1];
            gQueryStats.stackOverflows = s[2];
        }
    } catch (...) {
        cudaFree(ws);
        cudaFree(offsets);
        if (keys) cudaFree(keys);
        throw;
    }
    cudaFree(ws);
    out.d_offsets = offsets;
    out.d_keys = keys;
    out.count = buf.count;
    return ms;
}

std::string validateAny(const GpuBVH& bvh, const void* host, size_t itemBytes, int n,
                        const AABB& bounds) {
    Impl* im = implOf(bvh);
    if (bvh.nodeCount != 2 * bvh.primCount - 1) return "nodeCount != 2n-1";
    if (n != bvh.primCount) return "prim count mismatch";
    void* src = stageOf(im, itemBytes * static_cast<size_t>(n) + 256);
    cudaOk(cudaMemcpy(src, host, itemBytes * static_cast<size_t>(n), cudaMemcpyHostToDevice),
           "validate H2D");
    const size_t wsb = qk_validate_workspace_bytes(n);
    void* ws = devAlloc(wsb + 256, "validate workspace");
    int32_t* dErr = reinterpret_cast<int32_t*>(static_cast<char*>(ws) + align256(wsb));
    int err[8] = {};
    try {
        qkOk(qk_validate(&im->t, src, dErr, ws, wsb, nullptr), "validate");
        cudaOk(cudaMemcpy(err, dErr, sizeof(err), cudaMemcpyDeviceToHost), "validate D2H");
    } catch (...) {
        cudaFree(ws);
        throw;
    }
    cudaFree(ws);
    float root[8];
    cudaOk(cudaMemcpy(root, bvh.d_nodes, sizeof(root), cudaMemcpyDeviceToHost), "root");
    const bool badRoot = root[0] != bounds.mn.x || root[1] != bounds.mn.y ||
                         root[2] != bounds.mn.z || root[3] != bounds.mx.x ||
                         root[4] != bounds.mx.y || root[5] != bounds.mx.z;
    std::string why;
    auto add = [&](const char* name, long long v) {
        char b[96];
        std::snprintf(b, sizeof(b), "%s%s=%lld", why.empty() ? "" : " ", name, v);
        why += b;
    };
    if (err[0]) add("bad_children_or_box", err[0]);
    if (err[1]) add("bad_leaf_box", err[1]);
    if (err[2]) add("bad_refcount", err[2]);
    if (err[3]) add("bad_leaf_id", err[3]);
    if (err[4]) add("bad_prim_map", err[4]);
    if (err[5]) add("bad_depth", err[5]);
    if (err[6]) add("bad_wide_node", err[6]);
    if (badRoot) add("root_box_mismatch", 1);
    return why;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// API
// ---------------------------------------------------------------------------------------
bool gpuDescribe(std::string* why) {
    char buf[256];
    if (!qk_describe(buf, sizeof(buf))) {
        if (why) *why = "no CUDA device";
        return false;
    }
    if (why) *why = buf;
    return true;
}

GpuBVH buildBVHGPU(const Scene& scene, GpuBuildTimings* timings) {
    return buildImpl(QK_TRI, scene.tris.data(), sizeof(Tri), static_cast<int>(scene.tris.size()),
                     QK_BUILD_LBVH, timings);
}
GpuBVH buildBVHSahGPU(const Scene& scene, GpuBuildTimings* timings) {
    return buildImpl(QK_TRI, scene.tris.data(), sizeof(Tri), static_cast<int>(scene.tris.size()),
                     QK_BUILD_SAH, timings);
}
GpuBVH buildPointBVHGPU(const PointCloud& cloud, GpuBuildTimings* timings) {
    return buildImpl(QK_POINT, cloud.pts.data(), sizeof(Vec3), static_cast<int>(cloud.pts.size()),
                     QK_BUILD_LBVH, timings);
}
GpuBVH buildPointBVHSahGPU(const PointCloud& cloud, GpuBuildTimings* timings) {
    return buildImpl(QK_POINT, cloud.pts.data(), sizeof(Vec3), static_cast<int>(cloud.pts.size()),
                     QK_BUILD_SAH, timings);
}
GpuBVH buildGaussianBVHGPU(const GaussianCloud& cloud, GpuBuildTimings* timings) {
    return buildImpl(QK_GAUSS, cloud.gaussians.data(), sizeof(Gaussian),
                     static_cast<int>(cloud.gaussians.size()), QK_BUILD_LBVH, timings);
}
GpuBVH buildGaussianBVHSahGPU(const GaussianCloud& cloud, GpuBuildTimings* timings) {
    return buildImpl(QK_GAUSS, cloud.gaussians.data(), sizeof(Gaussian),
                     static_cast<int>(cloud.gaussians.size()), QK_BUILD_SAH, timings);
}
GpuBVH buildBVHSah4GPU(const Scene& scene, GpuBuildTimings* timings) {
    return buildImpl(QK_TRI, scene.tris.data(), sizeof(Tri), static_cast<int>(scene.tris.size()),
                     QK_BUILD_SAH4, timings);
}
GpuBVH buildPointBVHSah4GPU(const PointCloud& cloud, GpuBuildTimings* timings) {
    return buildImpl(QK_POINT, cloud.pts.data(), sizeof(Vec3), static_cast<int>(cloud.pts.size()),
                     QK_BUILD_SAH4, timings);
}
GpuBVH buildGaussianBVHSah4GPU(const GaussianCloud& cloud, GpuBuildTimings* timings) {
    return buildImpl(QK_GAUSS, cloud.gaussians.data(), sizeof(Gaussian),
                     static_cast<int>(cloud.gaussians.size()), QK_BUILD_SAH4, timings);
}

void warmupBuildGPU() {
    // a tiny build touches every build kernel once so module loading is not timed later
    std::vector<Vec3> pts = {{0, 0, 0}, {1, 1, 1}, {2, 0, 1}};
    PointCloud c;
    c.pts = pts;
    GpuBVH b = buildPointBVHGPU(c);
    destroyBVHGPU(b);
}

double refitBVHGPU(GpuBVH& bvh, const Scene& scene, GpuRefitTimings* timings) {
    return refitImpl<Tri>(bvh, scene.tris, nullptr, timings);
}
double refitBVHGPU(GpuBVH& bvh, const Scene& scene, const std::vector<int>& dirty,
                   GpuRefitTimings* timings) {
    return refitImpl<Tri>(bvh, scene.tris, &dirty, timings);
}
double refitPointBVHGPU(GpuBVH& bvh, const PointCloud& cloud, GpuRefitTimings* timings) {
    return refitImpl<Vec3>(bvh, cloud.pts, nullptr, timings);
}
double refitPointBVHGPU(GpuBVH& bvh, const PointCloud& cloud, const std::vector<int>& dirty,
                        GpuRefitTimings* timings) {
    return refitImpl<Vec3>(bvh, cloud.pts, &dirty, timings);
}
double refitGaussianBVHGPU(GpuBVH& bvh, const GaussianCloud& cloud, GpuRefitTimings* timings) {
    return refitImpl<Gaussian>(bvh, cloud.gaussians, nullptr, timings);
}
double refitGaussianBVHGPU(GpuBVH& bvh, const GaussianCloud& cloud, const std::vector<int>& dirty,
                           GpuRefitTimings* timings) {
    return refitImpl<Gaussian>(bvh, cloud.gaussians, &dirty, timings);
}

double updateBVHGPU(GpuBVH& bvh, const Scene& scene, const GpuTopoEdit& edit,
                    GpuTopoUpdateTimings* timings) {
    return updateImpl<Tri>(bvh, QK_TRI, scene.tris, edit, timings);
}
double updatePointBVHGPU(GpuBVH& bvh, const PointCloud& cloud, const GpuTopoEdit& edit,
                         GpuTopoUpdateTimings* timings) {
    return updateImpl<Vec3>(bvh, QK_POINT, cloud.pts, edit, timings);
}
double updateGaussianBVHGPU(GpuBVH& bvh, const GaussianCloud& cloud, const GpuTopoEdit& edit,
                            GpuTopoUpdateTimings* timings) {
    return updateImpl<Gaussian>(bvh, QK_GAUSS, cloud.gaussians, edit, timings);
}

void destroyBVHGPU(GpuBVH& bvh) {
    freeImpl(static_cast<Impl*>(bvh.impl));
    bvh = GpuBVH{};
}

double buildWideNodesGPU(GpuBVH& bvh) {
    Impl* im = implOf(bvh);
    Timer timer;
    void* old = im->t.wide;
    im->t.wide = nullptr;
    // a leaf-size-4 SAH tree gets the 4-wide form with leaf-range slots
    auto wide_build = im->builder == QK_BUILD_SAH4 ? qk_wide_build_leaf4 : qk_wide_build;
    qkOk(wide_build(&im->t, im->ws, im->wsBytes, nullptr), "wide count");
    if (old) cudaFree(old);
    im->t.wide = devAlloc(static_cast<size_t>(im->t.wide_count) * 128, "wide nodes");
    qkOk(wide_build(&im->t, im->ws, im->wsBytes, nullptr), "wide emit");
    const double ms = timer.stop();
    syncPublic(bvh, im);
    return ms;
}

GpuRayBuffer uploadRaysGPU(const std::vector<Ray>& rays) {
    GpuRayBuffer buf;
    buf.count = static_cast<int>(rays.size());
    if (buf.count == 0) return buf;
    buf.d_rays = devAlloc(sizeof(Ray) * rays.size(), "rays");
    buf.d_results = devAlloc(sizeof(uint64_t) * rays.size(), "results");
    buf.d_sortScratch = devAlloc(align256(qk_query_workspace_bytes(buf.count, QK_ORDER_MORTON)) + 256,
                                 "ray workspace");
    cudaOk(cudaMemcpy(buf.d_rays, rays.data(), sizeof(Ray) * rays.size(), cudaMemcpyHostToDevice),
           "H2D rays");
    return buf;
}

void destroyRayBufferGPU(GpuRayBuffer& buf) {
    devFree(buf.d_rays);
    devFree(buf.d_results);
    devFree(buf.d_sortScratch);
    buf = GpuRayBuffer{};
}

double raycastGPU(const GpuBVH& bvh, GpuRayBuffer& buf, bool collectStats, RayOrder order,
                  bool wide) {
    gRayStats = GpuTraversalStats{};
    if (buf.count <= 0 || bvh.nodeCount <= 0) return 0.0;
    requireWide(bvh, wide, "raycastGPU");
    Impl* im = implOf(bvh);
    const QueryWs w = queryWs(buf.d_sortScratch, buf.count);
    unsigned flags = wide ? QK_WIDE : 0u;
    if (order == RayOrder::Morton) flags |= QK_ORDER_MORTON;
    if (order == RayOrder::MortonDirection) flags |= QK_ORDER_DIRECTION;
    if (order == RayOrder::Coherent) flags |= QK_ORDER_COHERENT;
    if (collectStats) cudaOk(cudaMemset(w.stats, 0, 32), "stats");
    Timer timer;
    qkOk(qk_raycast(&im->t, buf.d_rays, buf.count, static_cast<uint64_t*>(buf.d_results), flags,
                    collectStats ? w.stats : nullptr, w.ws, w.bytes, nullptr),
         "raycast");
    const double ms = timer.stop();
    if (collectStats) {
        uint64_t s[4];
        cudaOk(cudaMemcpy(s, w.stats, sizeof(s), cudaMemcpyDeviceToHost), "stats");
        gRayStats.nodeTests = s[0];
        gRayStats.triTests = s[1];
        gRayStats.stackOverflows = s[2];
    }
    return ms;
}

RayStats summarizeGPU(const GpuRayBuffer& buf, std::vector<uint64_t>* perRay) {
    RayStats stats;
    if (buf.count <= 0) return stats;
    std::vector<uint64_t> host(static_cast<size_t>(buf.count));
    cudaOk(cudaMemcpy(host.data(), buf.d_results, host.size() * sizeof(uint64_t),
                      cudaMemcpyDeviceToHost),
           "D2H results");
    for (uint64_t v : host) {
        RayHit h;
        h.hit = (v >> 32) != 0;
        if (h.hit) {
            const uint32_t bits = static_cast<uint32_t>(v);
            std::memcpy(&h.t, &bits, sizeof(bits));
        }
        stats.add(h);
    }
    if (perRay) *perRay = std::move(host);
    return stats;
}

GpuTraversalStats lastTraversalStatsGPU() { return gRayStats; }

GpuPointBuffer uploadPointsGPU(const std::vector<Vec3>& points, int resultsPerPoint) {
    GpuPointBuffer buf;
    buf.count = static_cast<int>(points.size());
    buf.stride = resultsPerPoint > 0 ? resultsPerPoint : 1;
    if (buf.count == 0) return buf;
    buf.bounds = AABB{};
    for (const Vec3& p : points) buf.bounds.extend(p);
    buf.d_points = devAlloc(sizeof(Vec3) * points.size(), "points");
    buf.d_results = devAlloc(sizeof(GpuClosestResult) * points.size() * buf.stride, "query results");
    buf.d_sortScratch = devAlloc(align256(qk_query_workspace_bytes(buf.count, QK_ORDER_MORTON)) + 256,
                                 "query workspace");
    cudaOk(cudaMemcpy(buf.d_points, points.data(), sizeof(Vec3) * points.size(),
                      cudaMemcpyHostToDevice),
           "H2D points");
    return buf;
}

void destroyPointBufferGPU(GpuPointBuffer& buf) {
    devFree(buf.d_points);
    devFree(buf.d_results);
    devFree(buf.d_sortScratch);
    buf = GpuPointBuffer{};
}

double closestPointGPU(const GpuBVH& bvh, GpuPointBuffer& buf, bool s, QueryOrder o, bool w) {
    return closestAny(bvh, buf, s, o, w);
}
double closestVertexGPU(const GpuBVH& bvh, GpuPointBuffer& buf, bool s, QueryOrder o, bool w) {
    return closestAny(bvh, buf, s, o, w);
}
double closestGaussianGPU(const GpuBVH& bvh, GpuPointBuffer& buf, bool s, QueryOrder o, bool w) {
    return closestAny(bvh, buf, s, o, w);
}
double kNearestGPU(const GpuBVH& bvh, GpuPointBuffer& buf, int k, bool s, QueryOrder o, bool w) {
    return knnAny(bvh, buf, k, s, o, w);
}
double kNearestVertexGPU(const GpuBVH& bvh, GpuPointBuffer& buf, int k, bool s, QueryOrder o,
                         bool w) {
    return knnAny(bvh, buf, k, s, o, w);
}
double kNearestGaussianGPU(const GpuBVH& bvh, GpuPointBuffer& buf, int k, bool s, QueryOrder o,
                           bool w) {
    return knnAny(bvh, buf, k, s, o, w);
}
double radiusQueryGPU(const GpuBVH& bvh, GpuPointBuffer& buf, float r, GpuRadiusBuffer& out,
                      bool s, QueryOrder o, bool w) {
    return radiusAny(bvh, buf, r, out, s, o, w);
}
double radiusQueryVertexGPU(const GpuBVH& bvh, GpuPointBuffer& buf, float r, GpuRadiusBuffer& out,
                            bool s, QueryOrder o, bool w) {
    return radiusAny(bvh, buf, r, out, s, o, w);
}
double radiusQueryGaussianGPU(const GpuBVH& bvh, GpuPointBuffer& buf, float r,
                              GpuRadiusBuffer& out, bool s, QueryOrder o, bool w) {
    return radiusAny(bvh, buf, r, out, s, o, w);
}

void destroyRadiusBufferGPU(GpuRadiusBuffer& buf) {
    devFree(buf.d_offsets);
    devFree(buf.d_keys);
    buf = GpuRadiusBuffer{};
}

std::vector<std::vector<ClosestHit>> readRadiusResultsGPU(const GpuRadiusBuffer& buf) {
    std::vector<std::vector<ClosestHit>> out;
    if (buf.count <= 0) return out;
    out.resize(static_cast<size_t>(buf.count));
    std::vector<int> offsets(static_cast<size_t>(buf.count) + 1);
    cudaOk(cudaMemcpy(offsets.data(), buf.d_offsets, offsets.size() * sizeof(int),
                      cudaMemcpyDeviceToHost),
           "D2H radius offsets");
    std::vector<uint64_t> keys(static_cast<size_t>(buf.total));
    if (buf.total > 0) {
        cudaOk(cudaMemcpy(keys.data(), buf.d_keys, keys.size() * sizeof(uint64_t),
                          cudaMemcpyDeviceToHost),
               "D2H radius keys");
    }
    for (int i = 0; i < buf.count; ++i) {
        auto& list = out[static_cast<size_t>(i)];
        list.reserve(static_cast<size_t>(offsets[i + 1] - offsets[i]));
        for (int j = offsets[i]; j < offsets[i + 1]; ++j) {
            ClosestHit h;
            h.found = true;
            const uint32_t bits = static_cast<uint32_t>(keys[static_cast<size_t>(j)] >> 32);
            std::memcpy(&h.dist2, &bits, sizeof(float));
            h.triangle = static_cast<int>(static_cast<uint32_t>(keys[static_cast<size_t>(j)]));
            list.push_back(h);
        }
    }
    return out;
}

std::vector<GpuClosestResult> readQueryResultsGPU(const GpuPointBuffer& buf) {
    std::vector<GpuClosestResult> host(static_cast<size_t>(buf.count) * buf.stride);
    if (buf.count <= 0) return host;
    cudaOk(cudaMemcpy(host.data(), buf.d_results, host.size() * sizeof(GpuClosestResult),
                      cudaMemcpyDeviceToHost),
           "D2H query results");
    return host;
}

GpuQueryStats lastQueryStatsGPU() { return gQueryStats; }

void warmupQueryGPU() {
    std::vector<Vec3> pts = {{0, 0, 0}, {1, 1, 1}, {2, 0, 1}};
    PointCloud c;
    c.pts = pts;
    GpuBVH b = buildPointBVHGPU(c);
    GpuPointBuffer q = uploadPointsGPU(pts, 1);
    closestVertexGPU(b, q);
    destroyPointBufferGPU(q);
    destroyBVHGPU(b);
}

std::string validateBVHGPU(const GpuBVH& bvh, const Scene& scene) {
    return validateAny(bvh, scene.tris.data(), sizeof(Tri), static_cast<int>(scene.tris.size()),
                       scene.bounds);
}
std::string validatePointBVHGPU(const GpuBVH& bvh, const PointCloud& cloud) {
    return validateAny(bvh, cloud.pts.data(), sizeof(Vec3), static_cast<int>(cloud.pts.size()),
                       cloud.bounds);
}
std::string validateGaussianBVHGPU(const GpuBVH& bvh, const GaussianCloud& cloud) {
    return validateAny(bvh, cloud.gaussians.data(), sizeof(Gaussian),
                       static_cast<int>(cloud.gaussians.size()), cloud.bounds);
}

const qk_tree* gpuTreeView(const GpuBVH& bvh) { return &implOf(bvh)->t; }

uint64_t treeHashGPU(const GpuBVH& bvh) {
    std::vector<unsigned char> bytes(static_cast<size_t>(bvh.nodeCount) * 32);
    if (!bytes.empty()) {
        cudaOk(cudaMemcpy(bytes.data(), bvh.d_nodes, bytes.size(), cudaMemcpyDeviceToHost),
               "tree hash D2H");
    }
    uint64_t h = 0xcbf29ce484222325ull;
    for (unsigned char c : bytes) h = (h ^ static_cast<uint64_t>(c)) * 0x100000001b3ull;
    return h;
}

// ---------------------------------------------------------------------------------------
// core: demo inputs (src/core/scene.cpp, point_cloud.cpp, gaussian.cpp) and Gaussian bounds
// ---------------------------------------------------------------------------------------
namespace {

void gaussAxes(const Quat& q, Vec3& u, Vec3& v, Vec3& w) {
    const float lenSq = std::fma(q.w, q.w, std::fma(q.z, q.z, std::fma(q.y, q.y, q.x * q.x)));
    float inv = 1.0f;
    if (lenSq > 0.0f) inv = 1.0f / std::sqrt(lenSq);
    const float qx = q.x * inv, qy = q.y * inv, qz = q.z * inv, qw = q.w * inv;
    const float yyzz = std::fma(qy, qy, qz * qz);
    const float xxzz = std::fma(qx, qx, qz * qz);
    const float xxyy = std::fma(qx, qx, qy * qy);
    u = {std::fma(-2.0f, yyzz, 1.0f), 2.0f * std::fma(qx, qy, qz * qw), 2.0f * std::fma(qx, qz, -(qy * qw))};
    v = {2.0f * std::fma(qx, qy, -(qz * qw)), std::fma(-2.0f, xxzz, 1.0f), 2.0f * std::fma(qy, qz, qx * qw)};
    w = {2.0f * std::fma(qx, qz, qy * qw), 2.0f * std::fma(qy, qz, -(qx * qw)), std::fma(-2.0f, xxyy, 1.0f)};
}

// padded ellipsoid box, the engine's leaf box (gaussian.h:46-64 of the reference)
AABB gaussBox(const Gaussian& g) {
    Vec3 u, v, w;
    gaussAxes(g.rot, u, v, w);
    const float a2 = g.scale.x * g.scale.x, b2 = g.scale.y * g.scale.y, c2 = g.scale.z * g.scale.z;
    const float uu[3] = {u.x, u.y, u.z}, vv[3] = {v.x, v.y, v.z}, ww[3] = {w.x, w.y, w.z};
    const float m[3] = {g.mean.x, g.mean.y, g.mean.z};
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        const float half = std::sqrt(std::fma(c2, ww[a] * ww[a], std::fma(b2, vv[a] * vv[a], a2 * uu[a] * uu[a])));
        const float pad = half + 1e-6f * (1.0f + std::fabs(m[a]) + half);
        lo[a] = m[a] - pad;
        hi[a] = m[a] + pad;
    }
    AABB b;
    b.mn = {lo[0], lo[1], lo[2]};
    b.mx = {hi[0], hi[1], hi[2]};
    return b;
}

}  // namespace

void GaussianCloud::updateBounds() {
    bounds = AABB{};
    for (const Gaussian& g : gaussians) bounds.extend(gaussBox(g));
}

float terrainHeight(float x, float z) {
    return 3.0f * std::sin(0.13f * x) * std::cos(0.11f * z) +
           1.2f * std::sin(0.37f * x + 0.7f) * std::sin(0.31f * z + 1.3f) +
           0.4f * std::sin(0.90f * x) * std::sin(0.80f * z);
}

Scene buildScene(const SceneSpec& spec) {
    int kind = -1;
    if (spec.kind == "terrain") kind = 0;
    else if (spec.kind == "random") kind = 1;
    else if (spec.kind == "mixed") kind = 2;
    else if (spec.kind == "city") kind = 3;
    Scene s;
    if (kind < 0) return s;
    const int64_t n = qs_demo_mesh(kind, spec.grid, spec.randomTris, spec.seed, spec.buildings, nullptr);
    s.tris.resize(static_cast<size_t>(n));
    qs_demo_mesh(kind, spec.grid, spec.randomTris, spec.seed, spec.buildings,
                 reinterpret_cast<float*>(s.tris.data()));
    s.updateBounds();
    return s;
}

PointCloud buildPointCloud(const PointCloudSpec& spec) {
    PointCloud c;
    if (spec.count <= 0) return c;
    // PCG32 stream 4 (point_cloud.cpp:118-143 of the reference), via the demo Gaussian
    // generator's sibling in scenes.c is not exposed; restate here with the same draws
    struct Pcg {
        uint64_t state = 0, inc = 0;
        uint32_t next() {
            const uint64_t old = state;
            state = old * 6364136223846793005ull + inc;
            const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
            const uint32_t rot = static_cast<uint32_t>(old >> 59u);
            return (xs >> rot) | (xs << ((0u - rot) & 31u));
        }
        float u01() { return static_cast<float>(next() >> 8) * (1.0f / 16777216.0f); }
        float uni(float lo, float hi) { return lo + (hi - lo) * u01(); }
    } rng;
    rng.inc = (4ull << 1u) | 1u;
    rng.next();
    rng.state += 0x853c49e6748fea9bull;
    rng.next();
    rng.state += spec.seed;
    rng.next();
    const float half = 50.0f;
    c.pts.reserve(static_cast<size_t>(spec.count));
    for (int i = 0; i < spec.count; ++i) {
        if (spec.kind == "volume") {
            const float x = rng.uni(-half, half);
            const float y = rng.uni(-half, half);
            const float z = rng.uni(-half, half);
            c.pts.push_back({x, y, z});
        } else {
            const float x = rng.uni(-half, half);
            const float z = rng.uni(-half, half);
            const float y = terrainHeight(x, z) + rng.uni(-0.02f, 0.02f);
            c.pts.push_back({x, y, z});
        }
    }
    c.updateBounds();
    return c;
}

GaussianCloud buildGaussianCloud(const GaussianCloudSpec& spec) {
    GaussianCloud c;
    if (spec.count <= 0) return c;
    c.gaussians.resize(static_cast<size_t>(spec.count));
    qs_demo_gaussians(spec.kind == "volume" ? 1 : 0, spec.count, spec.seed,
                      reinterpret_cast<float*>(c.gaussians.data()));
    c.updateBounds();
    return c;
}

std::vector<Ray> makeRays(const AABB& bounds, RayMode mode, int count, uint64_t seed) {
    struct Pcg {
        uint64_t state = 0, inc = 0;
        uint32_t next() {
            const uint64_t old = state;
            state = old * 6364136223846793005ull + inc;
            const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
            const uint32_t rot = static_cast<uint32_t>(old >> 59u);
            return (xs >> rot) | (xs << ((0u - rot) & 31u));
        }
        float u01() { return static_cast<float>(next() >> 8) * (1.0f / 16777216.0f); }
        float uni(float lo, float hi) { return lo + (hi - lo) * u01(); }
    } rng;
    rng.inc = (2ull << 1u) | 1u;
    rng.next();
    rng.state += 0x853c49e6748fea9bull;
    rng.next();
    rng.state += seed;
    rng.next();
    std::vector<Ray> rays;
    rays.reserve(static_cast<size_t>(count));
    const Vec3 center = bounds.center();
    const Vec3 ext = bounds.extent();
    if (mode == RayMode::Down) {
        for (int i = 0; i < count; ++i) {
            Ray r;
            const float x = rng.uni(bounds.mn.x, bounds.mx.x);
            const float z = rng.uni(bounds.mn.z, bounds.mx.z);
            r.origin = {x, bounds.mx.y + 10.0f, z};
            r.dir = {0.0f, -1.0f, 0.0f};
            r.tMax = ext.y + 20.0f;
            rays.push_back(r);
        }
        return rays;
    }
    const float radius = 1.6f * length(ext);
    for (int i = 0; i < count; ++i) {
        const float theta = rng.uni(0.0f, 6.2831853f);
        const float phi = std::acos(rng.uni(-1.0f, 1.0f));
        const Vec3 origin{center.x + radius * std::sin(phi) * std::cos(theta),
                          center.y + radius * std::sin(phi) * std::sin(theta),
                          center.z + radius * std::cos(phi)};
        const float tx = rng.uni(-1.0f, 1.0f), ty = rng.uni(-1.0f, 1.0f), tz = rng.uni(-1.0f, 1.0f);
        const Vec3 target{center.x + tx * ext.x * 0.9f, center.y + ty * ext.y * 0.9f,
                          center.z + tz * ext.z * 0.9f};
        Ray r;
        r.origin = origin;
        r.dir = normalize(target - origin);
        r.tMax = radius * 4.0f;
        rays.push_back(r);
    }
    return rays;
}

const char* rayModeName(RayMode mode) { return mode == RayMode::Down ? "down" : "random"; }

std::vector<Vec3> makeQueryPoints(const AABB& bounds, int count, uint64_t seed) {
    struct Pcg {
        uint64_t state = 0, inc = 0;
        uint32_t next() {
            const uint64_t old = state;
            state = old * 6364136223846793005ull + inc;
            const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
            const uint32_t rot = static_cast<uint32_t>(old >> 59u);
            return (xs >> rot) | (xs << ((0u - rot) & 31u));
        }
        float u01() { return static_cast<float>(next() >> 8) * (1.0f / 16777216.0f); }
        float uni(float lo, float hi) { return lo + (hi - lo) * u01(); }
    } rng;
    rng.inc = (3ull << 1u) | 1u;
    rng.next();
    rng.state += 0x853c49e6748fea9bull;
    rng.next();
    rng.state += seed;
    rng.next();
    std::vector<Vec3> pts;
    pts.reserve(static_cast<size_t>(count));
    const Vec3 c = bounds.center();
    const Vec3 h = bounds.extent() * 0.6f;
    for (int i = 0; i < count; ++i) {
        const float x = rng.uni(-h.x, h.x), y = rng.uni(-h.y, h.y), z = rng.uni(-h.z, h.z);
        pts.push_back({c.x + x, c.y + y, c.z + z});
    }
    return pts;
}
