// quarry_py.cpp -- the Python module `quarry` over the C++ API (include/gpu/gpu_bvh.h).
//
// Same surface as quarry's bindings/python/quarry_py.cpp:887-1050: describe, demo_mesh,
// demo_gaussians and the Scene / PointCloud / GaussianCloud classes with their properties,
// update / update_topology methods and closest / knn / radius / raycast queries.  Inputs are
// float32 / int32 numpy arrays (cast when needed), results come back as numpy arrays, the
// GIL is released around device work, bad input raises ValueError (std::invalid_argument)
// and CUDA failures RuntimeError.  Additive over the reference: wide=True on every query
// (4-wide traversal, built on first use), order= on raycast ("input", "morton",
// "direction", "coherent") and order="coherent" on the point queries.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpu/gpu_bvh.h"
#include "quarry_b200.h"

namespace py = pybind11;

namespace {

using F32 = py::array_t<float, py::array::c_style | py::array::forcecast>;
using I32 = py::array_t<int32_t, py::array::c_style | py::array::forcecast>;

enum class Leaf { Tri, Point, Gauss };

QueryOrder queryOrder(const std::string& s) {
    if (s == "input") return QueryOrder::Input;
    if (s == "morton") return QueryOrder::Morton;
    if (s == "coherent") return QueryOrder::Coherent;
    throw std::invalid_argument("order must be 'input', 'morton' or 'coherent'");
}

RayOrder rayOrder(const std::string& s) {
    if (s == "input") return RayOrder::Input;
    if (s == "morton") return RayOrder::Morton;
    if (s == "direction") return RayOrder::MortonDirection;
    if (s == "coherent") return RayOrder::Coherent;
    throw std::invalid_argument("order must be 'input', 'morton', 'direction' or 'coherent'");
}

// 0: LBVH, 1: binned SAH, 2: leaf-size-4 binned SAH ("sah4", an engine addition)
int sahBuilder(const std::string& s) {
    if (s == "lbvh") return 0;
    if (s == "sah") return 1;
    if (s == "sah4") return 2;
    throw std::invalid_argument("builder must be 'lbvh' or 'sah'");
}

std::vector<Vec3> points3(const F32& a, const char* what) {
    if (a.ndim() != 2 || a.shape(1) != 3)
        throw std::invalid_argument(std::string(what) + " must have shape (N, 3)");
    std::vector<Vec3> out(static_cast<size_t>(a.shape(0)));
    if (!out.empty()) std::memcpy(out.data(), a.data(), out.size() * sizeof(Vec3));
    return out;
}

std::vector<Tri> triangles(const F32& a) {
    if (a.ndim() != 3 || a.shape(1) != 3 || a.shape(2) != 3)
        throw std::invalid_argument("triangles must have shape (M, 3, 3)");
    if (a.shape(0) < 2) throw std::invalid_argument("at least 2 triangles are required");
    std::vector<Tri> out(static_cast<size_t>(a.shape(0)));
    std::memcpy(out.data(), a.data(), out.size() * sizeof(Tri));
    return out;
}

std::vector<Tri> meshTriangles(const std::vector<Vec3>& v, const std::vector<int32_t>& idx) {
    const size_t m = idx.size() / 3;
    const int n = static_cast<int>(v.size());
    std::vector<Tri> out(m);
    for (size_t i = 0; i < m; ++i) {
        const int a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
        if (a < 0 || b < 0 || c < 0 || a >= n || b >= n || c >= n)
            throw std::invalid_argument("indices out of range");
        out[i] = {v[static_cast<size_t>(a)], v[static_cast<size_t>(b)], v[static_cast<size_t>(c)]};
    }
    return out;
}

std::vector<Gaussian> gaussians(const F32& means, const F32& rot, const F32& scale) {
    if (means.ndim() != 2 || means.shape(1) != 3 || scale.ndim() != 2 || scale.shape(1) != 3)
        throw std::invalid_argument("means and scales must have shape (N, 3)");
    if (rot.ndim() != 2 || rot.shape(1) != 4)
        throw std::invalid_argument("rotations must have shape (N, 4) as xyzw quaternions");
    const py::ssize_t n = means.shape(0);
    if (rot.shape(0) != n || scale.shape(0) != n)
        throw std::invalid_argument("means, rotations and scales must have the same length");
    std::vector<Gaussian> out(static_cast<size_t>(n));
    const float* m = means.data();
    const float* q = rot.data();
    const float* s = scale.data();
    for (py::ssize_t i = 0; i < n; ++i) {
        Gaussian& g = out[static_cast<size_t>(i)];
        g.mean = {m[3 * i], m[3 * i + 1], m[3 * i + 2]};
        g.rot = {q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]};
        g.scale = {s[3 * i], s[3 * i + 1], s[3 * i + 2]};
        if (!(g.scale.x > 0.0f) || !(g.scale.y > 0.0f) || !(g.scale.z > 0.0f))
            throw std::invalid_argument("semi-axes must be positive");
    }
    return out;
}

py::dict boundsDict(const AABB& b) {
    py::dict d;
    d["min"] = py::make_tuple(b.mn.x, b.mn.y, b.mn.z);
    d["max"] = py::make_tuple(b.mx.x, b.mx.y, b.mx.z);
    return d;
}

GpuTopoEdit topoEdit(const py::object& deleted, const py::object& moved,
                     const py::object& inserted, long long oldCount, long long newCount) {
    GpuTopoEdit e;
    auto take = [](const py::object& o, std::vector<int>& dst) {
        if (o.is_none()) return;
        const I32 a = o.cast<I32>();
        dst.assign(a.data(), a.data() + a.size());
    };
    take(deleted, e.deleted);
    take(moved, e.moved);
    take(inserted, e.inserted);
    const long long appended = newCount - oldCount + static_cast<long long>(e.deleted.size()) -
                               static_cast<long long>(e.inserted.size());
    if (appended < 0 || appended > std::numeric_limits<int>::max())
        throw std::invalid_argument(
            "new primitive count must be old count - deleted + inserted + appended");
    e.appended = static_cast<int>(appended);
    return e;
}

// The edit names the survivors' new places only through `deleted` and `inserted`; `moved`
// names those whose geometry changed.  A script that places an insertion one index off
// (quarry's own edge-insert check passes [0, n] for items that np.insert put at 0 and n + 1)
// leaves a survivor on an index whose primitive is not the one it was, and the tree would keep
// the old geometry there.  So every survivor is compared, byte for byte, with the primitive now
// at its new index, and each one that differs joins `moved`: the tree always describes the
// scene passed in.  Host work, linear in the scene, beside the conversion the module already
// does.
template <class T>
void addChangedSurvivors(const std::vector<T>& before, const std::vector<T>& after,
                         GpuTopoEdit& e) {
    const long long nOld = static_cast<long long>(before.size());
    const long long nNew = static_cast<long long>(after.size());
    const long long tail = nNew - e.appended;
    std::vector<char> named(static_cast<size_t>(nNew), 0);
    for (int id : e.moved)
        if (id >= 0 && id < nNew) named[static_cast<size_t>(id)] = 1;
    size_t di = 0, ii = 0;
    long long j = 0;  // new index of the next survivor
    for (long long k = 0; k < nOld; ++k) {
        if (di < e.deleted.size() && e.deleted[di] == k) {
            ++di;
            continue;
        }
        while (ii < e.inserted.size() && e.inserted[ii] == j) {
            ++ii;
            ++j;
        }
        if (j >= tail) break;  // a malformed script: the update itself rejects it
        if (!named[static_cast<size_t>(j)] &&
            std::memcmp(&before[static_cast<size_t>(k)], &after[static_cast<size_t>(j)], sizeof(T)) != 0)
            e.moved.push_back(static_cast<int>(j));
        ++j;
    }
}

py::dict topoDict(const GpuTopoUpdateTimings& t) {
    py::dict d;
    d["upload_ms"] = t.uploadMs;
    d["plan_ms"] = t.planMs;
    d["surgery_ms"] = t.surgeryMs;
    d["relayout_ms"] = t.relayoutMs;
    d["merge_ms"] = t.mergeMs;
    d["wide_ms"] = t.wideMs;
    d["total_ms"] = t.totalMs;
    d["refit_ms"] = t.refitMs;
    d["deleted"] = t.deleted;
    d["moved"] = t.moved;
    d["inserted"] = t.inserted;
    d["appended"] = t.appended;
    d["surgery_roots"] = t.surgeryRoots;
    d["rebuilt_leaves"] = t.rebuiltLeaves;
    d["new_depth"] = t.newDepth;
    d["full_rebuild"] = t.fullRebuild;
    return d;
}

std::vector<int> dirtyIds(const py::object& dirty) {
    std::vector<int> ids;
    if (!dirty.is_none()) {
        const I32 a = dirty.cast<I32>();
        ids.assign(a.data(), a.data() + a.size());
    }
    return ids;
}

// Shared state and queries of the three classes.
struct Base {
    GpuBVH bvh;
    GpuBuildTimings timings{};
    GpuRefitTimings refitTimings{};
    GpuTopoUpdateTimings topoTimings{};
    AABB bounds;
    double buildMs = 0.0, lastQueryMs = 0.0, refitMs = 0.0;
    int sah = 0;  // sahBuilder's code
    bool wideBuilt = false;
    Leaf leaf = Leaf::Tri;

    ~Base() { destroyBVHGPU(bvh); }

    void ensureWide(bool wide) {
        if (wide && !wideBuilt) {
            py::gil_scoped_release r;
            buildWideNodesGPU(bvh);
            wideBuilt = true;
        }
    }

    py::dict buildStats() const {
        py::dict d;
        d["morton_ms"] = timings.mortonMs;
        d["sort_ms"] = timings.sortMs;
        d["scatter_ms"] = timings.scatterMs;
        d["tree_ms"] = timings.treeMs;
        d["refit_ms"] = timings.refitMs;
        d["total_ms"] = timings.totalMs;
        d["sah_bin_ms"] = timings.sahBinMs;
        d["sah_split_ms"] = timings.sahSplitMs;
        d["sah_partition_ms"] = timings.sahPartMs;
        return d;
    }

    py::dict refitStats() const {
        py::dict d;
        d["upload_ms"] = refitTimings.uploadMs;
        d["scatter_ms"] = refitTimings.gatherMs;
        d["tree_ms"] = refitTimings.treeMs;
        d["mark_ms"] = refitTimings.markMs;
        d["merge_ms"] = refitTimings.mergeMs;
        d["total_ms"] = refitTimings.totalMs;
        d["updated"] = refitTimings.updated;
        return d;
    }

    py::tuple closest(const F32& points, const std::string& order, bool wide) {
        const std::vector<Vec3> pts = points3(points, "points");
        const QueryOrder o = queryOrder(order);
        ensureWide(wide);
        std::vector<GpuClosestResult> res;
        {
            py::gil_scoped_release r;
            GpuPointBuffer buf = uploadPointsGPU(pts, 1);
            try {
                lastQueryMs = leaf == Leaf::Tri     ? closestPointGPU(bvh, buf, false, o, wide)
                              : leaf == Leaf::Point ? closestVertexGPU(bvh, buf, false, o, wide)
                                                    : closestGaussianGPU(bvh, buf, false, o, wide);
                res = readQueryResultsGPU(buf);
            } catch (...) {
                destroyPointBufferGPU(buf);
                throw;
            }
            destroyPointBufferGPU(buf);
        }
        py::array_t<float> d2(static_cast<py::ssize_t>(res.size()));
        py::array_t<int32_t> id(static_cast<py::ssize_t>(res.size()));
        float* pd = d2.mutable_data();
        int32_t* pi = id.mutable_data();
        for (size_t i = 0; i < res.size(); ++i) {
            std::memcpy(&pd[i], &res[i].dist2Bits, sizeof(float));
            pi[i] = res[i].triangle;
        }
        return py::make_tuple(d2, id);
    }

    py::tuple knn(const F32& points, int k, const std::string& order, bool wide) {
        if (k < 1 || k > 32) throw std::invalid_argument("k must be in [1, 32]");
        const std::vector<Vec3> pts = points3(points, "points");
        const QueryOrder o = queryOrder(order);
        ensureWide(wide);
        std::vector<GpuClosestResult> res;
        {
            py::gil_scoped_release r;
            GpuPointBuffer buf = uploadPointsGPU(pts, k);
            try {
                lastQueryMs = leaf == Leaf::Tri ? kNearestGPU(bvh, buf, k, false, o, wide)
                              : leaf == Leaf::Point
                                  ? kNearestVertexGPU(bvh, buf, k, false, o, wide)
                                  : kNearestGaussianGPU(bvh, buf, k, false, o, wide);
                res = readQueryResultsGPU(buf);
            } catch (...) {
                destroyPointBufferGPU(buf);
                throw;
            }
            destroyPointBufferGPU(buf);
        }
        const py::ssize_t n = static_cast<py::ssize_t>(pts.size());
        py::array_t<float> d2({n, static_cast<py::ssize_t>(k)});
        py::array_t<int32_t> id({n, static_cast<py::ssize_t>(k)});
        float* pd = d2.mutable_data();
        int32_t* pi = id.mutable_data();
        for (size_t i = 0; i < res.size(); ++i) {
            std::memcpy(&pd[i], &res[i].dist2Bits, sizeof(float));
            pi[i] = res[i].triangle;
        }
        return py::make_tuple(d2, id);
    }

    py::tuple radius(const F32& points, float radius, const std::string& order, bool wide) {
        if (!(radius >= 0.0f)) throw std::invalid_argument("radius must be >= 0");
        const std::vector<Vec3> pts = points3(points, "points");
        const QueryOrder o = queryOrder(order);
        ensureWide(wide);
        std::vector<std::vector<ClosestHit>> hits;
        {
            py::gil_scoped_release r;
            GpuPointBuffer buf = uploadPointsGPU(pts, 1);
            GpuRadiusBuffer out;
            try {
                lastQueryMs =
                    leaf == Leaf::Tri     ? radiusQueryGPU(bvh, buf, radius, out, false, o, wide)
                    : leaf == Leaf::Point ? radiusQueryVertexGPU(bvh, buf, radius, out, false, o, wide)
                                          : radiusQueryGaussianGPU(bvh, buf, radius, out, false, o, wide);
                hits = readRadiusResultsGPU(out);
            } catch (...) {
                destroyRadiusBufferGPU(out);
                destroyPointBufferGPU(buf);
                throw;
            }
            destroyRadiusBufferGPU(out);
            destroyPointBufferGPU(buf);
        }
        const py::ssize_t n = static_cast<py::ssize_t>(pts.size());
        py::array_t<int64_t> offsets(n + 1);
        int64_t* po = offsets.mutable_data();
        po[0] = 0;
        size_t total = 0;
        for (py::ssize_t i = 0; i < n; ++i) {
            total += hits.empty() ? 0 : hits[static_cast<size_t>(i)].size();
            po[i + 1] = static_cast<int64_t>(total);
        }
        py::array_t<float> d2(static_cast<py::ssize_t>(total));
        py::array_t<int32_t> id(static_cast<py::ssize_t>(total));
        float* pd = d2.mutable_data();
        int32_t* pi = id.mutable_data();
        size_t at = 0;
        for (const auto& list : hits) {
            for (const ClosestHit& h : list) {
                pd[at] = h.dist2;
                pi[at] = h.triangle;
                ++at;
            }
        }
        return py::make_tuple(offsets, d2, id);
    }
};

class PyScene : public Base {
public:
    PyScene(const F32& tris, const std::string& builder) {
        leaf = Leaf::Tri;
        sah = sahBuilder(builder);
        tris_ = triangles(tris);
        build();
    }
    PyScene(const F32& vertices, const I32& indices, const std::string& builder) {
        leaf = Leaf::Tri;
        sah = sahBuilder(builder);
        const std::vector<Vec3> v = points3(vertices, "vertices");
        if (indices.ndim() != 2 || indices.shape(1) != 3)
            throw std::invalid_argument("indices must have shape (M, 3)");
        if (indices.shape(0) < 2) throw std::invalid_argument("at least 2 triangles are required");
        indices_.assign(indices.data(), indices.data() + indices.size());
        tris_ = meshTriangles(v, indices_);
        build();
    }

    int triangleCount() const { return bvh.primCount; }
    std::string validate() const {
        py::gil_scoped_release r;
        return validateBVHGPU(bvh, scene_);
    }

    py::tuple raycast(const F32& origins, const F32& dirs, float tmax, const std::string& order,
                      bool wide) {
        const std::vector<Vec3> o = points3(origins, "origins");
        const std::vector<Vec3> d = points3(dirs, "dirs");
        if (o.size() != d.size()) throw std::invalid_argument("origins and dirs must match");
        const RayOrder ro = rayOrder(order);
        ensureWide(wide);
        std::vector<Ray> rays(o.size());
        for (size_t i = 0; i < o.size(); ++i) rays[i] = {o[i], d[i], 1e-6f, tmax};
        std::vector<uint64_t> per;
        {
            py::gil_scoped_release r;
            GpuRayBuffer buf = uploadRaysGPU(rays);
            try {
                lastQueryMs = raycastGPU(bvh, buf, false, ro, wide);
                summarizeGPU(buf, &per);
            } catch (...) {
                destroyRayBufferGPU(buf);
                throw;
            }
            destroyRayBufferGPU(buf);
        }
        py::array_t<bool> hit(static_cast<py::ssize_t>(per.size()));
        py::array_t<float> t(static_cast<py::ssize_t>(per.size()));
        bool* ph = hit.mutable_data();
        float* pt = t.mutable_data();
        for (size_t i = 0; i < per.size(); ++i) {
            ph[i] = (per[i] >> 32) != 0;
            if (ph[i]) {
                const uint32_t bits = static_cast<uint32_t>(per[i]);
                std::memcpy(&pt[i], &bits, sizeof(float));
            } else {
                pt[i] = std::numeric_limits<float>::infinity();
            }
        }
        return py::make_tuple(hit, t);
    }

    void updateTriangles(const F32& tris, const py::object& dirty) { update(triangles(tris), dirty); }

    void updateVertices(const F32& vertices, const py::object& dirty) {
        if (indices_.empty())
            throw std::invalid_argument("Scene was built from triangles; use update_triangles");
        update(meshTriangles(points3(vertices, "vertices"), indices_), dirty);
    }

    py::dict updateTopology(const F32& tris, const py::object& deleted, const py::object& moved,
                            const py::object& inserted) {
        std::vector<Tri> t = triangles(tris);
        GpuTopoEdit e = topoEdit(deleted, moved, inserted, bvh.primCount,
                                 static_cast<long long>(t.size()));
        addChangedSurvivors(tris_, t, e);
        Scene view;
        view.tris = t;
        view.updateBounds();
        {
            py::gil_scoped_release r;
            updateBVHGPU(bvh, view, e, &topoTimings);
        }
        wideBuilt = bvh.d_wideNodes != nullptr;
        tris_ = std::move(t);
        indices_.clear();
        scene_ = std::move(view);
        bounds = scene_.bounds;
        refitMs = topoTimings.refitMs;
        return topoDict(topoTimings);
    }

private:
    void build() {
        scene_.tris = tris_;
        scene_.updateBounds();
        bounds = scene_.bounds;
        {
            py::gil_scoped_release r;
            bvh = sah == 2 ? buildBVHSah4GPU(scene_, &timings)
                  : sah ? buildBVHSahGPU(scene_, &timings) : buildBVHGPU(scene_, &timings);
        }
        buildMs = timings.totalMs;
    }

    void update(std::vector<Tri> t, const py::object& dirty) {
        if (static_cast<int>(t.size()) != bvh.primCount)
            throw std::invalid_argument("update must keep the triangle count; rebuild instead");
        const bool partial = !dirty.is_none();
        const std::vector<int> ids = dirtyIds(dirty);
        tris_ = std::move(t);
        scene_.tris = tris_;
        scene_.updateBounds();
        bounds = scene_.bounds;
        py::gil_scoped_release r;
        refitMs = partial ? refitBVHGPU(bvh, scene_, ids, &refitTimings)
                          : refitBVHGPU(bvh, scene_, &refitTimings);
    }

    std::vector<Tri> tris_;
    std::vector<int32_t> indices_;
    Scene scene_;
};

class PyPointCloud : public Base {
public:
    PyPointCloud(const F32& points, const std::string& builder) {
        leaf = Leaf::Point;
        sah = sahBuilder(builder);
        std::vector<Vec3> p = points3(points, "points");
        if (p.size() < 2) throw std::invalid_argument("at least 2 points are required");
        cloud_.pts = std::move(p);
        cloud_.updateBounds();
        bounds = cloud_.bounds;
        py::gil_scoped_release r;
        bvh = sah == 2 ? buildPointBVHSah4GPU(cloud_, &timings)
              : sah ? buildPointBVHSahGPU(cloud_, &timings) : buildPointBVHGPU(cloud_, &timings);
        buildMs = timings.totalMs;
    }

    int pointCount() const { return bvh.primCount; }
    std::string validate() const {
        py::gil_scoped_release r;
        return validatePointBVHGPU(bvh, cloud_);
    }

    void updatePoints(const F32& points, const py::object& dirty) {
        std::vector<Vec3> p = points3(points, "points");
        if (static_cast<int>(p.size()) != bvh.primCount)
            throw std::invalid_argument("update must keep the point count; rebuild instead");
        const bool partial = !dirty.is_none();
        const std::vector<int> ids = dirtyIds(dirty);
        cloud_.pts = std::move(p);
        cloud_.updateBounds();
        bounds = cloud_.bounds;
        py::gil_scoped_release r;
        refitMs = partial ? refitPointBVHGPU(bvh, cloud_, ids, &refitTimings)
                          : refitPointBVHGPU(bvh, cloud_, &refitTimings);
    }

    py::dict updateTopology(const F32& points, const py::object& deleted, const py::object& moved,
                            const py::object& inserted) {
        std::vector<Vec3> p = points3(points, "points");
        GpuTopoEdit e = topoEdit(deleted, moved, inserted, bvh.primCount,
                                 static_cast<long long>(p.size()));
        addChangedSurvivors(cloud_.pts, p, e);
        PointCloud view;
        view.pts = std::move(p);
        view.updateBounds();
        {
            py::gil_scoped_release r;
            updatePointBVHGPU(bvh, view, e, &topoTimings);
        }
        wideBuilt = bvh.d_wideNodes != nullptr;
        cloud_ = std::move(view);
        bounds = cloud_.bounds;
        refitMs = topoTimings.refitMs;
        return topoDict(topoTimings);
    }

private:
    PointCloud cloud_;
};

class PyGaussianCloud : public Base {
public:
    PyGaussianCloud(const F32& means, const F32& rot, const F32& scale, const std::string& builder) {
        leaf = Leaf::Gauss;
        sah = sahBuilder(builder);
        std::vector<Gaussian> g = gaussians(means, rot, scale);
        if (g.size() < 2) throw std::invalid_argument("at least 2 gaussians required");
        cloud_.gaussians = std::move(g);
        cloud_.updateBounds();
        bounds = cloud_.bounds;
        py::gil_scoped_release r;
        bvh = sah == 2 ? buildGaussianBVHSah4GPU(cloud_, &timings)
              : sah ? buildGaussianBVHSahGPU(cloud_, &timings) : buildGaussianBVHGPU(cloud_, &timings);
        buildMs = timings.totalMs;
    }

    int gaussianCount() const { return bvh.primCount; }
    std::string validate() const {
        py::gil_scoped_release r;
        return validateGaussianBVHGPU(bvh, cloud_);
    }

    void update(const F32& means, const F32& rot, const F32& scale, const py::object& dirty) {
        std::vector<Gaussian> g = gaussians(means, rot, scale);
        if (static_cast<int>(g.size()) != bvh.primCount)
            throw std::invalid_argument("update must keep the gaussian count; rebuild instead");
        const bool partial = !dirty.is_none();
        const std::vector<int> ids = dirtyIds(dirty);
        cloud_.gaussians = std::move(g);
        cloud_.updateBounds();
        bounds = cloud_.bounds;
        py::gil_scoped_release r;
        refitMs = partial ? refitGaussianBVHGPU(bvh, cloud_, ids, &refitTimings)
                          : refitGaussianBVHGPU(bvh, cloud_, &refitTimings);
    }

    py::dict updateTopology(const F32& means, const F32& rot, const F32& scale,
                            const py::object& deleted, const py::object& moved,
                            const py::object& inserted) {
        std::vector<Gaussian> g = gaussians(means, rot, scale);
        GpuTopoEdit e = topoEdit(deleted, moved, inserted, bvh.primCount,
                                 static_cast<long long>(g.size()));
        addChangedSurvivors(cloud_.gaussians, g, e);
        GaussianCloud view;
        view.gaussians = std::move(g);
        view.updateBounds();
        {
            py::gil_scoped_release r;
            updateGaussianBVHGPU(bvh, view, e, &topoTimings);
        }
        wideBuilt = bvh.d_wideNodes != nullptr;
        cloud_ = std::move(view);
        bounds = cloud_.bounds;
        refitMs = topoTimings.refitMs;
        return topoDict(topoTimings);
    }

private:
    GaussianCloud cloud_;
};

py::tuple demoMesh(const std::string& kind, int grid, int randomTris, uint64_t seed, int buildings) {
    SceneSpec spec;
    spec.kind = kind;
    spec.grid = grid;
    spec.randomTris = randomTris;
    spec.seed = seed;
    spec.buildings = buildings;
    const Scene s = buildScene(spec);
    const py::ssize_t m = static_cast<py::ssize_t>(s.tris.size());
    py::array_t<float> v({m * 3, static_cast<py::ssize_t>(3)});
    py::array_t<int32_t> idx({m, static_cast<py::ssize_t>(3)});
    if (m > 0) std::memcpy(v.mutable_data(), s.tris.data(), s.tris.size() * sizeof(Tri));
    int32_t* pi = idx.mutable_data();
    for (py::ssize_t i = 0; i < 3 * m; ++i) pi[i] = static_cast<int32_t>(i);
    return py::make_tuple(v, idx);
}

py::tuple demoGaussians(const std::string& kind, int count, uint64_t seed) {
    GaussianCloudSpec spec;
    spec.kind = kind;
    spec.count = count;
    spec.seed = seed;
    const GaussianCloud c = buildGaussianCloud(spec);
    const py::ssize_t n = static_cast<py::ssize_t>(c.gaussians.size());
    py::array_t<float> means({n, static_cast<py::ssize_t>(3)});
    py::array_t<float> rot({n, static_cast<py::ssize_t>(4)});
    py::array_t<float> scale({n, static_cast<py::ssize_t>(3)});
    for (py::ssize_t i = 0; i < n; ++i) {
        const Gaussian& g = c.gaussians[static_cast<size_t>(i)];
        std::memcpy(means.mutable_data() + 3 * i, &g.mean, 12);
        std::memcpy(rot.mutable_data() + 4 * i, &g.rot, 16);
        std::memcpy(scale.mutable_data() + 3 * i, &g.scale, 12);
    }
    return py::make_tuple(means, rot, scale);
}

template <class C>
void commonProps(py::class_<C>& c) {
    c.def_property_readonly("node_count", [](const C& s) { return s.bvh.nodeCount; })
        .def_property_readonly("depth", [](const C& s) { return s.bvh.depth; })
        .def_property_readonly("build_ms", [](const C& s) { return s.buildMs; })
        .def_property_readonly("last_query_ms", [](const C& s) { return s.lastQueryMs; },
                               "Device time of the most recent query (CUDA events, no copies)")
        .def_property_readonly("refit_ms", [](const C& s) { return s.refitMs; })
        .def_property_readonly("refit_stats", [](const C& s) { return s.refitStats(); })
        .def_property_readonly("bounds", [](const C& s) { return boundsDict(s.bounds); })
        .def_property_readonly("build_stats", [](const C& s) { return s.buildStats(); })
        .def("validate", &C::validate, "Check tree invariants; empty string means pass")
        .def("_tree_view",
             [](C& s, bool wide) {
                 s.ensureWide(wide);
                 const qk_tree* t = gpuTreeView(s.bvh);
                 auto u = [](const void* p) { return reinterpret_cast<uintptr_t>(p); };
                 return py::make_tuple(t->kind, t->n, t->depth, t->wide_count, u(t->nodes),
                                       u(t->items), u(t->prim_ids), u(t->parent), u(t->depth_arr),
                                       u(t->bnodes), u(t->leaves), u(t->slot_of), u(t->flags),
                                       u(t->wide), u(t->wide_id));
             },
             py::arg("wide") = false,
             "Device arrays of the tree (C ABI qk_tree fields) for the zero-copy CUDA path")
        .def("closest", &C::closest, py::arg("points"), py::arg("order") = "input",
             py::arg("wide") = false,
             "Return (dist2 float32[N], index int32[N]); index is -1 on a miss")
        .def("knn", &C::knn, py::arg("points"), py::arg("k"), py::arg("order") = "input",
             py::arg("wide") = false,
             "Return (dist2 float32[N,k], index int32[N,k]) sorted by (dist2, index); missing "
             "slots are -1")
        .def("radius", &C::radius, py::arg("points"), py::arg("radius"),
             py::arg("order") = "input", py::arg("wide") = false,
             "Return CSR (offsets int64[N+1], dist2 float32[total], index int32[total]) sorted "
             "by (dist2, index) inside each segment");
}

}  // namespace

PYBIND11_MODULE(_quarry, m) {
    m.doc() = "GPU spatial queries on B200: LBVH / SAH build, ray casting, closest / kNN / radius";
    m.attr("__version__") = "1.1.0-b200";
    m.def("describe", []() {
        std::string why;
        return gpuDescribe(&why) ? why : std::string();
    });
    m.def("demo_mesh", &demoMesh, py::arg("kind") = "terrain", py::arg("grid") = 64,
          py::arg("random_tris") = 0, py::arg("seed") = 1, py::arg("buildings") = 65536,
          "Return (vertices (N,3) float32, indices (M,3) int32) for a demo scene");
    m.def("demo_gaussians", &demoGaussians, py::arg("kind") = "sheet", py::arg("count") = 131072,
          py::arg("seed") = 1,
          "Return (means (N,3), rot (N,4) xyzw, scales (N,3)) for a demo gaussian cloud");

    py::class_<PyScene> scene(m, "Scene", "Static triangle mesh with a GPU BVH");
    scene.def(py::init<const F32&, const std::string&>(), py::arg("triangles"),
              py::arg("builder") = "lbvh")
        .def(py::init<const F32&, const I32&, const std::string&>(), py::arg("vertices"),
             py::arg("indices"), py::arg("builder") = "lbvh")
        .def_property_readonly("triangle_count", &PyScene::triangleCount)
        .def("update_triangles", &PyScene::updateTriangles, py::arg("triangles"),
             py::arg("dirty") = py::none())
        .def("update_vertices", &PyScene::updateVertices, py::arg("vertices"),
             py::arg("dirty") = py::none())
        .def("update_topology", &PyScene::updateTopology, py::arg("triangles"),
             py::arg("deleted") = py::none(), py::arg("moved") = py::none(),
             py::arg("inserted") = py::none())
        .def("raycast", &PyScene::raycast, py::arg("origins"), py::arg("dirs"),
             py::arg("tmax") = std::numeric_limits<float>::infinity(),
             py::arg("order") = "input", py::arg("wide") = false,
             "Return (hit bool[N], t float32[N]); t is inf on a miss");
    commonProps(scene);

    py::class_<PyPointCloud> cloud(m, "PointCloud", "Static point cloud with a GPU BVH");
    cloud.def(py::init<const F32&, const std::string&>(), py::arg("points"),
              py::arg("builder") = "lbvh")
        .def_property_readonly("point_count", &PyPointCloud::pointCount)
        .def("update_points", &PyPointCloud::updatePoints, py::arg("points"),
             py::arg("dirty") = py::none())
        .def("update_topology", &PyPointCloud::updateTopology, py::arg("points"),
             py::arg("deleted") = py::none(), py::arg("moved") = py::none(),
             py::arg("inserted") = py::none());
    commonProps(cloud);

    py::class_<PyGaussianCloud> gc(m, "GaussianCloud",
                                   "Static gaussian cloud; queries see the solid ellipsoid");
    gc.def(py::init<const F32&, const F32&, const F32&, const std::string&>(), py::arg("means"),
           py::arg("rot"), py::arg("scale"), py::arg("builder") = "lbvh")
        .def_property_readonly("gaussian_count", &PyGaussianCloud::gaussianCount)
        .def("update", &PyGaussianCloud::update, py::arg("means"), py::arg("rot"),
             py::arg("scale"), py::arg("dirty") = py::none())
        .def("update_topology", &PyGaussianCloud::updateTopology, py::arg("means"),
             py::arg("rot"), py::arg("scale"), py::arg("deleted") = py::none(),
             py::arg("moved") = py::none(), py::arg("inserted") = py::none());
    commonProps(gc);
}
