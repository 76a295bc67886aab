// ref_shim.cpp -- C entry points over quarry's own CPU reference (its src/core and src/cpu
// sources, compiled unchanged where they lie by oracle/Makefile into oracle/_ref/).
//
// TEST INFRASTRUCTURE ONLY: the checker that pins oracle/quarry_oracle.c and the timed
// CPU baseline of bench.py.  The product never loads it.
//
// Each entry point builds the reference's own acceleration structure for the primitive kind
// (buildBVH for triangles, buildPointKdTree for points, buildGaussBVH for Gaussians; see
// src/cpu/bvh.h:30-43, src/cpu/point_kd.h:225-229, src/cpu/gauss_bvh.h:30-35) and answers
// queries with the matching reference function, fanning queries out over std::thread static
// chunks (the functions keep their scratch thread_local, src/cpu/bvh.cpp:206).
#include <chrono>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "core/fingerprint.h"
#include "core/gaussian.h"
#include "core/geometry.h"
#include "core/point_cloud.h"
#include "core/scene.h"
#include "cpu/brute.h"
#include "cpu/bvh.h"
#include "cpu/gauss_bvh.h"
#include "cpu/point_kd.h"
#include "cpu/selftest.h"

namespace {

template <typename F>
void parallelChunks(int count, int threads, F&& fn) {
    if (threads <= 0) threads = static_cast<int>(std::thread::hardware_concurrency());
    if (threads < 1) threads = 1;
    if (threads == 1 || count < 64) {
        fn(0, count);
        return;
    }
    std::vector<std::thread> pool;
    const int chunk = (count + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const int b = t * chunk;
        const int e = std::min(count, b + chunk);
        if (b >= e) break;
        pool.emplace_back([&fn, b, e]() { fn(b, e); });
    }
    for (auto& th : pool) th.join();
}

Scene sceneFrom(const float* tris9, int n) {
    Scene s;
    s.tris.resize(static_cast<size_t>(n));
    std::memcpy(s.tris.data(), tris9, sizeof(Tri) * static_cast<size_t>(n));
    s.updateBounds();
    return s;
}

PointCloud cloudFrom(const float* p3, int n) {
    PointCloud c;
    c.pts.resize(static_cast<size_t>(n));
    std::memcpy(c.pts.data(), p3, sizeof(Vec3) * static_cast<size_t>(n));
    c.updateBounds();
    return c;
}

GaussianCloud gaussFrom(const float* g10, int n) {
    GaussianCloud c;
    c.gaussians.resize(static_cast<size_t>(n));
    std::memcpy(c.gaussians.data(), g10, sizeof(Gaussian) * static_cast<size_t>(n));
    c.updateBounds();
    return c;
}

uint32_t bitsOf(float f) {
    uint32_t b;
    std::memcpy(&b, &f, sizeof(b));
    return b;
}

void putHit(uint32_t* out2, const ClosestHit& h) {
    out2[0] = h.found ? bitsOf(h.dist2) : 0u;
    out2[1] = static_cast<uint32_t>(h.found ? h.triangle : -1);
}

// One reference structure per kind, built once per call.
struct Index {
    int kind = 0;
    BVH tri;
    PointKdTree pts;
    GaussBVH gs;

    Index(int k, const float* items, int n) : kind(k) {
        if (k == 0) tri = buildBVH(sceneFrom(items, n));
        else if (k == 1) pts = buildPointKdTree(cloudFrom(items, n));
        else gs = buildGaussBVH(gaussFrom(items, n));
    }

    ClosestHit closest(const Vec3& p) const {
        if (kind == 0) return closestPointBVH(tri, p);
        if (kind == 1) return kdClosest(pts, p);
        return closestGaussianBVH(gs, p);
    }
    std::vector<ClosestHit> knn(const Vec3& p, int k) const {
        if (kind == 0) return kNearestBVH(tri, p, k);
        if (kind == 1) return kdKNearest(pts, p, k);
        return kNearestGaussianBVH(gs, p, k);
    }
    std::vector<ClosestHit> radius(const Vec3& p, float r) const {
        if (kind == 0) return radiusBVH(tri, p, r);
        if (kind == 1) return kdRadius(pts, p, r);
        return radiusGaussianBVH(gs, p, r);
    }
};

struct RadiusResult {
    std::vector<std::vector<ClosestHit>> lists;
};

double nowMs() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" {

// reference selftest (src/cpu/selftest.cpp:534-550); returns 1 when every check passes
int qr_selftest(void) { return runSelfTest() ? 1 : 0; }

// ---- leaf tests (src/core/geometry.h, src/core/gaussian.h) ----
int qr_intersect_triangle(const float* ray8, const float* tri9, float* t) {
    Ray r;
    std::memcpy(&r, ray8, sizeof(Ray));
    Tri tri;
    std::memcpy(&tri, tri9, sizeof(Tri));
    return intersectTriangle(r, tri, *t) ? 1 : 0;
}

float qr_closest_point_dist2(const float* p3, const float* tri9) {
    Vec3 p;
    std::memcpy(&p, p3, sizeof(Vec3));
    Tri tri;
    std::memcpy(&tri, tri9, sizeof(Tri));
    return closestPointOnTriangle(p, tri).dist2;
}

float qr_gaussian_dist2(const float* p3, const float* g10) {
    Vec3 p;
    std::memcpy(&p, p3, sizeof(Vec3));
    Gaussian g;
    std::memcpy(&g, g10, sizeof(Gaussian));
    return gaussianDist2(p, g);
}

void qr_gaussian_bounds(const float* g10, float* box6) {
    Gaussian g;
    std::memcpy(&g, g10, sizeof(Gaussian));
    const AABB b = gaussianBounds(g);
    std::memcpy(box6, &b, sizeof(float) * 6);
}

float qr_dist2_aabb(const float* p3, const float* box6) {
    Vec3 p;
    std::memcpy(&p, p3, sizeof(Vec3));
    AABB b;
    std::memcpy(&b, box6, sizeof(float) * 6);
    return distanceSquaredToAABB(p, b);
}

// ---- rays: buildBVH + raycastBVH (src/cpu/bvh.cpp:136-178) ----
// Returns the query time in ms (build excluded); *build_ms gets the build time.
double qr_raycast(const float* tris9, int n, const float* rays8, int nrays, uint64_t* out,
                  int threads, double* build_ms) {
    const double t0 = nowMs();
    const BVH bvh = buildBVH(sceneFrom(tris9, n));
    const double t1 = nowMs();
    parallelChunks(nrays, threads, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            Ray r;
            std::memcpy(&r, rays8 + 8 * static_cast<size_t>(i), sizeof(Ray));
            const RayHit h = raycastBVH(bvh, r);
            out[i] = h.hit ? ((uint64_t{1} << 32) | bitsOf(h.t)) : 0ull;
        }
    });
    const double t2 = nowMs();
    if (build_ms) *build_ms = t1 - t0;
    return t2 - t1;
}

void qr_raycast_brute(const float* tris9, int n, const float* rays8, int nrays, uint64_t* out) {
    const Scene s = sceneFrom(tris9, n);
    for (int i = 0; i < nrays; ++i) {
        Ray r;
        std::memcpy(&r, rays8 + 8 * static_cast<size_t>(i), sizeof(Ray));
        const RayHit h = raycastBrute(s, r);
        out[i] = h.hit ? ((uint64_t{1} << 32) | bitsOf(h.t)) : 0ull;
    }
}

// ---- point queries: kind 0 triangles, 1 points, 2 Gaussians ----
double qr_closest(int kind, const float* items, int n, const float* q3, int nq, uint32_t* out2,
                  int threads, double* build_ms) {
    const double t0 = nowMs();
    const Index idx(kind, items, n);
    const double t1 = nowMs();
    parallelChunks(nq, threads, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            Vec3 p;
            std::memcpy(&p, q3 + 3 * static_cast<size_t>(i), sizeof(Vec3));
            putHit(out2 + 2 * static_cast<size_t>(i), idx.closest(p));
        }
    });
    const double t2 = nowMs();
    if (build_ms) *build_ms = t1 - t0;
    return t2 - t1;
}

double qr_knn(int kind, const float* items, int n, const float* q3, int nq, int k,
              uint32_t* out2, int threads, double* build_ms) {
    const double t0 = nowMs();
    const Index idx(kind, items, n);
    const double t1 = nowMs();
    parallelChunks(nq, threads, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            Vec3 p;
            std::memcpy(&p, q3 + 3 * static_cast<size_t>(i), sizeof(Vec3));
            const std::vector<ClosestHit> list = idx.knn(p, k);
            uint32_t* dst = out2 + 2 * static_cast<size_t>(i) * static_cast<size_t>(k);
            for (int j = 0; j < k; ++j) {
                if (j < static_cast<int>(list.size())) {
                    putHit(dst + 2 * j, list[static_cast<size_t>(j)]);
                } else {
                    dst[2 * j] = 0u;
                    dst[2 * j + 1] = static_cast<uint32_t>(-1);
                }
            }
        }
    });
    const double t2 = nowMs();
    if (build_ms) *build_ms = t1 - t0;
    return t2 - t1;
}

// Radius: returns an opaque handle holding the per-query lists; read it back with
// qr_radius_total / qr_radius_copy and release it with qr_radius_free.
void* qr_radius(int kind, const float* items, int n, const float* q3, int nq, float radius,
                int threads, double* query_ms) {
    auto* res = new RadiusResult;
    res->lists.resize(static_cast<size_t>(nq));
    const Index idx(kind, items, n);
    const double t1 = nowMs();
    parallelChunks(nq, threads, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            Vec3 p;
            std::memcpy(&p, q3 + 3 * static_cast<size_t>(i), sizeof(Vec3));
            res->lists[static_cast<size_t>(i)] = idx.radius(p, radius);
        }
    });
    if (query_ms) *query_ms = nowMs() - t1;
    return res;
}

int64_t qr_radius_total(void* h) {
    int64_t total = 0;
    for (const auto& l : static_cast<RadiusResult*>(h)->lists) total += static_cast<int64_t>(l.size());
    return total;
}

void qr_radius_copy(void* h, int64_t* offsets, uint64_t* keys) {
    const auto& lists = static_cast<RadiusResult*>(h)->lists;
    int64_t at = 0;
    offsets[0] = 0;
    for (size_t i = 0; i < lists.size(); ++i) {
        for (const ClosestHit& c : lists[i]) {
            keys[at++] = (static_cast<uint64_t>(bitsOf(c.dist2)) << 32) |
                         static_cast<uint32_t>(c.triangle);
        }
        offsets[i + 1] = at;
    }
}

void qr_radius_free(void* h) { delete static_cast<RadiusResult*>(h); }

// One scene, every query set: the reference structure is built once (*build_ms) and answers
// nc closest points, nk k-nearest (k per query, padded with id -1), nr radius queries
// (returned as a handle like qr_radius) and, for triangles, nrays rays; each set fans out
// over `threads`.  ms[0..3]: closest, kNN, radius and ray query times.
void* qr_scene(int kind, const float* items, int n, const float* qc, int nc, uint32_t* out_c,
               const float* qk, int nk, int k, uint32_t* out_k, const float* qr, int nr,
               float radius, const float* rays8, int nrays, uint64_t* out_r, int threads,
               double* build_ms, double* ms) {
    const double t0 = nowMs();
    const Index idx(kind, items, n);
    const double t1 = nowMs();
    if (build_ms) *build_ms = t1 - t0;
    parallelChunks(nc, threads, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            Vec3 p;
            std::memcpy(&p, qc + 3 * static_cast<size_t>(i), sizeof(Vec3));
            putHit(out_c + 2 * static_cast<size_t>(i), idx.closest(p));
        }
    });
    const double t2 = nowMs();
    parallelChunks(nk, threads, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            Vec3 p;
            std::memcpy(&p, qk + 3 * static_cast<size_t>(i), sizeof(Vec3));
            const std::vector<ClosestHit> list = idx.knn(p, k);
            uint32_t* dst = out_k + 2 * static_cast<size_t>(i) * static_cast<size_t>(k);
            for (int j = 0; j < k; ++j) {
                if (j < static_cast<int>(list.size())) {
                    putHit(dst + 2 * j, list[static_cast<size_t>(j)]);
                } else {
                    dst[2 * j] = 0u;
                    dst[2 * j + 1] = static_cast<uint32_t>(-1);
                }
            }
        }
    });
    const double t3 = nowMs();
    auto* res = new RadiusResult;
    res->lists.resize(static_cast<size_t>(nr));
    parallelChunks(nr, threads, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            Vec3 p;
            std::memcpy(&p, qr + 3 * static_cast<size_t>(i), sizeof(Vec3));
            res->lists[static_cast<size_t>(i)] = idx.radius(p, radius);
        }
    });
    const double t4 = nowMs();
    if (kind == 0 && nrays > 0) {
        parallelChunks(nrays, threads, [&](int b, int e) {
            for (int i = b; i < e; ++i) {
                Ray r;
                std::memcpy(&r, rays8 + 8 * static_cast<size_t>(i), sizeof(Ray));
                const RayHit h = raycastBVH(idx.tri, r);
                out_r[i] = h.hit ? ((uint64_t{1} << 32) | bitsOf(h.t)) : 0ull;
            }
        });
    }
    const double t5 = nowMs();
    if (ms) {
        ms[0] = t2 - t1;
        ms[1] = t3 - t2;
        ms[2] = t4 - t3;
        ms[3] = t5 - t4;
    }
    return res;
}

// ---- brute force point queries (src/cpu/brute.cpp:62-197) ----
void qr_closest_brute(int kind, const float* items, int n, const float* q3, int nq,
                      uint32_t* out2) {
    Scene s;
    PointCloud pc;
    GaussianCloud gc;
    if (kind == 0) s = sceneFrom(items, n);
    else if (kind == 1) pc = cloudFrom(items, n);
    else gc = gaussFrom(items, n);
    for (int i = 0; i < nq; ++i) {
        Vec3 p;
        std::memcpy(&p, q3 + 3 * static_cast<size_t>(i), sizeof(Vec3));
        const ClosestHit h = kind == 0   ? closestPointBrute(s, p)
                             : kind == 1 ? closestVertexBrute(pc, p)
                                         : closestGaussianBrute(gc, p);
        putHit(out2 + 2 * static_cast<size_t>(i), h);
    }
}

// ---- fingerprints exactly as RayStats / QueryStats fold them (src/core/fingerprint.h) ----
uint64_t qr_ray_hash(const uint64_t* res, int64_t n, uint64_t* hits) {
    RayStats st;
    for (int64_t i = 0; i < n; ++i) {
        RayHit h;
        h.hit = (res[i] >> 32) != 0;
        if (h.hit) {
            const uint32_t bits = static_cast<uint32_t>(res[i]);
            std::memcpy(&h.t, &bits, sizeof(bits));
        }
        st.add(h);
    }
    if (hits) *hits = st.hits;
    return st.hash;
}

uint64_t qr_closest_hash(const uint32_t* res2, int64_t n) {
    QueryStats st;
    for (int64_t i = 0; i < n; ++i) {
        ClosestHit h;
        h.triangle = static_cast<int32_t>(res2[2 * i + 1]);
        h.found = h.triangle >= 0;
        if (h.found) std::memcpy(&h.dist2, &res2[2 * i], sizeof(float));
        st.add(h);
    }
    return st.hash;
}

uint64_t qr_list_hash(const int64_t* offsets, const uint64_t* keys, int64_t n) {
    QueryStats st;
    for (int64_t i = 0; i < n; ++i) {
        std::vector<ClosestHit> list;
        for (int64_t j = offsets[i]; j < offsets[i + 1]; ++j) {
            ClosestHit h;
            h.found = true;
            const uint32_t bits = static_cast<uint32_t>(keys[j] >> 32);
            std::memcpy(&h.dist2, &bits, sizeof(float));
            h.triangle = static_cast<int32_t>(static_cast<uint32_t>(keys[j]));
            list.push_back(h);
        }
        st.add(list);
    }
    return st.hash;
}

}  // extern "C"
