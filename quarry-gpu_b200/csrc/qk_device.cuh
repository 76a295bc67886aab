// qk_device.cuh -- device-side arithmetic and memory layouts of the B200 spatial-query engine.
//
// Bit-exactness contract: every function here evaluates the same IEEE-754 float operations,
// in the same order, as quarry's reference leaf tests (src/core/geometry.h,
// src/core/gaussian.h), with fmaf exactly where the reference writes QUARRY_FMA.  The
// library is compiled with --fmad=false and without fast-math, so no contraction, IEEE
// division and IEEE sqrt.  Hoisting a per-ray reciprocal 1/d out of the traversal loop is
// allowed because 1/d is the same correctly rounded value every time it is recomputed.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace qk {

constexpr int kTri = 0;
constexpr int kPoint = 1;
constexpr int kGauss = 2;

constexpr float kInf = __builtin_huge_valf();
constexpr float kMarginMul = 1.0f + 1e-6f;  // intersectAABB prune margin (geometry.h:284)
constexpr float kMarginAdd = 1e-6f;
constexpr int kEmptySlot = (-2147483647 - 1);  // empty 4-wide slot (gpu_node.h:46)

// ---------------------------------------------------------------------------------------
// memory layouts
// ---------------------------------------------------------------------------------------
// Canonical node (32 B): the API's GpuBVHNode.  Internal nodes 0..n-2, leaf of slot s at
// n-1+s with left = -(s+1), right = 1 (src/gpu/gpu_node.h:9-14).
struct Node {
    float mn[3];
    float mx[3];
    int left;
    int right;
};
static_assert(sizeof(Node) == 32, "node is 32 bytes");

// Traversal node (64 B, one per internal node, four 16-byte vector loads): both child boxes
// inline so one fetch decides both children.  Child reference >= 0 is an internal node,
// < 0 is ~slot of a leaf (the same -(slot+1) code the canonical leaves use).
//   v0 = L.mn.x L.mn.y L.mn.z L.mx.x
//   v1 = L.mx.y L.mx.z R.mn.x R.mn.y
//   v2 = R.mn.z R.mx.x R.mx.y R.mx.z
//   v3 = left   right  lsmall rsmall
// lsmall / rsmall: 0, or (first slot << 2) | (leaves - 1) when that child's subtree holds 2..4
// leaves on contiguous slots (written by the bottom-up pass, kept by refits).
struct alignas(64) BNode {
    float4 v0, v1, v2, v3;
};
static_assert(sizeof(BNode) == 64, "traversal node is 64 bytes");

// 4-wide node (128 B): the API's GpuBVH4Node (src/gpu/gpu_node.h:48-57).
struct WideEntry {
    float mn[3];
    float mx[3];
    int child;
    int pad;
};
struct alignas(128) WideNode {
    WideEntry c[4];
};
static_assert(sizeof(WideNode) == 128, "wide node is 128 bytes");

struct Box {
    float3 lo, hi;
};

// ---------------------------------------------------------------------------------------
// small vector helpers: one rounding per operation, evaluated left to right
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 mul3(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// union of two boxes as the reference's refit writes it: l < r ? l : r (lbvh.cu:504-509)
__device__ __forceinline__ float fmin_t(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmax_t(float a, float b) { return a > b ? a : b; }
// AABB::extend(p) (geometry.h:57-64): p < cur ? p : cur -- differs from fmin_t on +0/-0 ties
__device__ __forceinline__ float ext_min(float cur, float p) { return p < cur ? p : cur; }
__device__ __forceinline__ float ext_max(float cur, float p) { return p > cur ? p : cur; }

// ---------------------------------------------------------------------------------------
// rays
// ---------------------------------------------------------------------------------------
// Ray prepared once per thread: origin, direction, per-axis reciprocal and "parallel" mask
// (|d| < 1e-20 takes the containment branch of the slab test, geometry.h:292-295).
struct RayPre {
    float3 o, d, inv;
    float tmin, tmax;
    bool px, py, pz;
    int mode;  // tmin / tmax not NaN: the parallel-axis mask px | py << 1 | pz << 2; else -1
};

__device__ __forceinline__ RayPre prepare_ray(float4 r0, float4 r1) {
    RayPre r;
    r.o = f3(r0.x, r0.y, r0.z);
    r.d = f3(r0.w, r1.x, r1.y);
    r.tmin = r1.z;
    r.tmax = r1.w;
    r.px = fabsf(r.d.x) < 1e-20f;
    r.py = fabsf(r.d.y) < 1e-20f;
    r.pz = fabsf(r.d.z) < 1e-20f;
    r.inv = f3(r.px ? 0.0f : 1.0f / r.d.x, r.py ? 0.0f : 1.0f / r.d.y, r.pz ? 0.0f : 1.0f / r.d.z);
    r.mode = (r.tmin == r.tmin && r.tmax == r.tmax)
                 ? (static_cast<int>(r.px) | static_cast<int>(r.py) << 1 | static_cast<int>(r.pz) << 2)
                 : -1;
    return r;
}

// kMode: -1 for any ray (the reference's branch on `par`), else the ray's RayPre::mode known
// at compile time: tmin / tmax are not NaN and bit kAxis says whether this axis is parallel.
// Then the branch is compiled out, and t0 / t1, which start at tmin / bound, are never NaN, so
// `x > t0 ? x : t0` is fmaxf(t0, x) and `x < t1 ? x : t1` is fminf(t1, x) for every x, NaN
// included (both keep t0 / t1); a zero's sign may differ, which no later comparison sees.
// The swap keeps its compare: with a NaN slab end it must not reorder.
template <int kMode = -1, int kAxis = 0>
__device__ __forceinline__ void slab_axis(bool par, float o, float inv, float lo, float hi,
                                          float& t0, float& t1, bool& ok) {
    if (kMode >= 0 && ((kMode >> kAxis) & 1)) {
        ok = ok && !(o < lo || o > hi);
    } else if (kMode >= 0) {
        const float ta = (lo - o) * inv;
        const float tb = (hi - o) * inv;
        const bool sw = ta > tb;
        t0 = fmaxf(t0, sw ? tb : ta);
        t1 = fminf(t1, sw ? ta : tb);
    } else if (par) {
        ok = ok && !(o < lo || o > hi);
    } else {
        float ta = (lo - o) * inv;
        float tb = (hi - o) * inv;
        if (ta > tb) {
            const float s = ta;
            ta = tb;
            tb = s;
        }
        t0 = ta > t0 ? ta : t0;
        t1 = tb < t1 ? tb : t1;
    }
}

// intersectAABB (geometry.h:282-316) with t1 seeded by bound = tMax*(1+1e-6)+1e-6.  The
// reference's per-axis early exit tests a condition that can only get worse on later axes
// (t0 grows, t1 shrinks), so one test after all three axes gives the same answer.
template <int kMode = -1>
__device__ __forceinline__ bool ray_box(const RayPre& r, float3 lo, float3 hi, float bound,
                                        float& tenter) {
    float t0 = r.tmin, t1 = bound;
    bool ok = true;
    slab_axis<kMode, 0>(r.px, r.o.x, r.inv.x, lo.x, hi.x, t0, t1, ok);
    slab_axis<kMode, 1>(r.py, r.o.y, r.inv.y, lo.y, hi.y, t0, t1, ok);
    slab_axis<kMode, 2>(r.pz, r.o.z, r.inv.z, lo.z, hi.z, t0, t1, ok);
    tenter = t0;
    return ok && !(t0 > t1 * kMarginMul + kMarginAdd);
}

// hitParamInsideBox (geometry.h:112-143)
template <int kMode = -1>
__device__ __forceinline__ bool hit_inside_box(const RayPre& r, float3 lo, float3 hi, float t) {
    float t0 = r.tmin, t1 = kInf;
    bool ok = true;
    slab_axis<kMode, 0>(r.px, r.o.x, r.inv.x, lo.x, hi.x, t0, t1, ok);
    slab_axis<kMode, 1>(r.py, r.o.y, r.inv.y, lo.y, hi.y, t0, t1, ok);
    slab_axis<kMode, 2>(r.pz, r.o.z, r.inv.z, lo.z, hi.z, t0, t1, ok);
    if (!ok || t0 > t1) return false;
    return t >= t0 * (1.0f - 1e-6f) - 1e-6f && t <= t1 * (1.0f + 1e-6f) + 1e-6f;
}

// Moller-Trumbore with the self-box guard (geometry.h:146-176); tMax is the ray's own.
template <int kMode = -1>
__device__ __forceinline__ bool ray_tri(const RayPre& r, float3 a, float3 b, float3 c, float& tout) {
    const float3 e1 = sub3(b, a);
    const float3 e2 = sub3(c, a);
    const float3 p = cross3(r.d, e2);
    const float det = dot3(e1, p);
    if (fabsf(det) < 1e-7f) return false;
    const float inv = 1.0f / det;
    const float3 tv = sub3(r.o, a);
    const float u = dot3(tv, p) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    const float3 q = cross3(tv, e1);
    const float v = dot3(r.d, q) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    const float t = dot3(e2, q) * inv;
    if (t < r.tmin || t > r.tmax) return false;
    // Tri::bounds: extend(a), extend(b), extend(c) from an empty box (geometry.h:94-100)
    const float3 lo = f3(ext_min(ext_min(a.x, b.x), c.x), ext_min(ext_min(a.y, b.y), c.y),
                         ext_min(ext_min(a.z, b.z), c.z));
    const float3 hi = f3(ext_max(ext_max(a.x, b.x), c.x), ext_max(ext_max(a.y, b.y), c.y),
                         ext_max(ext_max(a.z, b.z), c.z));
    if (!hit_inside_box<kMode>(r, lo, hi, t)) return false;
    tout = t;
    return true;
}

// ---------------------------------------------------------------------------------------
// point queries
// ---------------------------------------------------------------------------------------
// distanceSquaredToAABB (geometry.h:262-277)
// Branch-free, with the reference's values: per axis the gap is lo - p below the box, p - hi
// above it, else 0 (max(max(lo - p, p - hi), 0): below the box p - hi < 0 < lo - p, above it
// the reverse, inside both <= 0; a NaN end or coordinate leaves the other operand, as the
// reference's comparisons do), and adding the square of a zero gap to the running sum (never
// negative) changes nothing, so skipping it and adding it give the same bits.
__device__ __forceinline__ float dist2_axis(float p, float lo, float hi) {
    const float d = fmaxf(fmaxf(lo - p, p - hi), 0.0f);
    return d * d;
}

__device__ __forceinline__ float dist2_box(float3 p, float3 lo, float3 hi) {
    float d2 = 0.0f;
    d2 += dist2_axis(p.x, lo.x, hi.x);
    d2 += dist2_axis(p.y, lo.y, hi.y);
    d2 += dist2_axis(p.z, lo.z, hi.z);
    return d2;
}

__device__ __forceinline__ float d2_pts(float3 p, float3 q) {
    const float3 d = sub3(p, q);
    return dot3(d, d);
}

// closestPointOnTriangle, squared distance only (geometry.h:198-259)
__device__ __forceinline__ float closest_tri_d2(float3 p, float3 a, float3 b, float3 c) {
    const float3 ab = sub3(b, a);
    const float3 ac = sub3(c, a);
    const float3 ap = sub3(p, a);
    const float d1 = dot3(ab, ap);
    const float d2 = dot3(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) return d2_pts(p, a);
    const float3 bp = sub3(p, b);
    const float d3 = dot3(ab, bp);
    const float d4 = dot3(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) return d2_pts(p, b);
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float t = d1 / (d1 - d3);
        return d2_pts(p, add3(a, mul3(ab, t)));
    }
    const float3 cp = sub3(p, c);
    const float d5 = dot3(ab, cp);
    const float d6 = dot3(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) return d2_pts(p, c);
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float t = d2 / (d2 - d6);
        return d2_pts(p, add3(a, mul3(ac, t)));
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return d2_pts(p, add3(b, mul3(sub3(c, b), t)));
    }
    const float denom = va + vb + vc;
    if (!(denom > 1e-20f)) {
        float best = d2_pts(p, a);
        const float hb = d2_pts(p, b);
        const float hc = d2_pts(p, c);
        if (hb < best) best = hb;
        if (hc < best) best = hc;
        return best;
    }
    const float b1 = vb / denom;
    const float b2 = vc / denom;
    return d2_pts(p, add3(add3(a, mul3(ab, b1)), mul3(ac, b2)));
}

// gaussianAxes (gaussian.h:23-41)
__device__ __forceinline__ void gauss_axes(float4 q, float3& u, float3& v, float3& w) {
    const float lenSq = fmaf(q.w, q.w, fmaf(q.z, q.z, fmaf(q.y, q.y, q.x * q.x)));
    float inv = 1.0f;
    if (lenSq > 0.0f) inv = 1.0f / sqrtf(lenSq);
    const float qx = q.x * inv, qy = q.y * inv, qz = q.z * inv, qw = q.w * inv;
    const float yyzz = fmaf(qy, qy, qz * qz);
    const float xxzz = fmaf(qx, qx, qz * qz);
    const float xxyy = fmaf(qx, qx, qy * qy);
    u = f3(fmaf(-2.0f, yyzz, 1.0f), 2.0f * fmaf(qx, qy, qz * qw), 2.0f * fmaf(qx, qz, -(qy * qw)));
    v = f3(2.0f * fmaf(qx, qy, -(qz * qw)), fmaf(-2.0f, xxzz, 1.0f), 2.0f * fmaf(qy, qz, qx * qw));
    w = f3(2.0f * fmaf(qx, qz, qy * qw), 2.0f * fmaf(qy, qz, -(qx * qw)), fmaf(-2.0f, xxyy, 1.0f));
}

// gaussianBounds (gaussian.h:46-64)
__device__ __forceinline__ Box gauss_bounds(float3 mean, float4 q, float3 s) {
    float3 u, v, w;
    gauss_axes(q, u, v, w);
    const float a2 = s.x * s.x, b2 = s.y * s.y, c2 = s.z * s.z;
    const float hx = sqrtf(fmaf(c2, w.x * w.x, fmaf(b2, v.x * v.x, a2 * u.x * u.x)));
    const float hy = sqrtf(fmaf(c2, w.y * w.y, fmaf(b2, v.y * v.y, a2 * u.y * u.y)));
    const float hz = sqrtf(fmaf(c2, w.z * w.z, fmaf(b2, v.z * v.z, a2 * u.z * u.z)));
    const float px = hx + 1e-6f * (1.0f + fabsf(mean.x) + hx);
    const float py = hy + 1e-6f * (1.0f + fabsf(mean.y) + hy);
    const float pz = hz + 1e-6f * (1.0f + fabsf(mean.z) + hz);
    Box b;
    b.lo = f3(mean.x - px, mean.y - py, mean.z - pz);
    b.hi = f3(mean.x + px, mean.y + py, mean.z + pz);
    return b;
}

// gaussianDist2 (gaussian.h:80-131): exact distance to the solid ellipsoid, 14 bracketed
// Newton / bisection steps on Eberly's secular equation, no early exit.
__device__ __forceinline__ float gauss_d2(float3 p, float3 mean, float4 q, float3 s) {
    float3 u, v, w;
    gauss_axes(q, u, v, w);
    const float3 d = sub3(p, mean);
    const float y0 = dot3(d, u), y1 = dot3(d, v), y2 = dot3(d, w);
    const float a = s.x, b = s.y, c = s.z;
    const float aa = a * a, bb = b * b, cc = c * c;
    const float gy0 = a * y0, gy1 = b * y1, gy2 = c * y2;
    {
        const float r0 = y0 / a, r1 = y1 / b, r2 = y2 / c;
        if (fmaf(r2, r2, fmaf(r1, r1, r0 * r0)) <= 1.0f) return 0.0f;
    }
    const float lenSq = fmaf(y2, y2, fmaf(y1, y1, y0 * y0));
    const float len = sqrtf(lenSq);
    const float amax = a > b ? (a > c ? a : c) : (b > c ? b : c);
    float lo = 0.0f;
    float hi = 2.0f * amax * len;
    float t = 0.0f;
    if (len > amax) t = amax * (len - amax);
#pragma unroll 2
    for (int iter = 0; iter < 14; ++iter) {
        const float ir0 = 1.0f / (t + aa), ir1 = 1.0f / (t + bb), ir2 = 1.0f / (t + cc);
        const float s0 = gy0 * ir0, s1 = gy1 * ir1, s2 = gy2 * ir2;
        const float f = fmaf(s2, s2, fmaf(s1, s1, s0 * s0)) - 1.0f;
        if (f > 0.0f) lo = t; else hi = t;
        const float fp = -2.0f * (s0 * s0 * ir0 + s1 * s1 * ir1 + s2 * s2 * ir2);
        float next = 0.5f * (lo + hi);
        if (fp < 0.0f) {
            const float newton = t - f / fp;
            if (newton > lo && newton < hi) next = newton;
        }
        t = next;
    }
    const float ir0 = 1.0f / (t + aa), ir1 = 1.0f / (t + bb), ir2 = 1.0f / (t + cc);
    const float e0 = y0 - gy0 * ir0 * a;
    const float e1 = y1 - gy1 * ir1 * b;
    const float e2 = y2 - gy2 * ir2 * c;
    return fmaf(e2, e2, fmaf(e1, e1, e0 * e0));
}

// ---------------------------------------------------------------------------------------
// primitive traits.  Scene-order items use the API layouts (Tri 36 B, Vec3 12 B,
// Gaussian 40 B); traversal reads leaf payloads of 16-byte vectors in leaf order:
//   triangle  {a.xyz, id} {b.xyz, 0} {c.xyz, 0}
//   point     {p.xyz, id}
//   gaussian  {mean.xyz, id} {quat.xyzw} {scale.xyz, 0}
// ---------------------------------------------------------------------------------------
struct TriOps {
    static constexpr int kFloats = 9;
    static constexpr int kVec4 = 3;
    __device__ static Box bounds(const float* it) {
        Box b;
        b.lo = f3(ext_min(ext_min(it[0], it[3]), it[6]), ext_min(ext_min(it[1], it[4]), it[7]),
                  ext_min(ext_min(it[2], it[5]), it[8]));
        b.hi = f3(ext_max(ext_max(it[0], it[3]), it[6]), ext_max(ext_max(it[1], it[4]), it[7]),
                  ext_max(ext_max(it[2], it[5]), it[8]));
        return b;
    }
    // prim_ops.h:80-83: sum then divide, per axis
    __device__ static float3 centroid(const float* it) {
        return f3((it[0] + it[3] + it[6]) / 3.0f, (it[1] + it[4] + it[7]) / 3.0f,
                  (it[2] + it[5] + it[8]) / 3.0f);
    }
    __device__ static void pack(const float* it, int id, float4* out) {
        out[0] = make_float4(it[0], it[1], it[2], __int_as_float(id));
        out[1] = make_float4(it[3], it[4], it[5], 0.0f);
        out[2] = make_float4(it[6], it[7], it[8], 0.0f);
    }
    __device__ static float dist2(float3 p, const float4* __restrict__ leaf, int slot, int& id) {
        const float4 a = __ldg(leaf + 3 * slot), b = __ldg(leaf + 3 * slot + 1),
                     c = __ldg(leaf + 3 * slot + 2);
        id = __float_as_int(a.w);
        return closest_tri_d2(p, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), f3(c.x, c.y, c.z));
    }
};

struct PointOps {
    static constexpr int kFloats = 3;
    static constexpr int kVec4 = 1;
    // AABB{}.extend(p): mn = p < inf ? p : inf = p (prim_ops.h:93-97)
    __device__ static Box bounds(const float* it) {
        Box b;
        b.lo = f3(it[0], it[1], it[2]);
        b.hi = b.lo;
        return b;
    }
    __device__ static float3 centroid(const float* it) { return f3(it[0], it[1], it[2]); }
    __device__ static void pack(const float* it, int id, float4* out) {
        out[0] = make_float4(it[0], it[1], it[2], __int_as_float(id));
    }
    __device__ static float dist2(float3 p, const float4* __restrict__ leaf, int slot, int& id) {
        const float4 a = __ldg(leaf + slot);
        id = __float_as_int(a.w);
        return d2_pts(p, f3(a.x, a.y, a.z));
    }
};

struct GaussOps {
    static constexpr int kFloats = 10;
    static constexpr int kVec4 = 3;
    __device__ static Box bounds(const float* it) {
        return gauss_bounds(f3(it[0], it[1], it[2]), make_float4(it[3], it[4], it[5], it[6]),
                            f3(it[7], it[8], it[9]));
    }
    __device__ static float3 centroid(const float* it) { return f3(it[0], it[1], it[2]); }
    __device__ static void pack(const float* it, int id, float4* out) {
        out[0] = make_float4(it[0], it[1], it[2], __int_as_float(id));
        out[1] = make_float4(it[3], it[4], it[5], it[6]);
        out[2] = make_float4(it[7], it[8], it[9], 0.0f);
    }
    __device__ static float dist2(float3 p, const float4* __restrict__ leaf, int slot, int& id) {
        const float4 a = __ldg(leaf + 3 * slot), q = __ldg(leaf + 3 * slot + 1),
                     s = __ldg(leaf + 3 * slot + 2);
        id = __float_as_int(a.w);
        return gauss_d2(p, f3(a.x, a.y, a.z), q, f3(s.x, s.y, s.z));
    }
};

// (dist2, id) lexicographic order: closerHit (geometry.h:191-193)
__device__ __forceinline__ bool closer(float da, int ia, float db, int ib) {
    return da < db || (da == db && ia < ib);
}

}  // namespace qk
