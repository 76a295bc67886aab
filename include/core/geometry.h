// core/geometry.h -- value types of quarry's API (src/core/geometry.h:27-108, 178-193 of the
// reference): the same names, members and layouts, so callers of the C++ API compile
// unchanged.  The leaf tests themselves live in the engine's device code and in the oracle.
#pragma once

#include <cmath>
#include <limits>

struct Vec3 {
    float x = 0.0f, y = 0.0f, z = 0.0f;
};

inline Vec3 operator+(const Vec3& a, const Vec3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator-(const Vec3& a, const Vec3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator*(const Vec3& a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(const Vec3& a, const Vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec3 cross(const Vec3& a, const Vec3& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length(const Vec3& a) { return std::sqrt(dot(a, a)); }
inline Vec3 normalize(const Vec3& a) {
    const float l = length(a);
    return l > 0.0f ? a * (1.0f / l) : Vec3{};
}

// Axis-aligned box; extend() keeps the reference's "p < mn ? p : mn" rule.
struct AABB {
    Vec3 mn{std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity(),
            std::numeric_limits<float>::infinity()};
    Vec3 mx{-std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity(),
            -std::numeric_limits<float>::infinity()};

    void extend(const Vec3& p) {
        mn.x = p.x < mn.x ? p.x : mn.x;
        mn.y = p.y < mn.y ? p.y : mn.y;
        mn.z = p.z < mn.z ? p.z : mn.z;
        mx.x = p.x > mx.x ? p.x : mx.x;
        mx.y = p.y > mx.y ? p.y : mx.y;
        mx.z = p.z > mx.z ? p.z : mx.z;
    }
    void extend(const AABB& b) {
        if (!b.valid()) return;
        extend(b.mn);
        extend(b.mx);
    }
    bool valid() const { return mn.x <= mx.x && mn.y <= mx.y && mn.z <= mx.z; }
    Vec3 center() const { return (mn + mx) * 0.5f; }
    Vec3 extent() const { return mx - mn; }
    float surfaceArea() const {
        if (!valid()) return 0.0f;
        const Vec3 d = mx - mn;
        return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
    }
};

// 32 bytes: origin, direction (not necessarily unit), t range.
struct Ray {
    Vec3 origin;
    Vec3 dir;
    float tMin = 1e-6f;
    float tMax = std::numeric_limits<float>::infinity();
};

struct Tri {
    Vec3 a, b, c;
    AABB bounds() const {
        AABB box;
        box.extend(a);
        box.extend(b);
        box.extend(c);
        return box;
    }
};

struct RayHit {
    bool hit = false;
    float t = 0.0f;
    int triangle = -1;
};

struct ClosestHit {
    bool found = false;
    float dist2 = std::numeric_limits<float>::max();
    int triangle = -1;
    Vec3 point;
    float bary1 = 0.0f;
    float bary2 = 0.0f;
};

// (dist2, index) lexicographic order of every query result
inline bool closerHit(const ClosestHit& a, const ClosestHit& b) {
    return a.dist2 < b.dist2 || (a.dist2 == b.dist2 && a.triangle < b.triangle);
}
