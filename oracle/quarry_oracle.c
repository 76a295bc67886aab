/*
 * quarry_oracle.c -- CPU restatement of quarry's hot path.  TEST INFRASTRUCTURE ONLY:
 * the checker for the CUDA engine, never part of the product (see quarry_oracle.h).
 *
 * Build with -O2 -ffp-contract=off (no -ffast-math): every float operation below
 * must round exactly like the reference's.
 */
#define _GNU_SOURCE
#include "quarry_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------------- */
/* small vector helpers: each expression is evaluated left to right with one   */
/* rounding per operation, as Vec3 in src/core/geometry.h:31-39                */
/* ------------------------------------------------------------------------- */
typedef struct { float x, y, z; } v3;

static inline v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 scl(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float comp(const float* v, int a) { return v[a]; }

int qo_stride(int kind) {
    return kind == QO_TRI ? 9 : kind == QO_POINT ? 3 : kind == QO_GAUSS ? 10 : 0;
}

/* AABB::extend(Vec3) with the reference's ternaries (geometry.h:57-64) */
static inline void box_extend(float* box6, const float* p) {
    for (int a = 0; a < 3; ++a) {
        box6[a] = p[a] < box6[a] ? p[a] : box6[a];
        box6[3 + a] = p[a] > box6[3 + a] ? p[a] : box6[3 + a];
    }
}
static inline void box_empty(float* box6) {
    box6[0] = box6[1] = box6[2] = INFINITY;
    box6[3] = box6[4] = box6[5] = -INFINITY;
}

/* Tri::bounds (geometry.h:94-100) */
static void tri_bounds(const float* t9, float* box6) {
    box_empty(box6);
    box_extend(box6, t9);
    box_extend(box6, t9 + 3);
    box_extend(box6, t9 + 6);
}

/* ------------------------------------------------------------------------- */
/* ray / box / triangle (geometry.h:112-176, 279-316)                          */
/* ------------------------------------------------------------------------- */
int qo_intersect_aabb(const float* ray, const float* box, float tmax, float* tenter) {
    float t0 = ray[6];
    float t1 = tmax * (1.0f + 1e-6f) + 1e-6f;
    for (int a = 0; a < 3; ++a) {
        const float o = ray[a], d = ray[3 + a], lo = box[a], hi = box[3 + a];
        if (fabsf(d) < 1e-20f) {
            if (o < lo || o > hi) return 0;
            continue;
        }
        const float inv = 1.0f / d;
        float ta = (lo - o) * inv;
        float tb = (hi - o) * inv;
        if (ta > tb) { const float s = ta; ta = tb; tb = s; }
        t0 = ta > t0 ? ta : t0;
        t1 = tb < t1 ? tb : t1;
        if (t0 > t1 * (1.0f + 1e-6f) + 1e-6f) return 0;
    }
    *tenter = t0;
    return 1;
}

static int hit_param_inside_box(const float* ray, const float* box, float t) {
    float t0 = ray[6];
    float t1 = INFINITY;
    for (int a = 0; a < 3; ++a) {
        const float o = ray[a], d = ray[3 + a], lo = box[a], hi = box[3 + a];
        if (fabsf(d) < 1e-20f) {
            if (o < lo || o > hi) return 0;
            continue;
        }
        const float inv = 1.0f / d;
        float ta = (lo - o) * inv;
        float tb = (hi - o) * inv;
        if (ta > tb) { const float s = ta; ta = tb; tb = s; }
        t0 = ta > t0 ? ta : t0;
        t1 = tb < t1 ? tb : t1;
        if (t0 > t1) return 0;
    }
    return t >= t0 * (1.0f - 1e-6f) - 1e-6f && t <= t1 * (1.0f + 1e-6f) + 1e-6f;
}

int qo_intersect_triangle(const float* ray, const float* tri, float* tout) {
    const v3 o = ld3(ray), d = ld3(ray + 3);
    const v3 a = ld3(tri), b = ld3(tri + 3), c = ld3(tri + 6);
    const v3 e1 = sub(b, a);
    const v3 e2 = sub(c, a);
    const v3 p = cross(d, e2);
    const float det = dot(e1, p);
    if (fabsf(det) < 1e-7f) return 0;
    const float inv = 1.0f / det;
    const v3 tv = sub(o, a);
    const float u = dot(tv, p) * inv;
    if (u < 0.0f || u > 1.0f) return 0;
    const v3 q = cross(tv, e1);
    const float v = dot(d, q) * inv;
    if (v < 0.0f || u + v > 1.0f) return 0;
    const float t = dot(e2, q) * inv;
    if (t < ray[6] || t > ray[7]) return 0;
    float box[6];
    tri_bounds(tri, box);
    if (!hit_param_inside_box(ray, box, t)) return 0;
    *tout = t;
    return 1;
}

/* closestPointOnTriangle, returning only dist2 (geometry.h:198-259) */
static inline float d2_to(v3 p, v3 q) {
    const v3 d = sub(p, q);
    return dot(d, d);
}

float qo_closest_point_dist2(const float* p3, const float* tri) {
    const v3 p = ld3(p3), a = ld3(tri), b = ld3(tri + 3), c = ld3(tri + 6);
    const v3 ab = sub(b, a);
    const v3 ac = sub(c, a);
    const v3 ap = sub(p, a);
    const float d1 = dot(ab, ap);
    const float d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) return d2_to(p, a);
    const v3 bp = sub(p, b);
    const float d3 = dot(ab, bp);
    const float d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) return d2_to(p, b);
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float t = d1 / (d1 - d3);
        return d2_to(p, add(a, scl(ab, t)));
    }
    const v3 cp = sub(p, c);
    const float d5 = dot(ab, cp);
    const float d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) return d2_to(p, c);
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float t = d2 / (d2 - d6);
        return d2_to(p, add(a, scl(ac, t)));
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return d2_to(p, add(b, scl(sub(c, b), t)));
    }
    const float denom = va + vb + vc;
    if (!(denom > 1e-20f)) {
        float best = d2_to(p, a);
        const float hb = d2_to(p, b);
        const float hc = d2_to(p, c);
        if (hb < best) best = hb;
        if (hc < best) best = hc;
        return best;
    }
    const float b1 = vb / denom;
    const float b2 = vc / denom;
    return d2_to(p, add(add(a, scl(ab, b1)), scl(ac, b2)));
}

/* distanceSquaredToAABB (geometry.h:262-277) */
float qo_dist2_aabb(const float* p, const float* box) {
    float d2 = 0.0f;
    for (int a = 0; a < 3; ++a) {
        const float v = p[a], lo = box[a], hi = box[3 + a];
        if (v < lo) {
            const float d = lo - v;
            d2 += d * d;
        } else if (v > hi) {
            const float d = v - hi;
            d2 += d * d;
        }
    }
    return d2;
}

/* ------------------------------------------------------------------------- */
/* Gaussian ellipsoids (gaussian.h:23-131)                                     */
/* ------------------------------------------------------------------------- */
static void gaussian_axes(const float* q4, v3* u, v3* v, v3* w) {
    const float lenSq = fmaf(q4[3], q4[3], fmaf(q4[2], q4[2], fmaf(q4[1], q4[1], q4[0] * q4[0])));
    float inv = 1.0f;
    if (lenSq > 0.0f) inv = 1.0f / sqrtf(lenSq);
    const float qx = q4[0] * inv, qy = q4[1] * inv, qz = q4[2] * inv, qw = q4[3] * inv;
    const float yyzz = fmaf(qy, qy, qz * qz);
    const float xxzz = fmaf(qx, qx, qz * qz);
    const float xxyy = fmaf(qx, qx, qy * qy);
    *u = mk(fmaf(-2.0f, yyzz, 1.0f), 2.0f * fmaf(qx, qy, qz * qw), 2.0f * fmaf(qx, qz, -(qy * qw)));
    *v = mk(2.0f * fmaf(qx, qy, -(qz * qw)), fmaf(-2.0f, xxzz, 1.0f), 2.0f * fmaf(qy, qz, qx * qw));
    *w = mk(2.0f * fmaf(qx, qz, qy * qw), 2.0f * fmaf(qy, qz, -(qx * qw)), fmaf(-2.0f, xxyy, 1.0f));
}

void qo_gaussian_bounds(const float* g, float* box) {
    v3 u, v, w;
    gaussian_axes(g + 3, &u, &v, &w);
    const float a2 = g[7] * g[7];
    const float b2 = g[8] * g[8];
    const float c2 = g[9] * g[9];
    const float uu[3] = {u.x, u.y, u.z}, vv[3] = {v.x, v.y, v.z}, ww[3] = {w.x, w.y, w.z};
    for (int a = 0; a < 3; ++a) {
        const float ui = uu[a], vi = vv[a], wi = ww[a];
        const float half = sqrtf(fmaf(c2, wi * wi, fmaf(b2, vi * vi, a2 * ui * ui)));
        const float pad = half + 1e-6f * (1.0f + fabsf(g[a]) + half);
        box[a] = g[a] - pad;
        box[3 + a] = g[a] + pad;
    }
}

float qo_gaussian_dist2(const float* p3, const float* g) {
    v3 u, v, w;
    gaussian_axes(g + 3, &u, &v, &w);
    const v3 d = sub(ld3(p3), ld3(g));
    const float y0 = dot(d, u), y1 = dot(d, v), y2 = dot(d, w);
    const float a = g[7], b = g[8], c = g[9];
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

/* ------------------------------------------------------------------------- */
/* primitive traits (src/gpu/prim_ops.h:74-117)                                */
/* ------------------------------------------------------------------------- */
float qo_prim_dist2(int kind, const float* q, const float* item) {
    if (kind == QO_TRI) return qo_closest_point_dist2(q, item);
    if (kind == QO_POINT) {
        const v3 d = sub(ld3(q), ld3(item));
        return dot(d, d);
    }
    return qo_gaussian_dist2(q, item);
}

void qo_prim_bounds(int kind, const float* item, float* box) {
    if (kind == QO_TRI) {
        tri_bounds(item, box);
    } else if (kind == QO_POINT) {
        box_empty(box);
        box_extend(box, item);
    } else {
        qo_gaussian_bounds(item, box);
    }
}

void qo_prim_centroid(int kind, const float* item, float* c) {
    if (kind == QO_TRI) {
        c[0] = (item[0] + item[3] + item[6]) / 3.0f;
        c[1] = (item[1] + item[4] + item[7]) / 3.0f;
        c[2] = (item[2] + item[5] + item[8]) / 3.0f;
    } else {
        c[0] = item[0];
        c[1] = item[1];
        c[2] = item[2];
    }
}

/* ------------------------------------------------------------------------- */
/* LBVH (src/gpu/lbvh.cu:213-514, 1954-2041)                                   */
/* ------------------------------------------------------------------------- */
static uint32_t spread10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

/* quantize() of lbvh.cu:285-290 */
static uint32_t quant(float v, float lo, float extent) {
    if (extent <= 0.0f) return 0;
    const float q = (v - lo) / extent * 1023.0f + 0.5f;
    return (uint32_t)(int)fminf(1023.0f, fmaxf(0.0f, q));
}

static int cmp_u64(const void* a, const void* b) {
    const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : x > y ? 1 : 0;
}

static inline int clz64(uint64_t x) { return x == 0 ? 64 : __builtin_clzll(x); }

/* common-prefix length of sorted keys a and b; -1 outside [0, n) (Karras 2012) */
static inline int prefix(const uint64_t* keys, int n, int a, int b) {
    if (b < 0 || b >= n) return -1;
    return clz64(keys[a] ^ keys[b]);
}

static void union_box(const qo_node* l, const qo_node* r, qo_node* out) {
    for (int a = 0; a < 3; ++a) {
        out->mn[a] = l->mn[a] < r->mn[a] ? l->mn[a] : r->mn[a];
        out->mx[a] = l->mx[a] > r->mx[a] ? l->mx[a] : r->mx[a];
    }
}

static void refit_internal(qo_node* nodes, int n) {
    /* post-order over the internal nodes with an explicit stack */
    int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * (size_t)(2 * n + 8));
    uint8_t* seen = (uint8_t*)calloc((size_t)n, 1);
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const int i = stack[sp - 1];
        const qo_node* nd = &nodes[i];
        if (!seen[i]) {
            seen[i] = 1;
            if (nd->left < n - 1) stack[sp++] = nd->left;
            if (nd->right < n - 1) stack[sp++] = nd->right;
            continue;
        }
        --sp;
        union_box(&nodes[nd->left], &nodes[nd->right], &nodes[i]);
    }
    free(seen);
    free(stack);
}

int qo_lbvh_build(int kind, const float* items, int n, qo_node* nodes, float* sorted,
                  int32_t* prim_ids, int32_t* parent, int32_t* depth) {
    if (n < 2) return -1;
    const int s = qo_stride(kind);
    const int node_count = 2 * n - 1;

    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    float* cen = (float*)malloc(sizeof(float) * 3 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        qo_prim_centroid(kind, items + (size_t)i * s, cen + 3 * (size_t)i);
        for (int a = 0; a < 3; ++a) {
            lo[a] = fminf(lo[a], cen[3 * (size_t)i + a]);
            hi[a] = fmaxf(hi[a], cen[3 * (size_t)i + a]);
        }
    }
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        const float* c = cen + 3 * (size_t)i;
        const uint32_t code = spread10(quant(c[0], lo[0], hi[0] - lo[0])) |
                              (spread10(quant(c[1], lo[1], hi[1] - lo[1])) << 1) |
                              (spread10(quant(c[2], lo[2], hi[2] - lo[2])) << 2);
        keys[i] = ((uint64_t)code << 32) | (uint32_t)i;
    }
    free(cen);
    qsort(keys, (size_t)n, sizeof(uint64_t), cmp_u64);

    for (int k = 0; k < n; ++k) {
        const int src = (int)(uint32_t)keys[k];
        memcpy(sorted + (size_t)k * s, items + (size_t)src * s, sizeof(float) * (size_t)s);
        prim_ids[k] = src;
    }
    for (int i = 0; i < node_count; ++i) parent[i] = -1;

    for (int i = 0; i < n - 1; ++i) {
        const int dir = prefix(keys, n, i, i + 1) > prefix(keys, n, i, i - 1) ? 1 : -1;
        const int dmin = prefix(keys, n, i, i - dir);
        int lmax = 2;
        while (prefix(keys, n, i, i + lmax * dir) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t > 0; t /= 2) {
            if (prefix(keys, n, i, i + (l + t) * dir) > dmin) l += t;
        }
        const int j = i + l * dir;
        const int first = i < j ? i : j;
        const int last = i < j ? j : i;
        const int dnode = prefix(keys, n, i, j);
        /* split = last index in [first, last) whose prefix with `first` exceeds dnode */
        int split = first;
        int step = last - first;
        do {
            step = (step + 1) >> 1;
            const int cand = split + step;
            if (cand < last && prefix(keys, n, first, cand) > dnode) split = cand;
        } while (step > 1);
        const int left = split == first ? (n - 1 + split) : split;
        const int right = split + 1 == last ? (n - 1 + split + 1) : split + 1;
        nodes[i].left = left;
        nodes[i].right = right;
        parent[left] = i;
        parent[right] = i;
    }
    for (int k = 0; k < n; ++k) {
        qo_node* leaf = &nodes[n - 1 + k];
        float box[6];
        qo_prim_bounds(kind, sorted + (size_t)k * s, box);
        memcpy(leaf->mn, box, sizeof(float) * 3);
        memcpy(leaf->mx, box + 3, sizeof(float) * 3);
        leaf->left = -(k + 1);
        leaf->right = 1;
    }
    free(keys);
    refit_internal(nodes, n);

    /* depth = distance to the root, top-down over the parent-before-child order */
    int max_depth = 0;
    int32_t* queue = (int32_t*)malloc(sizeof(int32_t) * (size_t)node_count);
    int head = 0, tail = 0;
    queue[tail++] = 0;
    depth[0] = 0;
    while (head < tail) {
        const int i = queue[head++];
        if (depth[i] > max_depth) max_depth = depth[i];
        if (i < n - 1) {
            depth[nodes[i].left] = depth[i] + 1;
            depth[nodes[i].right] = depth[i] + 1;
            queue[tail++] = nodes[i].left;
            queue[tail++] = nodes[i].right;
        }
    }
    free(queue);
    return max_depth;
}

void qo_refit(int kind, qo_node* nodes, const float* sorted, int n) {
    const int s = qo_stride(kind);
    for (int k = 0; k < n; ++k) {
        float box[6];
        qo_prim_bounds(kind, sorted + (size_t)k * s, box);
        memcpy(nodes[n - 1 + k].mn, box, sizeof(float) * 3);
        memcpy(nodes[n - 1 + k].mx, box + 3, sizeof(float) * 3);
    }
    refit_internal(nodes, n);
}

/* 4-wide collapse: even-depth internal nodes take children + grandchildren */
static void wide_fill(qo_wide_entry* e, const qo_node* box, int32_t child) {
    memcpy(e->mn, box->mn, sizeof(float) * 3);
    memcpy(e->mx, box->mx, sizeof(float) * 3);
    e->child = child;
    e->pad = 0;
}

int qo_wide_collapse(const qo_node* nodes, const int32_t* depth, int n, int32_t* wide_id,
                     qo_wide_entry* wide) {
    int count = 0;
    for (int i = 0; i < n - 1; ++i) {
        wide_id[i] = count;
        if ((depth[i] & 1) == 0) ++count;
    }
    for (int i = 0; i < n - 1; ++i) {
        if (depth[i] & 1) continue;
        qo_wide_entry* out = wide + 4 * (size_t)wide_id[i];
        for (int s = 0; s < 4; ++s) {
            out[s].mn[0] = out[s].mn[1] = out[s].mn[2] = INFINITY;
            out[s].mx[0] = out[s].mx[1] = out[s].mx[2] = -INFINITY;
            out[s].child = INT32_MIN;
            out[s].pad = 0;
        }
        const int kids[2] = {nodes[i].left, nodes[i].right};
        int slot = 0;
        for (int k = 0; k < 2; ++k) {
            const int c = kids[k];
            if (c >= n - 1) {
                wide_fill(&out[slot++], &nodes[c], nodes[c].left);
                continue;
            }
            const int g[2] = {nodes[c].left, nodes[c].right};
            for (int j = 0; j < 2; ++j) {
                const int gc = g[j];
                wide_fill(&out[slot++], &nodes[gc], gc >= n - 1 ? nodes[gc].left : wide_id[gc]);
            }
        }
    }
    return count;
}

/* 4-wide collapse, leaf-size-4 form (the engine's qk_wide_build_leaf4; quarry has no
 * counterpart: it names leaf-size-4 SAH trees with 4-wide nodes as its next build lever,
 * docs/design.md:203,207).  A child or grandchild whose subtree holds 2..4 leaves on
 * contiguous slots is one slot: child = -(first slot + 1), pad = leaves; single leaves have
 * pad = 1; internal slots pad = 0.  Wide nodes: even-depth internal nodes that are the root or
 * not such a subtree themselves.  Slot ranges are derived bottom-up from the links: a node's
 * range is contiguous when both children's are and they abut. */
int qo_wide_collapse_leaf4(const qo_node* nodes, const int32_t* depth, int n, int32_t* wide_id,
                           qo_wide_entry* wide) {
    const int m = n - 1;
    int32_t* first = (int32_t*)malloc(sizeof(int32_t) * (size_t)m);
    int32_t* cnt = (int32_t*)malloc(sizeof(int32_t) * (size_t)m);
    int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * (size_t)(2 * n));
    uint8_t* seen = (uint8_t*)calloc((size_t)m, 1);
    if (!first || !cnt || !stack || !seen) {
        free(first); free(cnt); free(stack); free(seen);
        return -1;
    }
    /* post-order over internal nodes from the root (node 0) */
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const int i = stack[sp - 1];
        const int kids[2] = {nodes[i].left, nodes[i].right};
        if (!seen[i]) {
            seen[i] = 1;
            for (int k = 0; k < 2; ++k)
                if (kids[k] < m) stack[sp++] = kids[k];
            continue;
        }
        --sp;
        int f[2], c[2];
        for (int k = 0; k < 2; ++k) {
            if (kids[k] >= m) {
                f[k] = kids[k] - m;
                c[k] = 1;
            } else {
                f[k] = first[kids[k]];
                c[k] = cnt[kids[k]];
            }
        }
        const int lo = f[0] < f[1] ? f[0] : f[1];
        const int e0 = f[0] + c[0], e1 = f[1] + c[1];
        const int hi = e0 > e1 ? e0 : e1;
        first[i] = lo;
        cnt[i] = (c[0] > 0 && c[1] > 0 && hi - lo == c[0] + c[1]) ? c[0] + c[1] : 0;
    }
    /* code of internal node c: (first << 2) | (leaves - 1) for 2..4 contiguous leaves */
#define SMALL_CODE(c) ((cnt[c] >= 2 && cnt[c] <= 4) ? ((first[c] << 2) | (cnt[c] - 1)) : 0)
    int count = 0;
    for (int i = 0; i < m; ++i) {
        wide_id[i] = count;
        if ((depth[i] & 1) == 0 && (i == 0 || SMALL_CODE(i) == 0)) ++count;
    }
    for (int i = 0; i < m; ++i) {
        if ((depth[i] & 1) || (i != 0 && SMALL_CODE(i) != 0)) continue;
        qo_wide_entry* out = wide + 4 * (size_t)wide_id[i];
        for (int s = 0; s < 4; ++s) {
            out[s].mn[0] = out[s].mn[1] = out[s].mn[2] = INFINITY;
            out[s].mx[0] = out[s].mx[1] = out[s].mx[2] = -INFINITY;
            out[s].child = INT32_MIN;
            out[s].pad = 0;
        }
        int slot = 0;
        const int kids[2] = {nodes[i].left, nodes[i].right};
        for (int k = 0; k < 2; ++k) {
            const int c = kids[k];
            const int reps = (c >= m || SMALL_CODE(c) != 0) ? 1 : 2;
            for (int j = 0; j < reps; ++j) {
                const int x = reps == 1 ? c : (j == 0 ? nodes[c].left : nodes[c].right);
                qo_wide_entry* e = &out[slot++];
                if (x >= m) {
                    wide_fill(e, &nodes[x], nodes[x].left);
                    e->pad = 1;
                } else if (SMALL_CODE(x) != 0) {
                    wide_fill(e, &nodes[x], -(first[x] + 1));
                    e->pad = cnt[x];
                } else {
                    wide_fill(e, &nodes[x], wide_id[x]);
                }
            }
        }
    }
#undef SMALL_CODE
    free(first); free(cnt); free(stack); free(seen);
    return count;
}

/* ------------------------------------------------------------------------- */
/* a tiny parallel-for over query ranges                                       */
/* ------------------------------------------------------------------------- */
typedef void (*range_fn)(void* ctx, int begin, int end);
typedef struct {
    range_fn fn;
    void* ctx;
    int begin, end;
} task_t;

static void* task_main(void* p) {
    task_t* t = (task_t*)p;
    t->fn(t->ctx, t->begin, t->end);
    return NULL;
}

static void parallel_for(int count, int threads, range_fn fn, void* ctx) {
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    if (threads == 1 || count < 64) {
        fn(ctx, 0, count);
        return;
    }
    pthread_t tid[256];
    task_t tasks[256];
    const int chunk = (count + threads - 1) / threads;
    int used = 0;
    for (int t = 0; t < threads; ++t) {
        const int b = t * chunk;
        const int e = b + chunk < count ? b + chunk : count;
        if (b >= e) break;
        tasks[t].fn = fn;
        tasks[t].ctx = ctx;
        tasks[t].begin = b;
        tasks[t].end = e;
        pthread_create(&tid[t], NULL, task_main, &tasks[t]);
        ++used;
    }
    for (int t = 0; t < used; ++t) pthread_join(tid[t], NULL);
}

static void node_box(const qo_node* nd, float* box6) {
    memcpy(box6, nd->mn, sizeof(float) * 3);
    memcpy(box6 + 3, nd->mx, sizeof(float) * 3);
}

/* ------------------------------------------------------------------------- */
/* rays: depth-first, bestT as the prune bound (src/cpu/bvh.cpp:138-178)       */
/* ------------------------------------------------------------------------- */
typedef struct {
    const qo_node* nodes;
    const float* tris;
    const int32_t* ids;
    int n;
    const float* rays;
    uint64_t* out;
} ray_ctx;

static void ray_range(void* p, int begin, int end) {
    const ray_ctx* c = (const ray_ctx*)p;
    int32_t stack[256];
    for (int r = begin; r < end; ++r) {
        const float* ray = c->rays + 8 * (size_t)r;
        float best_t = ray[7];
        int hit = 0;
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const int i = stack[--sp];
            const qo_node* nd = &c->nodes[i];
            float box[6], tenter;
            node_box(nd, box);
            if (!qo_intersect_aabb(ray, box, best_t, &tenter)) continue;
            if (i >= c->n - 1) {
                const int slot = -nd->left - 1;
                float sub8[8];
                memcpy(sub8, ray, sizeof(sub8));
                sub8[7] = best_t;
                float t;
                if (qo_intersect_triangle(sub8, c->tris + 9 * (size_t)slot, &t)) {
                    best_t = t;
                    hit = 1;
                }
            } else {
                stack[sp++] = nd->right;
                stack[sp++] = nd->left;
            }
        }
        uint32_t bits = 0;
        if (hit) memcpy(&bits, &best_t, sizeof(bits));
        c->out[r] = hit ? ((1ull << 32) | bits) : 0ull;
    }
}

void qo_raycast(const qo_node* nodes, const float* tris, const int32_t* ids, int n,
                const float* rays, int nrays, uint64_t* out, int threads) {
    ray_ctx c = {nodes, tris, ids, n, rays, out};
    parallel_for(nrays, threads, ray_range, &c);
}

/* ------------------------------------------------------------------------- */
/* closest: best-first over a min-heap of (bound, node) (bvh.cpp:222-259)      */
/* ------------------------------------------------------------------------- */
typedef struct {
    float bound;
    int32_t node;
} nb_t;

typedef struct {
    nb_t* v;
    int size, cap;
} heap_t;

static void heap_push(heap_t* h, float bound, int node) {
    if (h->size == h->cap) {
        h->cap = h->cap ? 2 * h->cap : 256;
        h->v = (nb_t*)realloc(h->v, sizeof(nb_t) * (size_t)h->cap);
    }
    int i = h->size++;
    while (i > 0) {
        const int p = (i - 1) / 2;
        if (!(h->v[p].bound > bound)) break;
        h->v[i] = h->v[p];
        i = p;
    }
    h->v[i].bound = bound;
    h->v[i].node = node;
}

static nb_t heap_pop(heap_t* h) {
    const nb_t top = h->v[0];
    const nb_t last = h->v[--h->size];
    int i = 0;
    for (;;) {
        int c = 2 * i + 1;
        if (c >= h->size) break;
        if (c + 1 < h->size && h->v[c + 1].bound < h->v[c].bound) ++c;
        if (!(h->v[c].bound < last.bound)) break;
        h->v[i] = h->v[c];
        i = c;
    }
    if (h->size > 0) h->v[i] = last;
    return top;
}

/* (dist2, id) lexicographic order = closerHit (geometry.h:191-193) */
static inline int closer(float da, int ia, float db, int ib) {
    return da < db || (da == db && ia < ib);
}

typedef struct {
    int kind, stride;
    const qo_node* nodes;
    const float* items;
    const int32_t* ids;
    int n;
    const float* q;
    int k;
    float r2;
    uint32_t* out2;
    int32_t* counts;
    const int64_t* offsets;
    uint64_t* keys;
} q_ctx;

static void closest_range(void* p, int begin, int end) {
    const q_ctx* c = (const q_ctx*)p;
    heap_t h = {0, 0, 0};
    float box[6];
    for (int qi = begin; qi < end; ++qi) {
        const float* q = c->q + 3 * (size_t)qi;
        int found = 0, best_id = -1;
        float best = INFINITY;
        h.size = 0;
        node_box(&c->nodes[0], box);
        heap_push(&h, qo_dist2_aabb(q, box), 0);
        while (h.size > 0) {
            const nb_t cur = heap_pop(&h);
            if (found && cur.bound > best) break;
            if (cur.node >= c->n - 1) {
                const int slot = cur.node - (c->n - 1);
                const float d2 = qo_prim_dist2(c->kind, q, c->items + (size_t)slot * c->stride);
                const int id = c->ids[slot];
                if (!found || closer(d2, id, best, best_id)) {
                    best = d2;
                    best_id = id;
                    found = 1;
                }
                continue;
            }
            const int kids[2] = {c->nodes[cur.node].left, c->nodes[cur.node].right};
            for (int j = 0; j < 2; ++j) {
                node_box(&c->nodes[kids[j]], box);
                const float b = qo_dist2_aabb(q, box);
                if (!found || b <= best) heap_push(&h, b, kids[j]);
            }
        }
        uint32_t bits = 0;
        if (found) memcpy(&bits, &best, sizeof(bits));
        c->out2[2 * (size_t)qi] = bits;
        c->out2[2 * (size_t)qi + 1] = (uint32_t)(found ? best_id : -1);
    }
    free(h.v);
}

void qo_closest(int kind, const qo_node* nodes, const float* sorted, const int32_t* ids, int n,
                const float* q, int nq, uint32_t* out2, int threads) {
    q_ctx c;
    memset(&c, 0, sizeof(c));
    c.kind = kind;
    c.stride = qo_stride(kind);
    c.nodes = nodes;
    c.items = sorted;
    c.ids = ids;
    c.n = n;
    c.q = q;
    c.out2 = out2;
    parallel_for(nq, threads, closest_range, &c);
}

/* ------------------------------------------------------------------------- */
/* kNN: best-first with a bounded sorted candidate list (bvh.cpp:261-313).     */
/* The list keeps the k best by (dist2, id); a candidate enters only when it   */
/* is strictly closer than the current k-th, exactly the max-heap rule.        */
/* ------------------------------------------------------------------------- */
static void knn_insert(float* d, int32_t* id, int* m, int k, float dn, int idn) {
    int pos = *m;
    while (pos > 0 && closer(dn, idn, d[pos - 1], id[pos - 1])) --pos;
    if (*m == k && pos == k) return;
    if (*m < k) ++*m;
    for (int j = *m - 1; j > pos; --j) {
        d[j] = d[j - 1];
        id[j] = id[j - 1];
    }
    d[pos] = dn;
    id[pos] = idn;
}

static void knn_range(void* p, int begin, int end) {
    const q_ctx* c = (const q_ctx*)p;
    heap_t h = {0, 0, 0};
    float box[6];
    float d[64];
    int32_t id[64];
    const int k = c->k;
    for (int qi = begin; qi < end; ++qi) {
        const float* q = c->q + 3 * (size_t)qi;
        int m = 0;
        h.size = 0;
        node_box(&c->nodes[0], box);
        heap_push(&h, qo_dist2_aabb(q, box), 0);
        while (h.size > 0) {
            const nb_t cur = heap_pop(&h);
            if (m == k && cur.bound > d[k - 1]) break;
            if (cur.node >= c->n - 1) {
                const int slot = cur.node - (c->n - 1);
                const float d2 = qo_prim_dist2(c->kind, q, c->items + (size_t)slot * c->stride);
                const int pid = c->ids[slot];
                if (m == k && !closer(d2, pid, d[k - 1], id[k - 1])) continue;
                knn_insert(d, id, &m, k, d2, pid);
                continue;
            }
            const int kids[2] = {c->nodes[cur.node].left, c->nodes[cur.node].right};
            for (int j = 0; j < 2; ++j) {
                node_box(&c->nodes[kids[j]], box);
                const float b = qo_dist2_aabb(q, box);
                if (m < k || b <= d[k - 1]) heap_push(&h, b, kids[j]);
            }
        }
        uint32_t* dst = c->out2 + 2 * (size_t)qi * (size_t)k;
        for (int j = 0; j < k; ++j) {
            uint32_t bits = 0;
            if (j < m) memcpy(&bits, &d[j], sizeof(bits));
            dst[2 * j] = bits;
            dst[2 * j + 1] = (uint32_t)(j < m ? id[j] : -1);
        }
    }
    free(h.v);
}

void qo_knn(int kind, const qo_node* nodes, const float* sorted, const int32_t* ids, int n,
            const float* q, int nq, int k, uint32_t* out2, int threads) {
    if (k < 1 || k > 64) return;
    q_ctx c;
    memset(&c, 0, sizeof(c));
    c.kind = kind;
    c.stride = qo_stride(kind);
    c.nodes = nodes;
    c.items = sorted;
    c.ids = ids;
    c.n = n;
    c.q = q;
    c.k = k;
    c.out2 = out2;
    parallel_for(nq, threads, knn_range, &c);
}

/* ------------------------------------------------------------------------- */
/* radius: sphere-box culling, results sorted by (dist2, id) (bvh.cpp:315-349) */
/* ------------------------------------------------------------------------- */
static int cmp_key(const void* a, const void* b) { return cmp_u64(a, b); }

static void radius_range(void* p, int begin, int end) {
    const q_ctx* c = (const q_ctx*)p;
    int cap = 1024;
    int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
    int kcap = 256;
    uint64_t* tmp = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)kcap);
    float box[6];
    for (int qi = begin; qi < end; ++qi) {
        const float* q = c->q + 3 * (size_t)qi;
        int sp = 0, m = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const int i = stack[--sp];
            node_box(&c->nodes[i], box);
            if (qo_dist2_aabb(q, box) > c->r2) continue;
            if (i >= c->n - 1) {
                const int slot = i - (c->n - 1);
                const float d2 = qo_prim_dist2(c->kind, q, c->items + (size_t)slot * c->stride);
                if (d2 > c->r2) continue;
                if (c->keys) {
                    if (m == kcap) {
                        kcap *= 2;
                        tmp = (uint64_t*)realloc(tmp, sizeof(uint64_t) * (size_t)kcap);
                    }
                    uint32_t bits;
                    memcpy(&bits, &d2, sizeof(bits));
                    tmp[m] = ((uint64_t)bits << 32) | (uint32_t)c->ids[slot];
                }
                ++m;
            } else {
                if (sp + 2 > cap) {
                    cap *= 2;
                    stack = (int32_t*)realloc(stack, sizeof(int32_t) * (size_t)cap);
                }
                stack[sp++] = c->nodes[i].right;
                stack[sp++] = c->nodes[i].left;
            }
        }
        c->counts[qi] = m;
        if (c->keys) {
            qsort(tmp, (size_t)m, sizeof(uint64_t), cmp_key);
            memcpy(c->keys + c->offsets[qi], tmp, sizeof(uint64_t) * (size_t)m);
        }
    }
    free(tmp);
    free(stack);
}

int64_t qo_radius(int kind, const qo_node* nodes, const float* sorted, const int32_t* ids, int n,
                  const float* q, int nq, float radius, int32_t* counts, const int64_t* offsets,
                  uint64_t* keys, int threads) {
    if (radius < 0.0f) {
        for (int i = 0; i < nq; ++i) counts[i] = 0;
        return 0;
    }
    q_ctx c;
    memset(&c, 0, sizeof(c));
    c.kind = kind;
    c.stride = qo_stride(kind);
    c.nodes = nodes;
    c.items = sorted;
    c.ids = ids;
    c.n = n;
    c.q = q;
    c.r2 = radius * radius;
    c.counts = counts;
    c.offsets = offsets;
    c.keys = keys;
    parallel_for(nq, threads, radius_range, &c);
    int64_t total = 0;
    for (int i = 0; i < nq; ++i) total += counts[i];
    return total;
}

/* ------------------------------------------------------------------------- */
/* brute force (src/cpu/brute.cpp:37-197)                                      */
/* ------------------------------------------------------------------------- */
void qo_raycast_brute(const float* tris, int n, const float* rays, int nrays, uint64_t* out) {
    for (int r = 0; r < nrays; ++r) {
        float sub8[8];
        memcpy(sub8, rays + 8 * (size_t)r, sizeof(sub8));
        int hit = 0;
        float best = sub8[7];
        for (int i = 0; i < n; ++i) {
            float t;
            sub8[7] = best;
            if (qo_intersect_triangle(sub8, tris + 9 * (size_t)i, &t)) {
                best = t;
                hit = 1;
            }
        }
        uint32_t bits = 0;
        if (hit) memcpy(&bits, &best, sizeof(bits));
        out[r] = hit ? ((1ull << 32) | bits) : 0ull;
    }
}

void qo_closest_brute(int kind, const float* items, int n, const float* q, int nq,
                      uint32_t* out2) {
    const int s = qo_stride(kind);
    for (int qi = 0; qi < nq; ++qi) {
        float best = INFINITY;
        int best_id = -1;
        for (int i = 0; i < n; ++i) {
            const float d2 = qo_prim_dist2(kind, q + 3 * (size_t)qi, items + (size_t)i * s);
            if (best_id < 0 || d2 < best) {
                best = d2;
                best_id = i;
            }
        }
        uint32_t bits = 0;
        if (best_id >= 0) memcpy(&bits, &best, sizeof(bits));
        out2[2 * (size_t)qi] = bits;
        out2[2 * (size_t)qi + 1] = (uint32_t)best_id;
    }
}

void qo_knn_brute(int kind, const float* items, int n, const float* q, int nq, int k,
                  uint32_t* out2) {
    const int s = qo_stride(kind);
    float d[64];
    int32_t id[64];
    if (k < 1 || k > 64) return;
    for (int qi = 0; qi < nq; ++qi) {
        int m = 0;
        for (int i = 0; i < n; ++i) {
            const float d2 = qo_prim_dist2(kind, q + 3 * (size_t)qi, items + (size_t)i * s);
            if (m == k && !closer(d2, i, d[k - 1], id[k - 1])) continue;
            knn_insert(d, id, &m, k, d2, i);
        }
        uint32_t* dst = out2 + 2 * (size_t)qi * (size_t)k;
        for (int j = 0; j < k; ++j) {
            uint32_t bits = 0;
            if (j < m) memcpy(&bits, &d[j], sizeof(bits));
            dst[2 * j] = bits;
            dst[2 * j + 1] = (uint32_t)(j < m ? id[j] : -1);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* fingerprints: whole-word FNV-1a folds (src/core/fingerprint.h:226-303)      */
/* ------------------------------------------------------------------------- */
static const uint64_t kFnvBasis = 0xcbf29ce484222325ull;
static const uint64_t kFnvPrime = 0x100000001b3ull;

static inline uint64_t mix(uint64_t h, uint64_t v) { return (h ^ v) * kFnvPrime; }

uint64_t qo_ray_hash(const uint64_t* res, int64_t n, uint64_t* hits) {
    uint64_t h = kFnvBasis, count = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int hit = (res[i] >> 32) != 0;
        const uint64_t bits = hit ? (uint32_t)res[i] : 0u;
        count += (uint64_t)hit;
        h = mix(h, ((uint64_t)(hit ? 1u : 0u) << 32) | bits);
    }
    if (hits) *hits = count;
    return h;
}

uint64_t qo_closest_hash(const uint32_t* res2, int64_t n) {
    uint64_t h = kFnvBasis;
    for (int64_t i = 0; i < n; ++i) {
        const int32_t id = (int32_t)res2[2 * i + 1];
        const int found = id >= 0;
        h = mix(h, ((uint64_t)(found ? 1u : 0u) << 32) | (found ? res2[2 * i] : 0u));
        h = mix(h, found ? (uint64_t)id + 1u : 0u);
    }
    return h;
}

uint64_t qo_knn_hash(const uint32_t* res2, int64_t n, int k) {
    uint64_t h = kFnvBasis;
    for (int64_t i = 0; i < n; ++i) {
        const uint32_t* row = res2 + 2 * i * k;
        int m = 0;
        while (m < k && (int32_t)row[2 * m + 1] >= 0) ++m;
        h = mix(h, (uint64_t)m);
        for (int j = 0; j < m; ++j) {
            h = mix(h, row[2 * j]);
            h = mix(h, (uint64_t)(int64_t)(int32_t)row[2 * j + 1] + 1u);
        }
    }
    return h;
}

uint64_t qo_radius_hash(const int64_t* offsets, const uint64_t* keys, int64_t n) {
    uint64_t h = kFnvBasis;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t b = offsets[i], e = offsets[i + 1];
        h = mix(h, (uint64_t)(e - b));
        for (int64_t j = b; j < e; ++j) {
            h = mix(h, keys[j] >> 32);
            h = mix(h, (uint64_t)(int64_t)(int32_t)(uint32_t)keys[j] + 1u);
        }
    }
    return h;
}

/* treeHashGPU: byte-wise FNV-1a over the node array (lbvh.cu:3174-3188) */
uint64_t qo_bytes_hash(const void* bytes, size_t len) {
    const unsigned char* b = (const unsigned char*)bytes;
    uint64_t h = kFnvBasis;
    for (size_t i = 0; i < len; ++i) h = (h ^ b[i]) * kFnvPrime;
    return h;
}
