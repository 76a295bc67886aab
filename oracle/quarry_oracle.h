/*
 * quarry_oracle.h -- CPU restatement of quarry's spatial-query hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine in
 * quarry-gpu_b200/: only tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py load it.  Nothing in the product links or calls it.
 *
 * Every function restates the reference algorithm op for op (same IEEE float
 * operations in the same order, explicit fmaf where the reference writes
 * QUARRY_FMA, no contraction: build with -ffp-contract=off), so its results are
 * bit-identical to quarry's CPU reference.  Parity of this restatement with the
 * reference itself is pinned by tests/test_oracle_pin.py, which runs the
 * reference sources compiled into oracle/_ref/ on the same inputs, and by the
 * golden fixtures in tests/golden/ (generated from oracle/_ref by
 * tests/golden/make_golden.py).
 *
 * Data layouts (all little-endian, tightly packed float32 / int32):
 *   triangle  9 floats  a.xyz b.xyz c.xyz            (src/core/geometry.h:91-101)
 *   point     3 floats                               (src/core/point_cloud.h:9-17)
 *   gaussian 10 floats  mean.xyz quat.xyzw scale.xyz (src/core/gaussian.h:12-20)
 *   ray       8 floats  origin.xyz dir.xyz tMin tMax (src/core/geometry.h:84-89)
 *   node     32 bytes   mn.xyz mx.xyz left right     (src/gpu/gpu_node.h:9-14)
 *   wide     128 bytes  4 x {mn.xyz mx.xyz child pad}(src/gpu/gpu_node.h:46-57)
 *   ray result   uint64 (hit << 32) | bits(t)        (src/gpu/gpu_bvh.h:91-97)
 *   query result {uint32 dist2 bits, int32 id}       (src/gpu/gpu_bvh.h:250-253)
 */
#ifndef QUARRY_ORACLE_H
#define QUARRY_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { QO_TRI = 0, QO_POINT = 1, QO_GAUSS = 2 };

typedef struct {
    float mn[3];
    float mx[3];
    int32_t left;
    int32_t right;
} qo_node;

typedef struct {
    float mn[3];
    float mx[3];
    int32_t child;
    int32_t pad;
} qo_wide_entry;

/* floats per primitive of a kind (9, 3, 10); 0 for an unknown kind */
int qo_stride(int kind);

/* ---- leaf arithmetic (src/core/geometry.h, src/core/gaussian.h) ---- */
int qo_intersect_aabb(const float* ray8, const float* box6, float tmax, float* tenter);
int qo_intersect_triangle(const float* ray8, const float* tri9, float* t);
float qo_closest_point_dist2(const float* p3, const float* tri9);
float qo_dist2_aabb(const float* p3, const float* box6);
void qo_gaussian_bounds(const float* g10, float* box6);
float qo_gaussian_dist2(const float* p3, const float* g10);
float qo_prim_dist2(int kind, const float* q3, const float* item);
void qo_prim_bounds(int kind, const float* item, float* box6);
void qo_prim_centroid(int kind, const float* item, float* c3);

/* ---- LBVH build (src/gpu/lbvh.cu) ----
 * nodes: 2n-1 entries; sorted: n*stride floats; prim_ids, parent, depth: as named.
 * parent/depth have 2n-1 entries.  Returns the maximum depth, or -1 when n < 2. */
int qo_lbvh_build(int kind, const float* items, int n, qo_node* nodes, float* sorted,
                  int32_t* prim_ids, int32_t* parent, int32_t* depth);

/* 4-wide collapse of an LBVH (src/gpu/lbvh.cu:731-825).  wide_id has n-1 entries,
 * wide must hold n-1 nodes (4 entries each).  Returns the number of wide nodes. */
int qo_wide_collapse(const qo_node* nodes, const int32_t* depth, int n, int32_t* wide_id,
                     qo_wide_entry* wide);

/* 4-wide collapse in the leaf-size-4 form (leaf ranges of 2..4 contiguous slots take one
 * slot, pad = primitive count); same buffers; -1 when out of host memory. */
int qo_wide_collapse_leaf4(const qo_node* nodes, const int32_t* depth, int n, int32_t* wide_id,
                           qo_wide_entry* wide);

/* in-place refit: recompute leaf boxes from sorted items and every internal box */
void qo_refit(int kind, qo_node* nodes, const float* sorted, int n);

/* ---- queries over an LBVH built above (leaf size 1), src/cpu/bvh.cpp ----
 * threads <= 0 uses all cores. */
void qo_raycast(const qo_node* nodes, const float* sorted_tris, const int32_t* prim_ids, int n,
                const float* rays, int nrays, uint64_t* out, int threads);
void qo_closest(int kind, const qo_node* nodes, const float* sorted, const int32_t* prim_ids,
                int n, const float* q, int nq, uint32_t* out2, int threads);
void qo_knn(int kind, const qo_node* nodes, const float* sorted, const int32_t* prim_ids, int n,
            const float* q, int nq, int k, uint32_t* out2, int threads);
/* radius: counts[nq]; when keys != NULL also fills keys at offsets (exclusive sum of counts)
 * sorted by (dist2 bits, id).  Returns the total. */
int64_t qo_radius(int kind, const qo_node* nodes, const float* sorted, const int32_t* prim_ids,
                  int n, const float* q, int nq, float radius, int32_t* counts,
                  const int64_t* offsets, uint64_t* keys, int threads);

/* ---- brute force (src/cpu/brute.cpp) ---- */
void qo_raycast_brute(const float* tris, int n, const float* rays, int nrays, uint64_t* out);
void qo_closest_brute(int kind, const float* items, int n, const float* q, int nq,
                      uint32_t* out2);
void qo_knn_brute(int kind, const float* items, int n, const float* q, int nq, int k,
                  uint32_t* out2);

/* ---- fingerprints (src/core/fingerprint.h) ---- */
uint64_t qo_ray_hash(const uint64_t* res, int64_t n, uint64_t* hits);
uint64_t qo_closest_hash(const uint32_t* res2, int64_t n);
/* lists of stride k padded with id -1 (kNN output) */
uint64_t qo_knn_hash(const uint32_t* res2, int64_t n, int k);
uint64_t qo_radius_hash(const int64_t* offsets, const uint64_t* keys, int64_t n);
uint64_t qo_bytes_hash(const void* bytes, size_t len);

#ifdef __cplusplus
}
#endif

#endif
