// qk_traverse.cuh -- per-query stack traversals shared by the single-tree kernels
// (qk_query.cu) and the batched persistent kernels (qk_batch.cu).
//
// Each function runs one ray or query point through one tree to completion.  Binary nodes
// are 64-byte BNodes (both child boxes inline, four 16-byte loads); 4-wide nodes are 128-byte
// WideNodes.  Pruning follows the reference's rules exactly: the slab test with its 1e-6
// margins for rays, "bound <= best" for closest / kNN, "dist2 <= r2" for radius
// (src/gpu/raycast.cu:100-139, src/gpu/query.cu:74-116, 415-540), so every result is
// independent of tree shape and visit order.
//
// The stack is a template policy: LocalStack keeps every entry in local memory (the
// single-tree kernels), SplitStack keeps the first `sh` entries of every thread in shared
// memory (entry e of thread t at base[e * stride + t], conflict-free) and the rest in local
// memory -- the short-stack depth the batch autotuner chooses at run time.
#pragma once

#include "qk_internal.cuh"

namespace qk {

struct Trav {
    int nodes = 0;
    int leaves = 0;
    bool overflow = false;
};

// Per-thread stack in local memory: entry i is the pair (node, key bits), so a push is one
// 8-byte store and get() one 8-byte load.
template <int kCap>
struct LocalStack {
    static constexpr int kSize = kCap;
    int2 e[kCap];
    __device__ __forceinline__ void put(int i, int n, float k) { e[i] = make_int2(n, __float_as_int(k)); }
    __device__ __forceinline__ void put_node(int i, int n) { e[i].x = n; }
    __device__ __forceinline__ int get_node(int i) const { return e[i].x; }
    __device__ __forceinline__ float get_key(int i) const { return __int_as_float(e[i].y); }
    __device__ __forceinline__ void get(int i, int& n, float& k) const {
        const int2 v = e[i];
        n = v.x;
        k = __int_as_float(v.y);
    }
};

template <int kCap>
struct SplitStack {
    static constexpr int kSize = kCap;
    int* snode;   // this thread's column of the shared-memory part
    float* skey;
    int sh;       // entries kept in shared memory
    int stride;   // threads per block
    int node[kCap];
    float key[kCap];
    __device__ __forceinline__ void put(int i, int n, float k) {
        if (i < sh) {
            snode[i * stride] = n;
            skey[i * stride] = k;
        } else {
            node[i] = n;
            key[i] = k;
        }
    }
    __device__ __forceinline__ void put_node(int i, int n) {
        if (i < sh) snode[i * stride] = n;
        else node[i] = n;
    }
    __device__ __forceinline__ int get_node(int i) const { return i < sh ? snode[i * stride] : node[i]; }
    __device__ __forceinline__ float get_key(int i) const { return i < sh ? skey[i * stride] : key[i]; }
    __device__ __forceinline__ void get(int i, int& n, float& k) const {
        n = get_node(i);
        k = get_key(i);
    }
};

// ---------------------------------------------------------------------------------------
// node and leaf loads
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void load_bnode(const BNode* __restrict__ bn, int i, float3& llo,
                                           float3& lhi, float3& rlo, float3& rhi, int& lref,
                                           int& rref) {
    const float4* p = reinterpret_cast<const float4*>(bn + i);
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    llo = f3(a.x, a.y, a.z);
    lhi = f3(a.w, b.x, b.y);
    rlo = f3(b.z, b.w, c.x);
    rhi = f3(c.y, c.z, c.w);
    lref = __float_as_int(d.x);
    rref = __float_as_int(d.y);
}

// load_bnode plus the children's small-subtree codes (v3.z / v3.w): 0, or (first slot << 2)
// | (leaves - 1) for a child subtree of 2..4 leaves on contiguous slots
__device__ __forceinline__ void load_bnode_small(const BNode* __restrict__ bn, int i, float3& llo,
                                                 float3& lhi, float3& rlo, float3& rhi,
                                                 int& lref, int& rref, int& lsm, int& rsm) {
    const float4* p = reinterpret_cast<const float4*>(bn + i);
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    llo = f3(a.x, a.y, a.z);
    lhi = f3(a.w, b.x, b.y);
    rlo = f3(b.z, b.w, c.x);
    rhi = f3(c.y, c.z, c.w);
    lref = __float_as_int(d.x);
    rref = __float_as_int(d.y);
    lsm = __float_as_int(d.z);
    rsm = __float_as_int(d.w);
}

// box of the leaf in slot s; lnodes = the canonical nodes of the leaves (nodes + n - 1)
__device__ __forceinline__ Box leaf_box(const Node* __restrict__ lnodes, int s) {
    const float4* p = reinterpret_cast<const float4*>(lnodes + s);
    const float4 a = __ldg(p), b = __ldg(p + 1);
    Box bx;
    bx.lo = f3(a.x, a.y, a.z);
    bx.hi = f3(a.w, b.x, b.y);
    return bx;
}

__device__ __forceinline__ Box root_box(const Node* __restrict__ nodes) {
    const float4* p = reinterpret_cast<const float4*>(nodes);
    const float4 a = __ldg(p), b = __ldg(p + 1);
    Box bx;
    bx.lo = f3(a.x, a.y, a.z);
    bx.hi = f3(a.w, b.x, b.y);
    return bx;
}

// slot s of wide node `node`: box, child and the slot's primitive count -- max(pad, 1): 1 for
// every leaf slot of quarry's form (pad 0), up to 4 for a leaf range of the leaf-size-4 form
// (the primitives on slots ~child .. ~child + count - 1); meaningless for internal slots.  The
// traversals read the count only when instantiated for the leaf-size-4 form (kRange).
__device__ __forceinline__ void load_wide_entry(const WideNode* __restrict__ w, int node, int s,
                                                float3& lo, float3& hi, int& child, int& count) {
    const float4* p = reinterpret_cast<const float4*>(w + node) + 2 * s;
    const float4 a = __ldg(p), b = __ldg(p + 1);
    lo = f3(a.x, a.y, a.z);
    hi = f3(a.w, b.x, b.y);
    child = __float_as_int(b.z);
    count = max(__float_as_int(b.w), 1);
}

// statistics: warp-aggregated counters (src/gpu/raycast.cu:147-156)
template <bool kStats>
__device__ __forceinline__ void flush_stats(bool active, int nodes, int leaves, bool overflow,
                                            unsigned long long* stats) {
    if (stats == nullptr) return;
    const unsigned mask = __ballot_sync(0xffffffffu, active);
    const unsigned ovf = __ballot_sync(0xffffffffu, overflow);
    if (kStats) {
        const int sn = __reduce_add_sync(0xffffffffu, nodes);
        const int sl = __reduce_add_sync(0xffffffffu, leaves);
        if ((threadIdx.x & 31) == 0 && mask) {
            if (sn) atomicAdd(stats + 0, static_cast<unsigned long long>(sn));
            if (sl) atomicAdd(stats + 1, static_cast<unsigned long long>(sl));
        }
    }
    if ((threadIdx.x & 31) == 0 && ovf) atomicAdd(stats + 2, static_cast<unsigned long long>(__popc(ovf)));
}

// ---------------------------------------------------------------------------------------
// rays
// ---------------------------------------------------------------------------------------
// Leaf test.  The first hit is taken even at t == tMax (the CPU reference accepts t <= tMax,
// src/cpu/bvh.cpp:156-168); later hits only when closer.  Among hits at the same t the
// smallest scene index is kept, so the reported primitive does not depend on visit order.
template <int kMode = -1>
__device__ __forceinline__ void test_tri(const RayPre& R, const float4* __restrict__ leaves,
                                         int slot, float& best, float& bound, bool& any,
                                         int& best_id) {
    const float4 a = __ldg(leaves + 3 * slot), b = __ldg(leaves + 3 * slot + 1),
                 c = __ldg(leaves + 3 * slot + 2);
    float t;
    if (ray_tri<kMode>(R, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), f3(c.x, c.y, c.z), t)) {
        const int id = __float_as_int(a.w);
        if (!any || t < best || (t == best && id < best_id)) {
            best = t;
            bound = best * kMarginMul + kMarginAdd;
            any = true;
            best_id = id;
        }
    }
}

__device__ __forceinline__ unsigned long long pack_hit(bool any, float best) {
    return any ? ((1ull << 32) | static_cast<unsigned long long>(__float_as_uint(best))) : 0ull;
}

// First hit in a binary tree: near child followed, far child pushed with its entry bound,
// which is re-checked against the current best when popped (src/cpu/bvh.cpp:147-152).
// kMode >= 0: the ray's RayPre::mode, known at compile time (the slab tests drop their
// branch on parallel axes and use min / max); -1 for any ray.
template <class St, bool kLeaf4 = false, int kMode = -1>
__device__ __forceinline__ unsigned long long ray_bin_one(const BNode* __restrict__ bn,
                                                          const float4* __restrict__ leaves,
                                                          const Box& rb, const RayPre& R,
                                                          int max_iter, St& st, Trav& tv,
                                                          int& best_id,
                                                          const Node* __restrict__ lnodes = nullptr) {
    float best = R.tmax;
    float bound = best * kMarginMul + kMarginAdd;
    bool any = false;
    best_id = -1;
    float te;
    if (!ray_box<kMode>(R, rb.lo, rb.hi, bound, te)) return 0ull;
    ++tv.nodes;
    int sp = 0;
    int node = 0;
    for (int iter = 0;; ++iter) {
        if (iter >= max_iter) {
            tv.overflow = true;
            break;
        }
        float3 llo, lhi, rlo, rhi;
        int lref, rref, lsm = 0, rsm = 0;
        if constexpr (kLeaf4) load_bnode_small(bn, node, llo, lhi, rlo, rhi, lref, rref, lsm, rsm);
        else load_bnode(bn, node, llo, lhi, rlo, rhi, lref, rref);
        float tl, tr;
        bool hl = ray_box<kMode>(R, llo, lhi, bound, tl);
        bool hr = ray_box<kMode>(R, rlo, rhi, bound, tr);
        tv.nodes += static_cast<int>(hl) + static_cast<int>(hr);
        if (hl && lref < 0) {
            ++tv.leaves;
            test_tri<kMode>(R, leaves, ~lref, best, bound, any, best_id);
            hl = false;
        }
        if (hr && rref < 0) {
            ++tv.leaves;
            test_tri<kMode>(R, leaves, ~rref, best, bound, any, best_id);
            hr = false;
        }
        if constexpr (kLeaf4) {
            // subtrees of 2..4 triangles: test them now, the nearer first, the farther only
            // while its entry still passes the current bound
            const bool sl = hl && lsm != 0, sr = hr && rsm != 0;
            if (sl || sr) {
                const bool lnear = tl <= tr;
#pragma unroll
                for (int pass = 0; pass < 2; ++pass) {
                    const bool left = (pass == 0) == lnear;
                    const int code = left ? (sl ? lsm : 0) : (sr ? rsm : 0);
                    const float te = left ? tl : tr;
                    if (code && !(te > bound * kMarginMul + kMarginAdd)) {
                        const int first = code >> 2, cnt = (code & 3) + 1;
                        for (int j = 0; j < cnt; ++j) {
                            // the leaf's own box first, as a descent would test it
                            const Box lb = leaf_box(lnodes, first + j);
                            float tb;
                            if (!ray_box<kMode>(R, lb.lo, lb.hi, bound, tb)) continue;
                            ++tv.leaves;
                            test_tri<kMode>(R, leaves, first + j, best, bound, any, best_id);
                        }
                    }
                }
                if (sl) hl = false;
                if (sr) hr = false;
            }
        }
        if (hl && hr) {
            const bool lnear = tl <= tr;
            if (sp >= St::kSize) {
                tv.overflow = true;
                break;
            }
            st.put(sp, lnear ? rref : lref, lnear ? tr : tl);
            ++sp;
            node = lnear ? lref : rref;
        } else if (hl) {
            node = lref;
        } else if (hr) {
            node = rref;
        } else {
            // pop the next entry whose box could still hold a closer hit
            const float limit = bound * kMarginMul + kMarginAdd;
            node = -1;
            while (sp > 0) {
                --sp;
                int pn;
                float pk;
                st.get(sp, pn, pk);
                if (!(pk > limit)) {
                    node = pn;
                    break;
                }
            }
            if (node < 0) break;
        }
    }
    return pack_hit(any, best);
}

// First hit in a 4-wide tree: hit slots sorted by entry t, leaves tested nearest first,
// the nearest internal child followed and the others pushed far-first.
template <bool kRange = false, int kMode = -1, class St>
__device__ __forceinline__ unsigned long long ray_wide_one(const WideNode* __restrict__ wn,
                                                           const float4* __restrict__ leaves,
                                                           const RayPre& R, int max_iter, St& st,
                                                           Trav& tv, int& best_id) {
    float best = R.tmax;
    float bound = best * kMarginMul + kMarginAdd;
    bool any = false;
    best_id = -1;
    int sp = 0;
    int node = 0;  // the 4-wide root has no single box; start inside it (raycast.cu:182)
    for (int iter = 0;; ++iter) {
        if (iter >= max_iter) {
            tv.overflow = true;
            break;
        }
        int child[4], cnt[4];
        float key[4];
        int hits = 0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            float3 lo, hi;
            int c, nc;
            load_wide_entry(wn, node, s, lo, hi, c, nc);
            float t;
            if (c != kEmptySlot && ray_box<kMode>(R, lo, hi, bound, t)) {
                ++tv.nodes;
                int j = hits++;
                while (j > 0 && key[j - 1] > t) {
                    key[j] = key[j - 1];
                    child[j] = child[j - 1];
                    if (kRange) cnt[j] = cnt[j - 1];
                    --j;
                }
                key[j] = t;
                child[j] = c;
                if (kRange) cnt[j] = nc;
            }
        }
        int next = -1;
        float nextT = 0.0f;
        for (int j = 0; j < hits; ++j) {
            if (child[j] < 0) {
                const int nq = kRange ? cnt[j] : 1;
                for (int q = 0; q < nq; ++q) {
                    ++tv.leaves;
                    test_tri<kMode>(R, leaves, ~child[j] + q, best, bound, any, best_id);
                }
            }
        }
        for (int j = hits - 1; j >= 0; --j) {
            if (child[j] < 0) continue;
            if (next >= 0) {
                if (sp >= St::kSize) {
                    tv.overflow = true;
                    break;
                }
                st.put(sp, next, nextT);
                ++sp;
            }
            next = child[j];
            nextT = key[j];
        }
        if (tv.overflow) break;
        if (next >= 0) {
            node = next;
            continue;
        }
        const float limit = bound * kMarginMul + kMarginAdd;
        node = -1;
        while (sp > 0) {
            --sp;
            int pn;
            float pk;
            st.get(sp, pn, pk);
            if (!(pk > limit)) {
                node = pn;
                break;
            }
        }
        if (node < 0) break;
    }
    return pack_hit(any, best);
}

// ---------------------------------------------------------------------------------------
// closest
// ---------------------------------------------------------------------------------------
template <class Ops>
__device__ __forceinline__ void leaf_closest(float3 p, const float4* __restrict__ leaves, int slot,
                                             float& best, int& best_id) {
    int id;
    const float d2 = Ops::dist2(p, leaves, slot, id);
    if (best_id < 0 || closer(d2, id, best, best_id)) {
        best = d2;
        best_id = id;
    }
}

__device__ __forceinline__ uint2 pack_closest(float best, int best_id) {
    return best_id >= 0 ? make_uint2(__float_as_uint(best), static_cast<unsigned>(best_id))
                        : make_uint2(0u, 0xffffffffu);
}

template <class Ops, class St, bool kLeaf4 = false>
__device__ __forceinline__ uint2 closest_bin_one(const BNode* __restrict__ bn,
                                                 const float4* __restrict__ leaves, float3 p,
                                                 int max_iter, St& st, Trav& tv,
                                                 const Node* __restrict__ lnodes = nullptr) {
    float best = kInf;
    int best_id = -1;
    int sp = 0;
    int node = 0;
    for (int iter = 0;; ++iter) {
        if (iter >= max_iter) {
            tv.overflow = true;
            break;
        }
        ++tv.nodes;
        float3 llo, lhi, rlo, rhi;
        int lref, rref, lsm = 0, rsm = 0;
        if constexpr (kLeaf4) load_bnode_small(bn, node, llo, lhi, rlo, rhi, lref, rref, lsm, rsm);
        else load_bnode(bn, node, llo, lhi, rlo, rhi, lref, rref);
        const float dl = dist2_box(p, llo, lhi);
        const float dr = dist2_box(p, rlo, rhi);
        bool okl = best_id < 0 || dl <= best;
        bool okr = best_id < 0 || dr <= best;
        // leaves in near-first order so the second sees the tighter bound
        const bool lfirst = dl <= dr;
        if (lfirst) {
            if (okl && lref < 0) { ++tv.leaves; leaf_closest<Ops>(p, leaves, ~lref, best, best_id); okl = false; }
            if (okr && rref < 0 && (best_id < 0 || dr <= best)) { ++tv.leaves; leaf_closest<Ops>(p, leaves, ~rref, best, best_id); }
            if (rref < 0) okr = false;
        } else {
            if (okr && rref < 0) { ++tv.leaves; leaf_closest<Ops>(p, leaves, ~rref, best, best_id); okr = false; }
            if (okl && lref < 0 && (best_id < 0 || dl <= best)) { ++tv.leaves; leaf_closest<Ops>(p, leaves, ~lref, best, best_id); }
            if (lref < 0) okl = false;
        }
        if constexpr (kLeaf4) {
            const bool sl = okl && lsm != 0, sr = okr && rsm != 0;
            if (sl || sr) {
#pragma unroll
                for (int pass = 0; pass < 2; ++pass) {
                    const bool left = (pass == 0) == lfirst;
                    const int code = left ? (sl ? lsm : 0) : (sr ? rsm : 0);
                    const float dbox = left ? dl : dr;
                    if (code && (best_id < 0 || dbox <= best)) {
                        const int first = code >> 2, cnt = (code & 3) + 1;
                        for (int j = 0; j < cnt; ++j) {
                            const Box lb = leaf_box(lnodes, first + j);
                            if (!(best_id < 0 || dist2_box(p, lb.lo, lb.hi) <= best)) continue;
                            ++tv.leaves;
                            leaf_closest<Ops>(p, leaves, first + j, best, best_id);
                        }
                    }
                }
                if (sl) okl = false;
                if (sr) okr = false;
            }
        }
        if (okl && okr) {
            if (sp >= St::kSize) {
                tv.overflow = true;
                break;
            }
            st.put(sp, lfirst ? rref : lref, lfirst ? dr : dl);
            ++sp;
            node = lfirst ? lref : rref;
        } else if (okl) {
            node = lref;
        } else if (okr) {
            node = rref;
        } else {
            node = -1;
            while (sp > 0) {
                --sp;
                int pn;
                float pk;
                st.get(sp, pn, pk);
                if (best_id < 0 || pk <= best) {
                    node = pn;
                    break;
                }
            }
            if (node < 0) break;
        }
    }
    return pack_closest(best, best_id);
}

template <class Ops, bool kRange = false, class St>
__device__ __forceinline__ uint2 closest_wide_one(const WideNode* __restrict__ wn,
                                                  const float4* __restrict__ leaves, float3 p,
                                                  int max_iter, St& st, Trav& tv) {
    float best = kInf;
    int best_id = -1;
    int sp = 0;
    int node = 0;
    for (int iter = 0;; ++iter) {
        if (iter >= max_iter) {
            tv.overflow = true;
            break;
        }
        int child[4], cnt[4];
        float key[4];
        int hits = 0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            float3 lo, hi;
            int c, nc;
            load_wide_entry(wn, node, s, lo, hi, c, nc);
            if (c == kEmptySlot) continue;
            const float d = dist2_box(p, lo, hi);
            if (best_id >= 0 && d > best) continue;
            ++tv.nodes;
            int j = hits++;
            while (j > 0 && key[j - 1] > d) {
                key[j] = key[j - 1];
                child[j] = child[j - 1];
                if (kRange) cnt[j] = cnt[j - 1];
                --j;
            }
            key[j] = d;
            child[j] = c;
            if (kRange) cnt[j] = nc;
        }
        for (int j = 0; j < hits; ++j) {
            if (child[j] < 0 && (best_id < 0 || key[j] <= best)) {
                const int nq = kRange ? cnt[j] : 1;
                for (int q = 0; q < nq; ++q) {
                    ++tv.leaves;
                    leaf_closest<Ops>(p, leaves, ~child[j] + q, best, best_id);
                }
            }
        }
        int next = -1;
        float nextD = 0.0f;
        for (int j = hits - 1; j >= 0; --j) {
            if (child[j] < 0) continue;
            if (best_id >= 0 && key[j] > best) continue;
            if (next >= 0) {
                if (sp >= St::kSize) {
                    tv.overflow = true;
                    break;
                }
                st.put(sp, next, nextD);
                ++sp;
            }
            next = child[j];
            nextD = key[j];
        }
        if (tv.overflow) break;
        if (next >= 0) {
            node = next;
            continue;
        }
        node = -1;
        while (sp > 0) {
            --sp;
            int pn;
            float pk;
            st.get(sp, pn, pk);
            if (best_id < 0 || pk <= best) {
                node = pn;
                break;
            }
        }
        if (node < 0) break;
    }
    return pack_closest(best, best_id);
}

// ---------------------------------------------------------------------------------------
// kNN: the k best (dist2, id) pairs stay sorted in registers (unrolled insertion over a
// compile-time capacity K >= k).  Empty slots hold (+inf, INT_MAX), so "strictly closer than
// the k-th" is one comparison whether or not the table is full -- the reference's max-heap
// replacement rule (src/cpu/bvh.cpp:284-299, src/gpu/query.cu:145-158).
// ---------------------------------------------------------------------------------------
template <int K>
struct KnnTable {
    float d[K];
    int id[K];
    float kd;  // dist2 of entry k-1 (the pruning threshold)
    int kid;

    __device__ __forceinline__ void init() {
#pragma unroll
        for (int j = 0; j < K; ++j) {
            d[j] = kInf;
            id[j] = 0x7fffffff;
        }
        kd = kInf;
        kid = 0x7fffffff;
    }
    __device__ __forceinline__ void insert(float xd, int xid, int k) {
        if (!closer(xd, xid, kd, kid)) return;
#pragma unroll
        for (int j = K - 1; j > 0; --j) {
            const bool shift = closer(xd, xid, d[j - 1], id[j - 1]);
            const bool place = !shift && closer(xd, xid, d[j], id[j]);
            const float nd = shift ? d[j - 1] : (place ? xd : d[j]);
            const int ni = shift ? id[j - 1] : (place ? xid : id[j]);
            d[j] = nd;
            id[j] = ni;
        }
        if (closer(xd, xid, d[0], id[0])) {
            d[0] = xd;
            id[0] = xid;
        }
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (j == k - 1) {
                kd = d[j];
                kid = id[j];
            }
        }
    }
    // prune test for a subtree bound: keep while the table is not full or bound <= k-th
    __device__ __forceinline__ bool admits(float bound) const { return kid == 0x7fffffff || bound <= kd; }
};

template <class Ops, int K>
__device__ __forceinline__ void leaf_knn(float3 p, const float4* __restrict__ leaves, int slot,
                                         KnnTable<K>& tab, int k) {
    int id;
    const float d2 = Ops::dist2(p, leaves, slot, id);
    tab.insert(d2, id, k);
}

template <int K>
__device__ __forceinline__ void write_knn(const KnnTable<K>& tab, int k, uint2* __restrict__ dst) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
        if (j < k) {
            const bool valid = tab.id[j] != 0x7fffffff;
            dst[j] = valid ? make_uint2(__float_as_uint(tab.d[j]), static_cast<unsigned>(tab.id[j]))
                           : make_uint2(0u, 0xffffffffu);
        }
    }
}

template <class Ops, int K, class St, bool kLeaf4 = false>
__device__ __forceinline__ void knn_bin_one(const BNode* __restrict__ bn,
                                            const float4* __restrict__ leaves, float3 p, int k,
                                            int max_iter, St& st, Trav& tv, KnnTable<K>& tab,
                                            const Node* __restrict__ lnodes = nullptr) {
    tab.init();
    int sp = 0;
    int node = 0;
    for (int iter = 0;; ++iter) {
        if (iter >= max_iter) {
            tv.overflow = true;
            break;
        }
        ++tv.nodes;
        float3 llo, lhi, rlo, rhi;
        int lref, rref, lsm = 0, rsm = 0;
        if constexpr (kLeaf4) load_bnode_small(bn, node, llo, lhi, rlo, rhi, lref, rref, lsm, rsm);
        else load_bnode(bn, node, llo, lhi, rlo, rhi, lref, rref);
        const float dl = dist2_box(p, llo, lhi);
        const float dr = dist2_box(p, rlo, rhi);
        const bool lfirst = dl <= dr;
        bool okl = tab.admits(dl);
        bool okr = tab.admits(dr);
        if (lfirst) {
            if (okl && lref < 0) { ++tv.leaves; leaf_knn<Ops, K>(p, leaves, ~lref, tab, k); okl = false; }
            if (okr && rref < 0 && tab.admits(dr)) { ++tv.leaves; leaf_knn<Ops, K>(p, leaves, ~rref, tab, k); }
            if (rref < 0) okr = false;
        } else {
            if (okr && rref < 0) { ++tv.leaves; leaf_knn<Ops, K>(p, leaves, ~rref, tab, k); okr = false; }
            if (okl && lref < 0 && tab.admits(dl)) { ++tv.leaves; leaf_knn<Ops, K>(p, leaves, ~lref, tab, k); }
            if (lref < 0) okl = false;
        }
        if constexpr (kLeaf4) {
            const bool sl = okl && lsm != 0, sr = okr && rsm != 0;
            if (sl || sr) {
#pragma unroll
                for (int pass = 0; pass < 2; ++pass) {
                    const bool left = (pass == 0) == lfirst;
                    const int code = left ? (sl ? lsm : 0) : (sr ? rsm : 0);
                    const float dbox = left ? dl : dr;
                    if (code && tab.admits(dbox)) {
                        const int first = code >> 2, cnt = (code & 3) + 1;
                        for (int j = 0; j < cnt; ++j) {
                            const Box lb = leaf_box(lnodes, first + j);
                            if (!tab.admits(dist2_box(p, lb.lo, lb.hi))) continue;
                            ++tv.leaves;
                            leaf_knn<Ops, K>(p, leaves, first + j, tab, k);
                        }
                    }
                }
                if (sl) okl = false;
                if (sr) okr = false;
            }
        }
        if (okl && okr) {
            if (sp >= St::kSize) {
                tv.overflow = true;
                break;
            }
            st.put(sp, lfirst ? rref : lref, lfirst ? dr : dl);
            ++sp;
            node = lfirst ? lref : rref;
        } else if (okl) {
            node = lref;
        } else if (okr) {
            node = rref;
        } else {
            node = -1;
            while (sp > 0) {
                --sp;
                int pn;
                float pk;
                st.get(sp, pn, pk);
                if (tab.admits(pk)) {
                    node = pn;
                    break;
                }
            }
            if (node < 0) break;
        }
    }
}

template <class Ops, int K, bool kRange = false, class St>
__device__ __forceinline__ void knn_wide_one(const WideNode* __restrict__ wn,
                                             const float4* __restrict__ leaves, float3 p, int k,
                                             int max_iter, St& st, Trav& tv, KnnTable<K>& tab) {
    tab.init();
    int sp = 0;
    int node = 0;
    for (int iter = 0;; ++iter) {
        if (iter >= max_iter) {
            tv.overflow = true;
            break;
        }
        int child[4], cnt[4];
        float key[4];
        int hits = 0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            float3 lo, hi;
            int c, nc;
            load_wide_entry(wn, node, s, lo, hi, c, nc);
            if (c == kEmptySlot) continue;
            const float d = dist2_box(p, lo, hi);
            if (!tab.admits(d)) continue;
            ++tv.nodes;
            int j = hits++;
            while (j > 0 && key[j - 1] > d) {
                key[j] = key[j - 1];
                child[j] = child[j - 1];
                if (kRange) cnt[j] = cnt[j - 1];
                --j;
            }
            key[j] = d;
            child[j] = c;
            if (kRange) cnt[j] = nc;
        }
        for (int j = 0; j < hits; ++j) {
            if (child[j] < 0 && tab.admits(key[j])) {
                const int nq = kRange ? cnt[j] : 1;
                for (int q = 0; q < nq; ++q) {
                    ++tv.leaves;
                    leaf_knn<Ops, K>(p, leaves, ~child[j] + q, tab, k);
                }
            }
        }
        int next = -1;
        float nextD = 0.0f;
        for (int j = hits - 1; j >= 0; --j) {
            if (child[j] < 0 || !tab.admits(key[j])) continue;
            if (next >= 0) {
                if (sp >= St::kSize) {
                    tv.overflow = true;
                    break;
                }
                st.put(sp, next, nextD);
                ++sp;
            }
            next = child[j];
            nextD = key[j];
        }
        if (tv.overflow) break;
        if (next >= 0) {
            node = next;
            continue;
        }
        node = -1;
        while (sp > 0) {
            --sp;
            int pn;
            float pk;
            st.get(sp, pn, pk);
            if (tab.admits(pk)) {
                node = pn;
                break;
            }
        }
        if (node < 0) break;
    }
}

// ---------------------------------------------------------------------------------------
// radius: a box is entered when its squared distance <= r2, a primitive kept when its
// dist2 <= r2 (src/gpu/query.cu:415-540).  The fill pass writes (bits(d2) << 32 | id) keys
// from `write` on and never past `end`; both passes return the number found.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long radius_key(float d2, int id) {
    return (static_cast<unsigned long long>(__float_as_uint(d2)) << 32) | static_cast<unsigned>(id);
}

// Where a radius traversal puts its keys.  SegmentSink: the query's CSR segment
// keys[write, end) (the fill pass), never past its end.
struct SegmentSink {
    unsigned long long* keys;
    int write;
    int end;
    __device__ __forceinline__ void put(unsigned long long k) {
        if (write < end) keys[write++] = k;
    }
};

// PoolSink: the single-pass radius (QK_TUNE_STASH).  A query's first kRadiusStash keys go to
// its stash slots, later ones to chunks of kPoolChunk keys taken from a shared pool (one
// atomic per chunk) and chained per query: *first holds the query's first chunk, next[c] the
// chunk after c; the chain's length follows from the query's count, so it needs no end mark.
// When the pool runs out, *first becomes kPoolLost and the query's later keys are dropped;
// the fill pass traverses such a query again.  Only the thread that owns the query writes its
// stash, its *first and its chain links.
constexpr int kRadiusStash = 16;
constexpr int kPoolChunk = 32;
constexpr int kPoolLost = -2;

// The single-pass radius's buffers for `count` queries, carved from a workspace: the stash
// (kRadiusStash keys per query), the chain heads, the chunk counter, the chain links and the
// pool itself (kPoolPerQuery keys per query on average, shared by all queries).
constexpr int kPoolPerQuery = 128;

struct RadiusPool {
    unsigned long long* stash;
    int* first;
    int* taken;
    int* next;
    unsigned long long* keys;
    int chunks;
};

inline RadiusPool carve_pool(Carve& c, int count, int per_query = kPoolPerQuery) {
    RadiusPool p{};
    p.chunks = static_cast<int>((static_cast<long long>(count) * per_query + kPoolChunk - 1) /
                                kPoolChunk);
    p.stash = c.take<unsigned long long>(static_cast<size_t>(count) * kRadiusStash);
    p.first = c.take<int>(count);
    p.taken = c.take<int>(1);
    p.next = c.take<int>(p.chunks);
    p.keys = c.take<unsigned long long>(static_cast<size_t>(p.chunks) * kPoolChunk);
    return p;
}

struct PoolSink {
    unsigned long long* stash;   // this query's kRadiusStash slots
    unsigned long long* pool;    // chunks of kPoolChunk keys
    int* next;                   // chain links, one per chunk
    int* taken;                  // chunks handed out so far (shared counter)
    int chunks;                  // pool capacity in chunks
    int* first;                  // this query's first chunk, or kPoolLost
    int n;                       // keys seen so far
    int cur;                     // the chunk being filled, or kPoolLost
    __device__ __forceinline__ void put(unsigned long long k) {
        if (n < kRadiusStash) {
            stash[n++] = k;
            return;
        }
        const int j = (n - kRadiusStash) & (kPoolChunk - 1);
        const bool fresh = n == kRadiusStash;
        ++n;
        if (cur == kPoolLost) return;
        if (j == 0) {
            const int c = atomicAdd(taken, 1);
            if (c >= chunks) {
                cur = kPoolLost;
                *first = kPoolLost;
                return;
            }
            if (fresh) *first = c;
            else next[cur] = c;
            cur = c;
        }
        pool[static_cast<size_t>(cur) * kPoolChunk + j] = k;
    }
};

// Copies query q's keys (its stash, then its pool chain) into keys[begin, begin + cnt), one
// warp per query: lane l moves entry l of the stash and of every 32-key chunk, so the reads and
// writes are coalesced.  Every lane of the warp calls it for the same q.
static_assert(kPoolChunk == 32, "a pool chunk is one key per lane");
__device__ __forceinline__ void copy_pooled_warp(const RadiusPool& pool, int q, int begin, int cnt,
                                                 unsigned long long* __restrict__ keys, int lane) {
    const int head = cnt < kRadiusStash ? cnt : kRadiusStash;
    if (lane < head) keys[begin + lane] = pool.stash[static_cast<size_t>(q) * kRadiusStash + lane];
    int left = cnt - head;
    int w = begin + head;
    int c = left > 0 ? pool.first[q] : -1;
    while (left > 0) {
        const int m = left < kPoolChunk ? left : kPoolChunk;
        if (lane < m) keys[w + lane] = pool.keys[static_cast<size_t>(c) * kPoolChunk + lane];
        w += m;
        left -= m;
        if (left > 0) c = pool.next[c];
    }
}

// The copy pass of the single-pass radius: one warp per query whose keys the pool held (the
// others are traversed again); skipped, as the fill is, when offsets[count] exceeds cap (cap <
// 0: no limit).
static __global__ __launch_bounds__(256) void k_radius_gather(RadiusPool pool,
                                                       const int* __restrict__ offsets, int count,
                                                       unsigned long long* __restrict__ keys,
                                                       long long cap) {
    const int q = static_cast<int>((static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= count) return;
    if (cap >= 0 && static_cast<long long>(offsets[count]) > cap) return;
    const int begin = offsets[q], n = offsets[q + 1] - begin;
    if (n > kRadiusStash && pool.first[q] == kPoolLost) return;
    copy_pooled_warp(pool, q, begin, n, keys, lane);
}

template <class Ops, bool kFill, class St, bool kLeaf4, class Sink>
__device__ __forceinline__ int radius_bin_visit(const BNode* __restrict__ bn,
                                                const float4* __restrict__ leaves, const Box& rb,
                                                float3 p, float r2, Sink& sink, int max_iter,
                                                St& st, Trav& tv,
                                                const Node* __restrict__ lnodes = nullptr) {
    int found = 0;
    if (!(dist2_box(p, rb.lo, rb.hi) <= r2)) return 0;
    int sp = 0;
    int node = 0;
    for (int iter = 0;; ++iter) {
        if (iter >= max_iter) {
            tv.overflow = true;
            break;
        }
        ++tv.nodes;
        float3 llo, lhi, rlo, rhi;
        int lref, rref, lsm = 0, rsm = 0;
        if constexpr (kLeaf4) load_bnode_small(bn, node, llo, lhi, rlo, rhi, lref, rref, lsm, rsm);
        else load_bnode(bn, node, llo, lhi, rlo, rhi, lref, rref);
        bool okl = dist2_box(p, llo, lhi) <= r2;
        bool okr = dist2_box(p, rlo, rhi) <= r2;
        if (okl && lref < 0) {
            ++tv.leaves;
            int id;
            const float d2 = Ops::dist2(p, leaves, ~lref, id);
            if (d2 <= r2) {
                if (kFill) sink.put(radius_key(d2, id));
                ++found;
            }
            okl = false;
        }
        if (okr && rref < 0) {
            ++tv.leaves;
            int id;
            const float d2 = Ops::dist2(p, leaves, ~rref, id);
            if (d2 <= r2) {
                if (kFill) sink.put(radius_key(d2, id));
                ++found;
            }
            okr = false;
        }
        if constexpr (kLeaf4) {
#pragma unroll
            for (int pass = 0; pass < 2; ++pass) {
                const int code = pass == 0 ? (okl ? lsm : 0) : (okr ? rsm : 0);
                if (code) {
                    const int first = code >> 2, cnt = (code & 3) + 1;
                    for (int j = 0; j < cnt; ++j) {
                        const Box lb = leaf_box(lnodes, first + j);
                        if (!(dist2_box(p, lb.lo, lb.hi) <= r2)) continue;
                        ++tv.leaves;
                        int id;
                        const float d2 = Ops::dist2(p, leaves, first + j, id);
                        if (d2 <= r2) {
                            if (kFill) sink.put(radius_key(d2, id));
                            ++found;
                        }
                    }
                }
            }
            if (lsm) okl = false;
            if (rsm) okr = false;
        }
        if (okl && okr) {
            if (sp >= St::kSize) {
                tv.overflow = true;
                break;
            }
            st.put_node(sp++, rref);
            node = lref;
        } else if (okl) {
            node = lref;
        } else if (okr) {
            node = rref;
        } else {
            if (sp == 0) break;
            node = st.get_node(--sp);
        }
    }
    return found;
}

template <class Ops, bool kFill, class St, bool kLeaf4 = false>
__device__ __forceinline__ int radius_bin_one(const BNode* __restrict__ bn,
                                              const float4* __restrict__ leaves, const Box& rb,
                                              float3 p, float r2, int write, int end,
                                              unsigned long long* __restrict__ keys,
                                              int max_iter, St& st, Trav& tv,
                                              const Node* __restrict__ lnodes = nullptr) {
    SegmentSink sink{keys, write, end};
    return radius_bin_visit<Ops, kFill, St, kLeaf4>(bn, leaves, rb, p, r2, sink, max_iter, st, tv,
                                                    lnodes);
}

template <class Ops, bool kFill, bool kRange = false, class St, class Sink>
__device__ __forceinline__ int radius_wide_visit(const WideNode* __restrict__ wn,
                                                 const float4* __restrict__ leaves, float3 p,
                                                 float r2, Sink& sink, int max_iter, St& st,
                                                 Trav& tv) {
    int found = 0;
    int sp = 0;
    int node = 0;
    for (int iter = 0;; ++iter) {
        if (iter >= max_iter) {
            tv.overflow = true;
            break;
        }
        int next = -1;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            float3 lo, hi;
            int c, nc;
            load_wide_entry(wn, node, s, lo, hi, c, nc);
            if (c == kEmptySlot || !(dist2_box(p, lo, hi) <= r2)) continue;
            ++tv.nodes;
            if (c < 0) {
                const int nq = kRange ? nc : 1;
                for (int q = 0; q < nq; ++q) {
                    ++tv.leaves;
                    int id;
                    const float d2 = Ops::dist2(p, leaves, ~c + q, id);
                    if (d2 <= r2) {
                        if (kFill) sink.put(radius_key(d2, id));
                        ++found;
                    }
                }
            } else if (next < 0) {
                next = c;
            } else if (sp < St::kSize) {
                st.put_node(sp++, c);
            } else {
                tv.overflow = true;
            }
        }
        if (tv.overflow) break;
        if (next >= 0) {
            node = next;
        } else {
            if (sp == 0) break;
            node = st.get_node(--sp);
        }
    }
    return found;
}

template <class Ops, bool kFill, bool kRange = false, class St>
__device__ __forceinline__ int radius_wide_one(const WideNode* __restrict__ wn,
                                               const float4* __restrict__ leaves, float3 p,
                                               float r2, int write, int end,
                                               unsigned long long* __restrict__ keys,
                                               int max_iter, St& st, Trav& tv) {
    SegmentSink sink{keys, write, end};
    return radius_wide_visit<Ops, kFill, kRange>(wn, leaves, p, r2, sink, max_iter, st, tv);
}

// ---------------------------------------------------------------------------------------
// split mode (QK_TUNE_SPLIT): one warp per query point.  The top kSplitLevels levels of the
// binary tree are descended with lane l taking child bit ((l >> level) & 1), so the 32 lanes
// own 32 disjoint subtrees (a leaf met on the way belongs to the lowest lane that reaches
// it); each lane then runs the ordinary depth-first traversal of its subtree.  After every
// step the warp shares its pruning bound by shuffles, so a query whose search touches much of
// the tree (a point near the centre of a spherical shell) is spread over 32 lanes.  The
// subtrees partition the leaves and the shared bound only ever comes from found candidates,
// so results equal the one-thread-per-query kernels bit for bit.
//
// Groups (QK_TUNE_SPLIT8 / QK_TUNE_SPLIT4): the same with G = 8 or 4 lanes per query, the top
// log2(G) levels split, every exchange restricted to the query's G aligned lanes (shuffle
// width G, the group's bits of each ballot).  Few queries then fill more of the GPU without
// 32-fold redundancy.  Warp-wide loop conditions keep every lane of the warp in the same
// collectives; a group past the last query traces query 0 and writes nothing.
// ---------------------------------------------------------------------------------------
constexpr int kSplitLevels = 5;

constexpr int log2_lanes(int g) { return g <= 1 ? 0 : 1 + log2_lanes(g / 2); }

// first lane of this thread's group of G lanes in its warp, and the group's ballot bits
template <int G>
__device__ __forceinline__ int group_base() { return (threadIdx.x & 31) & ~(G - 1); }
template <int G>
__device__ __forceinline__ unsigned group_bits(unsigned ballot) {
    return G == 32 ? ballot : (ballot >> group_base<G>()) & ((1u << G) - 1u);
}
template <int G>
__device__ __forceinline__ bool group_any(bool v) {
    return group_bits<G>(__ballot_sync(0xffffffffu, v)) != 0u;
}

template <int G = 32>
__device__ __forceinline__ void warp_min_lex(float& d, int& id) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
        const float od = __shfl_xor_sync(0xffffffffu, d, o);
        const int oi = __shfl_xor_sync(0xffffffffu, id, o);
        if (closer(od, oi, d, id)) {
            d = od;
            id = oi;
        }
    }
}

// Forced descent of lane `lane` from the root: returns the subtree root the lane owns (an
// internal node) or -1; a leaf met on the way is handed to `on_leaf` by its owning lane.
// `keep(box)` decides whether a child box can still hold a result.
template <int kLevels = kSplitLevels, class Leaf, class Keep>
__device__ __forceinline__ int split_descend(const BNode* __restrict__ bn, int lane, Leaf on_leaf,
                                             Keep keep) {
    int node = 0;
    for (int d = 0; d < kLevels; ++d) {
        float3 llo, lhi, rlo, rhi;
        int lref, rref;
        load_bnode(bn, node, llo, lhi, rlo, rhi, lref, rref);
        const bool right = ((lane >> d) & 1) != 0;
        const int ref = right ? rref : lref;
        const float3 lo = right ? rlo : llo;
        const float3 hi = right ? rhi : lhi;
        if (ref < 0) {
            if ((lane >> (d + 1)) == 0 && keep(lo, hi)) on_leaf(~ref);
            return -1;
        }
        if (!keep(lo, hi)) return -1;
        node = ref;
    }
    return node;
}

template <class Ops, int G = 32>
__device__ __forceinline__ uint2 closest_split_one(const BNode* __restrict__ bn,
                                                   const float4* __restrict__ leaves, float3 p,
                                                   int lane, int max_iter, Trav& tv,
                                                   bool valid = true) {
    float best = kInf;
    int best_id = 0x7fffffff;
    auto on_leaf = [&](int slot) {
        ++tv.leaves;
        int id;
        const float d2 = Ops::dist2(p, leaves, slot, id);
        if (closer(d2, id, best, best_id)) {
            best = d2;
            best_id = id;
        }
    };
    int node = valid ? split_descend<log2_lanes(G)>(bn, lane, on_leaf,
                                                    [](float3, float3) { return true; })
                     : -1;
    warp_min_lex<G>(best, best_id);
    LocalStack<kStack> st;
    int sp = 0;
    bool active = node >= 0;
    for (int iter = 0; __any_sync(0xffffffffu, active); ++iter) {
        if (active) {
            if (iter >= max_iter) {
                tv.overflow = true;
                active = false;
            } else {
                ++tv.nodes;
                float3 llo, lhi, rlo, rhi;
                int lref, rref;
                load_bnode(bn, node, llo, lhi, rlo, rhi, lref, rref);
                const float dl = dist2_box(p, llo, lhi);
                const float dr = dist2_box(p, rlo, rhi);
                bool okl = dl <= best;
                bool okr = dr <= best;
                const bool lfirst = dl <= dr;
                if (lfirst) {
                    if (okl && lref < 0) { on_leaf(~lref); okl = false; }
                    if (okr && rref < 0 && dr <= best) on_leaf(~rref);
                    if (rref < 0) okr = false;
                } else {
                    if (okr && rref < 0) { on_leaf(~rref); okr = false; }
                    if (okl && lref < 0 && dl <= best) on_leaf(~lref);
                    if (lref < 0) okl = false;
                }
                if (okl && okr) {
                    if (sp >= kStack) {
                        tv.overflow = true;
                        active = false;
                    } else {
                        st.put(sp++, lfirst ? rref : lref, lfirst ? dr : dl);
                        node = lfirst ? lref : rref;
                    }
                } else if (okl) {
                    node = lref;
                } else if (okr) {
                    node = rref;
                } else {
                    node = -1;
                    while (sp > 0) {
                        --sp;
                        int pn;
                        float pk;
                        st.get(sp, pn, pk);
                        if (pk <= best) {
                            node = pn;
                            break;
                        }
                    }
                    if (node < 0) active = false;
                }
            }
        }
        warp_min_lex<G>(best, best_id);
    }
    return best_id != 0x7fffffff ? make_uint2(__float_as_uint(best), static_cast<unsigned>(best_id))
                                 : make_uint2(0u, 0xffffffffu);
}

// kNN, split: the k best candidates form ONE warp-wide sorted table, entry j held by lane j
// (k <= 32), so every lane prunes with the exact k-th distance of everything found so far.
// After each traversal step the lanes' new leaf candidates (up to two per lane) are inserted
// one at a time: a ballot gives the insertion rank, a shuffle shifts the tail down.
struct WarpTable {
    float d;   // this lane's entry
    int id;
    float kd;  // entry k-1, broadcast
    int kid;
    __device__ __forceinline__ void init() {
        d = kInf;
        id = 0x7fffffff;
        kd = kInf;
        kid = 0x7fffffff;
    }
    __device__ __forceinline__ bool admits(float bound) const {
        return kid == 0x7fffffff || bound <= kd;
    }
    // whole warp; x is the same on every lane of a group, `lane` the lane in the group; a group
    // with doit false keeps its table (every lane still takes part in the exchanges)
    template <int G = 32>
    __device__ __forceinline__ void insert(float xd, int xid, int k, int lane, bool doit = true) {
        if constexpr (G < 32) {
            const bool want = doit && closer(xd, xid, kd, kid);
            const unsigned before = group_bits<G>(
                __ballot_sync(0xffffffffu, lane < k && closer(d, id, xd, xid)));
            const int pos = __popc(before);
            const float pd = __shfl_up_sync(0xffffffffu, d, 1, G);
            const int pid = __shfl_up_sync(0xffffffffu, id, 1, G);
            if (want && lane < k) {
                if (lane == pos) {
                    d = xd;
                    id = xid;
                } else if (lane > pos) {
                    d = pd;
                    id = pid;
                }
            }
            kd = __shfl_sync(0xffffffffu, d, k - 1, G);
            kid = __shfl_sync(0xffffffffu, id, k - 1, G);
            return;
        }
        if (!closer(xd, xid, kd, kid)) return;
        const unsigned before = __ballot_sync(0xffffffffu, lane < k && closer(d, id, xd, xid));
        const int pos = __popc(before);
        const float pd = __shfl_up_sync(0xffffffffu, d, 1);
        const int pid = __shfl_up_sync(0xffffffffu, id, 1);
        if (lane < k) {
            if (lane == pos) {
                d = xd;
                id = xid;
            } else if (lane > pos) {
                d = pd;
                id = pid;
            }
        }
        kd = __shfl_sync(0xffffffffu, d, k - 1);
        kid = __shfl_sync(0xffffffffu, id, k - 1);
    }
};

// the warp's (group's) table holds the query's k best on return (entry j in lane j; k <= G)
template <class Ops, int G = 32>
__device__ __forceinline__ void knn_split_one(const BNode* __restrict__ bn,
                                              const float4* __restrict__ leaves, float3 p, int k,
                                              int lane, int max_iter, Trav& tv, WarpTable& tab,
                                              bool valid = true) {
    tab.init();
    tab.init();
    // up to two pending leaf candidates per lane, inserted by the whole warp
    float cd[2];
    int cid[2];
    bool has[2] = {false, false};
    auto leaf = [&](int slot, int c) {
        ++tv.leaves;
        cd[c] = Ops::dist2(p, leaves, slot, cid[c]);
        has[c] = true;
    };
    auto flush = [&]() {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if constexpr (G < 32) {
                // each group inserts its own candidates, lowest lane first; the rounds run
                // until no group of the warp has one left
                unsigned m = group_bits<G>(__ballot_sync(0xffffffffu, has[c]));
                while (__any_sync(0xffffffffu, m != 0u)) {
                    const bool doit = m != 0u;
                    const int src = doit ? __ffs(m) - 1 : 0;
                    const float xd = __shfl_sync(0xffffffffu, cd[c], src, G);
                    const int xid = __shfl_sync(0xffffffffu, cid[c], src, G);
                    tab.insert<G>(xd, xid, k, lane, doit);
                    if (doit) m &= m - 1;
                }
            } else {
                unsigned m = __ballot_sync(0xffffffffu, has[c]);
                while (m) {
                    const int src = __ffs(m) - 1;
                    const float xd = __shfl_sync(0xffffffffu, cd[c], src);
                    const int xid = __shfl_sync(0xffffffffu, cid[c], src);
                    tab.insert(xd, xid, k, lane);
                    m &= m - 1;
                }
            }
            has[c] = false;
        }
    };
    int node = valid ? split_descend<log2_lanes(G)>(bn, lane, [&](int slot) { leaf(slot, 0); },
                                                    [](float3, float3) { return true; })
                     : -1;
    flush();
    LocalStack<kStack> st;
    int sp = 0;
    bool active = node >= 0;
    for (int iter = 0; __any_sync(0xffffffffu, active); ++iter) {
        if (active) {
            if (iter >= max_iter) {
                tv.overflow = true;
                active = false;
            } else {
                ++tv.nodes;
                float3 llo, lhi, rlo, rhi;
                int lref, rref;
                load_bnode(bn, node, llo, lhi, rlo, rhi, lref, rref);
                const float dl = dist2_box(p, llo, lhi);
                const float dr = dist2_box(p, rlo, rhi);
                const bool lfirst = dl <= dr;
                bool okl = tab.admits(dl);
                bool okr = tab.admits(dr);
                if (okl && lref < 0) { leaf(~lref, 0); okl = false; }
                if (okr && rref < 0) { leaf(~rref, 1); okr = false; }
                if (okl && okr) {
                    if (sp >= kStack) {
                        tv.overflow = true;
                        active = false;
                    } else {
                        st.put(sp++, lfirst ? rref : lref, lfirst ? dr : dl);
                        node = lfirst ? lref : rref;
                    }
                } else if (okl) {
                    node = lref;
                } else if (okr) {
                    node = rref;
                } else {
                    node = -1;
                    while (sp > 0) {
                        --sp;
                        int pn;
                        float pk;
                        st.get(sp, pn, pk);
                        if (tab.admits(pk)) {
                            node = pn;
                            break;
                        }
                    }
                    if (node < 0) active = false;
                }
            }
        }
        flush();
    }
}

__device__ __forceinline__ uint2 warp_table_entry(const WarpTable& tab) {
    return tab.id != 0x7fffffff ? make_uint2(__float_as_uint(tab.d), static_cast<unsigned>(tab.id))
                                : make_uint2(0u, 0xffffffffu);
}

// radius, split: returns this lane's count; the fill pass writes the lane's keys from
// `write` on, never past `end` (the query's offset plus the counts of the lower lanes)
template <class Ops, bool kFill, int G = 32>
__device__ __forceinline__ int radius_split_one(const BNode* __restrict__ bn,
                                                const float4* __restrict__ leaves, float3 p,
                                                float r2, int lane, int write, int end,
                                                unsigned long long* __restrict__ keys,
                                                int max_iter, Trav& tv, bool valid = true) {
    int found = 0;
    auto keep = [&](float3 lo, float3 hi) { return dist2_box(p, lo, hi) <= r2; };
    auto on_leaf = [&](int slot) {
        ++tv.leaves;
        int id;
        const float d2 = Ops::dist2(p, leaves, slot, id);
        if (d2 <= r2) {
            if (kFill && write < end) keys[write++] = radius_key(d2, id);
            ++found;
        }
    };
    int node = valid ? split_descend<log2_lanes(G)>(bn, lane, on_leaf, keep) : -1;
    LocalStack<kStack> st;
    int sp = 0;
    for (int iter = 0; node >= 0; ++iter) {
        if (iter >= max_iter) {
            tv.overflow = true;
            break;
        }
        ++tv.nodes;
        float3 llo, lhi, rlo, rhi;
        int lref, rref;
        load_bnode(bn, node, llo, lhi, rlo, rhi, lref, rref);
        bool okl = keep(llo, lhi);
        bool okr = keep(rlo, rhi);
        if (okl && lref < 0) {
            on_leaf(~lref);
            okl = false;
        }
        if (okr && rref < 0) {
            on_leaf(~rref);
            okr = false;
        }
        if (okl && okr) {
            if (sp >= kStack) {
                tv.overflow = true;
                break;
            }
            st.put_node(sp++, rref);
            node = lref;
        } else if (okl) {
            node = lref;
        } else if (okr) {
            node = rref;
        } else {
            node = sp > 0 ? st.get_node(--sp) : -1;
        }
    }
    return found;
}

// exclusive prefix over the lanes of `v` (of the group of G lanes; `lane` the lane in it)
template <int G = 32>
__device__ __forceinline__ int warp_exclusive(int v, int lane) {
    int incl = v;
#pragma unroll
    for (int o = 1; o < G; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o, G);
        if (lane >= o) incl += u;
    }
    return incl - v;
}

// sum of `v` over the group of G lanes (every lane gets it)
template <int G>
__device__ __forceinline__ int group_sum(int v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace qk
