// qk_build.cuh -- device code shared by the single-tree builder (qk_build.cu) and the
// batched builder (qk_batch.cu): Morton quantisation, the Karras emit of one slot, the
// bottom-up climb of one leaf and the 4-wide node of one even-depth internal node.
#pragma once

#include "qk_internal.cuh"

namespace qk {

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// quantize (lbvh.cu:285-290): (v - lo) / extent * 1023 + 0.5, clamped, truncated
__device__ __forceinline__ uint32_t quant(float v, float lo, float extent) {
    if (extent <= 0.0f) return 0;
    const float q = (v - lo) / extent * 1023.0f + 0.5f;
    return static_cast<uint32_t>(static_cast<int>(fminf(1023.0f, fmaxf(0.0f, q))));
}

// 64-bit key of slot j: (code << 32) | scene index
__device__ __forceinline__ uint64_t key64(const uint32_t* codes, const uint32_t* ids, int j) {
    return (static_cast<uint64_t>(codes[j]) << 32) | ids[j];
}

// common-prefix length of keys a and b; -1 outside [0, n)
__device__ __forceinline__ int cpl(const uint32_t* codes, const uint32_t* ids, int n, uint64_t ka,
                                   int b) {
    if (b < 0 || b >= n) return -1;
    const uint64_t x = ka ^ key64(codes, ids, b);
    return x == 0 ? 64 : __clzll(x);
}

__device__ __forceinline__ void write_box(Node* nd, Box b) {
    float4* p = reinterpret_cast<float4*>(nd);
    const float4 a = p[1];
    p[0] = make_float4(b.lo.x, b.lo.y, b.lo.z, b.hi.x);
    p[1] = make_float4(b.hi.y, b.hi.z, a.z, a.w);
}

// Floats of shared staging per warp for emit_leaves_warp: 32 slots of the largest of the
// sorted item, the leaf node (8 floats) and the leaf payload.
template <class Ops>
constexpr int emit_stage_floats() {
    return 32 * (Ops::kFloats > 8 ? (Ops::kFloats > 4 * Ops::kVec4 ? Ops::kFloats : 4 * Ops::kVec4)
                                  : (8 > 4 * Ops::kVec4 ? 8 : 4 * Ops::kVec4));
}

// Leaves k0 .. k0 + m - 1 (m <= 32) of a tree of n leaves, by the whole warp: lane i < m holds
// the item (it) and scene index (src) of slot k0 + i.  For triangles and Gaussians (36- and
// 40-byte items, 48-byte payloads) the sorted items, leaf nodes and leaf payloads go out
// through the warp's shared staging (16-byte aligned, emit_stage_floats<Ops>() floats) so that
// each store instruction covers consecutive whole lines instead of one strided piece per lane
// (city LBVH build 0.587 -> 0.572 ms); points store per lane.
template <class Ops>
__device__ __forceinline__ void store_leaves_warp(const float (&it)[Ops::kFloats], int src, int n,
                                                  Node* __restrict__ nodes,
                                                  float* __restrict__ sorted,
                                                  int* __restrict__ prim_ids,
                                                  int* __restrict__ slot_of,
                                                  float4* __restrict__ leaves, int k0, int m,
                                                  float* stage) {
    const int lane = threadIdx.x & 31;
    const int k = k0 + lane;
    const bool ok = lane < m;
    if (ok) {
        prim_ids[k] = src;
        slot_of[src] = k;
    }
    if constexpr (Ops::kFloats <= 4) {
        // a point's 12 bytes: per-lane stores cost no more than the staging (measured)
        if (!ok) return;
#pragma unroll
        for (int j = 0; j < Ops::kFloats; ++j) sorted[static_cast<size_t>(k) * Ops::kFloats + j] = it[j];
        const Box b = Ops::bounds(it);
        float4* leafnode = reinterpret_cast<float4*>(nodes + (n - 1 + k));
        leafnode[0] = make_float4(b.lo.x, b.lo.y, b.lo.z, b.hi.x);
        leafnode[1] = make_float4(b.hi.y, b.hi.z, __int_as_float(-(k + 1)), __int_as_float(1));
        float4 pay[Ops::kVec4];
        Ops::pack(it, src, pay);
#pragma unroll
        for (int j = 0; j < Ops::kVec4; ++j) leaves[static_cast<size_t>(k) * Ops::kVec4 + j] = pay[j];
        return;
    }
    // sorted items
#pragma unroll
    for (int j = 0; j < Ops::kFloats; ++j) stage[lane * Ops::kFloats + j] = it[j];
    __syncwarp();
    float* sdst = sorted + static_cast<size_t>(k0) * Ops::kFloats;
    for (int t = lane; t < m * Ops::kFloats; t += 32) sdst[t] = stage[t];
    __syncwarp();
    // leaf nodes n - 1 + k: the box, -(slot + 1) and 1
    float4* st4 = reinterpret_cast<float4*>(stage);
    const Box b = Ops::bounds(it);
    st4[2 * lane] = make_float4(b.lo.x, b.lo.y, b.lo.z, b.hi.x);
    st4[2 * lane + 1] = make_float4(b.hi.y, b.hi.z, __int_as_float(-(k + 1)), __int_as_float(1));
    __syncwarp();
    float4* ndst = reinterpret_cast<float4*>(nodes + (n - 1 + k0));
    for (int t = lane; t < 2 * m; t += 32) ndst[t] = st4[t];
    __syncwarp();
    // leaf payloads
    float4 pay[Ops::kVec4];
    Ops::pack(it, src, pay);
#pragma unroll
    for (int j = 0; j < Ops::kVec4; ++j) st4[lane * Ops::kVec4 + j] = pay[j];
    __syncwarp();
    float4* ldst = leaves + static_cast<size_t>(k0) * Ops::kVec4;
    for (int t = lane; t < m * Ops::kVec4; t += 32) ldst[t] = st4[t];
    __syncwarp();
}

// Leaves k0 .. k0 + m - 1 (m <= 32) of the LBVH over sorted (code, id) pairs, by the whole
// warp: each lane gathers one primitive, then store_leaves_warp writes them.
template <class Ops>
__device__ __forceinline__ void emit_leaves_warp(
    const float* __restrict__ items, int n, const uint32_t* __restrict__ ids,
    Node* __restrict__ nodes, float* __restrict__ sorted, int* __restrict__ prim_ids,
    int* __restrict__ slot_of, float4* __restrict__ leaves, int k0, int m, float* stage) {
    const int lane = threadIdx.x & 31;
    const bool ok = lane < m;
    const int src = ok ? static_cast<int>(ids[k0 + lane]) : 0;
    float it[Ops::kFloats];
#pragma unroll
    for (int j = 0; j < Ops::kFloats; ++j)
        it[j] = ok ? items[static_cast<size_t>(src) * Ops::kFloats + j] : 0.0f;
    store_leaves_warp<Ops>(it, src, n, nodes, sorted, prim_ids, slot_of, leaves, k0, m, stage);
}

// Internal node k (k < n - 1) of the LBVH over sorted (code, id) pairs, its children's parent
// links, its slot range (with `ranges`) and its arrival counter; parent[0] = -1 for k = 0.
__device__ __forceinline__ void emit_internal(int n, const uint32_t* __restrict__ codes,
                                              const uint32_t* __restrict__ ids,
                                              Node* __restrict__ nodes, int* __restrict__ parent,
                                              BNode* __restrict__ bnodes, int* __restrict__ flags,
                                              int k, int2* __restrict__ ranges = nullptr) {
    if (k == 0) parent[0] = -1;
    if (k >= n - 1) return;

    // internal node k (Karras 2012): direction, range end by exponential + binary search,
    // then the split as the last index whose prefix with the first exceeds the node's
    const uint64_t kk = key64(codes, ids, k);
    const int dir = cpl(codes, ids, n, kk, k + 1) > cpl(codes, ids, n, kk, k - 1) ? 1 : -1;
    const int dmin = cpl(codes, ids, n, kk, k - dir);
    int lmax = 2;
    while (cpl(codes, ids, n, kk, k + lmax * dir) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t > 0; t /= 2) {
        if (cpl(codes, ids, n, kk, k + (l + t) * dir) > dmin) l += t;
    }
    const int j = k + l * dir;
    const int first = min(k, j), last = max(k, j);
    if (ranges) ranges[k] = make_int2(first, last - first + 1);
    const int dnode = cpl(codes, ids, n, kk, j);
    const uint64_t kf = key64(codes, ids, first);
    int split = first;
    int step = last - first;
    do {
        step = (step + 1) >> 1;
        const int cand = split + step;
        if (cand < last && cpl(codes, ids, n, kf, cand) > dnode) split = cand;
    } while (step > 1);
    const int left = split == first ? (n - 1 + split) : split;
    const int right = split + 1 == last ? (n - 1 + split + 1) : split + 1;
    *reinterpret_cast<int2*>(&nodes[k].left) = make_int2(left, right);
    parent[left] = k;
    parent[right] = k;
    const int lref = left >= n - 1 ? ~(left - (n - 1)) : left;
    const int rref = right >= n - 1 ? ~(right - (n - 1)) : right;
    bnodes[k].v3 = make_float4(__int_as_float(lref), __int_as_float(rref), 0.0f, 0.0f);
    flags[k] = 0;
}

__device__ __forceinline__ Box load_box_cg(const Node* nd) {
    const float4* p = reinterpret_cast<const float4*>(nd);
    const float4 a = __ldcg(p), b = __ldcg(p + 1);
    Box bx;
    bx.lo = f3(a.x, a.y, a.z);
    bx.hi = f3(a.w, b.x, b.y);
    return bx;
}

// Small-subtree code of a child (traversal node words v3.z / v3.w): a subtree of 2..kLeafMax
// leaves on contiguous slots is (first slot << 2) | (leaves - 1); anything else is 0.
constexpr int kLeafMax = 4;

__device__ __forceinline__ int small_code(int c, int n, int2 range) {
    return (c < n - 1 && range.y >= 2 && range.y <= kLeafMax) ? ((range.x << 2) | (range.y - 1)) : 0;
}

__device__ __forceinline__ Box load_box_ca(const Node* nd) {
    const float4* p = reinterpret_cast<const float4*>(nd);
    const float4 a = __ldca(p), b = __ldca(p + 1);
    Box bx;
    bx.lo = f3(a.x, a.y, a.z);
    bx.hi = f3(a.w, b.x, b.y);
    return bx;
}

// Complete internal node p from its final children given its links lr = (left, right) and the
// children's slot ranges (all static during the pass): box and traversal node, with the
// children's small-subtree codes.  kLocal: both children were finished by threads of this
// block, whose writes a plain load sees after the block fence; otherwise they are read from L2.
// kCodes false (refits): the small-subtree codes, which depend on the topology only, are kept.
template <bool kLocal, bool kCodes = true>
__device__ __forceinline__ void finish_node_links(Node* __restrict__ nodes,
                                                  BNode* __restrict__ bnodes, int p, int n,
                                                  int2 lr, int2 rl, int2 rr) {
    const int l = lr.x, r = lr.y;
    if (kCodes)
        *reinterpret_cast<float2*>(&bnodes[p].v3.z) = make_float2(
            __int_as_float(small_code(l, n, rl)), __int_as_float(small_code(r, n, rr)));
    const Box a = kLocal ? load_box_ca(nodes + l) : load_box_cg(nodes + l);
    const Box b = kLocal ? load_box_ca(nodes + r) : load_box_cg(nodes + r);
    Box u;
    u.lo = f3(fmin_t(a.lo.x, b.lo.x), fmin_t(a.lo.y, b.lo.y), fmin_t(a.lo.z, b.lo.z));
    u.hi = f3(fmax_t(a.hi.x, b.hi.x), fmax_t(a.hi.y, b.hi.y), fmax_t(a.hi.z, b.hi.z));
    float4* np = reinterpret_cast<float4*>(nodes + p);
    np[0] = make_float4(u.lo.x, u.lo.y, u.lo.z, u.hi.x);
    np[1] = make_float4(u.hi.y, u.hi.z, __int_as_float(l), __int_as_float(r));
    BNode& bn = bnodes[p];
    bn.v0 = make_float4(a.lo.x, a.lo.y, a.lo.z, a.hi.x);
    bn.v1 = make_float4(a.hi.y, a.hi.z, b.lo.x, b.lo.y);
    bn.v2 = make_float4(b.lo.z, b.hi.x, b.hi.y, b.hi.z);
}

// Refit: one leaf's climb toward the root of a tree whose topology is unchanged; flags[p]
// counts arrivals at internal node p, the second arrival finishes p's box and traversal node
// (its small-subtree codes kept), resets the counter and continues.  The next level's parent
// and links (static) are loaded while this level's arrival and boxes wait.
__device__ __forceinline__ void climb_refit(Node* __restrict__ nodes, BNode* __restrict__ bnodes,
                                            const int* __restrict__ parent,
                                            int* __restrict__ flags, int n, int k) {
    auto links = [&](int v) { return *reinterpret_cast<const int2*>(&nodes[v].left); };
    int p = parent[n - 1 + k];
    if (p < 0) return;
    int2 lr = links(p);
    int pn = parent[p];
    const int2 none = make_int2(0, 0);
    for (int guard = 0; guard < 4096; ++guard) {
        int2 lrn = none;
        int pnn = -1;
        if (pn >= 0) {
            lrn = links(pn);
            pnn = parent[pn];
        }
        if (arrive_add(&flags[p], 1) == 0) return;
        finish_node_links<false, false>(nodes, bnodes, p, n, lr, none, none);
        flags[p] = 0;
        if (pn < 0) return;
        p = pn;
        lr = lrn;
        pn = pnn;
    }
}

// One leaf's climb when every internal node's slot range is known (`ranges`).  The calling
// block starts climbs at the leaves of slots [base, base + kSpan).  A node whose whole range
// lies in those slots has both children finished by this block, so its two arrivals meet in
// the shared counter arrivals[gap - base] (gap: the last slot of its left child, unique per
// internal node) behind block fences; only nodes spanning blocks take the device-scope
// counter in flags[], which the finishing arrival resets.  Links, parents and ranges do not
// change during the pass, so the next level's are loaded while this level's arrival and box
// wait: after an arrival only the children's boxes remain on the chain of dependent loads.
template <int kSpan>
__device__ __forceinline__ void climb_ranged(Node* __restrict__ nodes, BNode* __restrict__ bnodes,
                                             const int* __restrict__ parent,
                                             int* __restrict__ flags, int n, int k, int base,
                                             int* arrivals, const int2* __restrict__ ranges) {
    // plain loads: the pass rewrites the links' 16-byte word (with the same values)
    auto links = [&](int v) { return *reinterpret_cast<const int2*>(&nodes[v].left); };
    auto crange = [&](int v) { return v >= n - 1 ? make_int2(v - (n - 1), 1) : __ldg(ranges + v); };
    int c = n - 1 + k;
    int2 rc = make_int2(k, 1);
    int p = parent[c];
    if (p < 0) return;
    int2 rp = __ldg(ranges + p), lr = links(p);
    int pn = parent[p];
    for (int guard = 0; guard < 4096; ++guard) {
        int2 rpn = make_int2(0, 0), lrn = make_int2(0, 0);
        int pnn = -1;
        if (pn >= 0) {
            rpn = __ldg(ranges + pn);
            lrn = links(pn);
            pnn = parent[pn];
        }
        const int2 rl = crange(lr.x), rr = crange(lr.y);
        const bool local = rp.x >= base && rp.x + rp.y <= base + kSpan;
        int old;
        if (local) {
            const int gap = lr.x == c ? rc.x + rc.y - 1 : rc.x - 1;
            __threadfence_block();
            old = atomicAdd(&arrivals[gap - base], 1);
            __threadfence_block();
        } else {
            old = arrive_add(&flags[p], 1);
        }
        if (old == 0) return;
        if (local) {
            finish_node_links<true>(nodes, bnodes, p, n, lr, rl, rr);
        } else {
            finish_node_links<false>(nodes, bnodes, p, n, lr, rl, rr);
            flags[p] = 0;
        }
        if (pn < 0) return;
        c = p;
        rc = rp;
        p = pn;
        rp = rpn;
        lr = lrn;
        pn = pnn;
    }
}

// depth of node i = length of its parent chain (lbvh.cu:419-431), bounded by `limit`
__device__ __forceinline__ int chain_depth(const int* __restrict__ parent, int i, int limit) {
    int d = 0;
    int p = i;
    while (p > 0 && d < limit) {
        p = parent[p];
        ++d;
    }
    return d;
}

// Depths in two passes.  Anchors, the internal nodes of at least kDepthAnchor leaves (a few
// per kDepthAnchor leaves, all near the root), walk their whole parent chain; every other node
// walks only up to its nearest anchor ancestor (a few steps: leaf counts grow toward the root)
// and adds that anchor's depth.  `ranges` holds each internal node's (first slot, leaves).
constexpr int kDepthAnchor = 64;

__device__ __forceinline__ bool depth_anchor(const int2* __restrict__ ranges, int i, int n) {
    return i < n - 1 && ranges[i].y >= kDepthAnchor;
}

// atomicMax of the block's largest v into *dst, one atomic per block (one per warp on a single
// address serialises in its L2 slice)
__device__ __forceinline__ void block_max_to(int v, int* dst) {
    __shared__ int wmax[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int m = wmax[0];
#pragma unroll
        for (int w = 1; w < kBlock / 32; ++w) m = max(m, wmax[w]);
        if (m > 0) atomicMax(dst, m);
    }
}

// depth of a node that is not an anchor (anchors' depths already in `depth`)
__device__ __forceinline__ int anchored_depth(const int* __restrict__ parent,
                                              const int2* __restrict__ ranges,
                                              const int* __restrict__ depth, int n, int i,
                                              int limit) {
    int d = 0;
    int p = i;
    while (p > 0 && d < limit) {
        p = parent[p];
        ++d;
        if (depth_anchor(ranges, p, n)) return d + depth[p];
    }
    return d;
}

__device__ __forceinline__ void wide_fill(WideEntry& e, const Node& src, int child) {
    e.mn[0] = src.mn[0];
    e.mn[1] = src.mn[1];
    e.mn[2] = src.mn[2];
    e.mx[0] = src.mx[0];
    e.mx[1] = src.mx[1];
    e.mx[2] = src.mx[2];
    e.child = child;
    e.pad = 0;
}

__device__ __forceinline__ void wide_node_of(const Node* __restrict__ nodes, int n, const int* __restrict__ wide_id,
                             int i, WideNode& out) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        out.c[s].mn[0] = out.c[s].mn[1] = out.c[s].mn[2] = kInf;
        out.c[s].mx[0] = out.c[s].mx[1] = out.c[s].mx[2] = -kInf;
        out.c[s].child = kEmptySlot;
        out.c[s].pad = 0;
    }
    const int kids[2] = {nodes[i].left, nodes[i].right};
    int slot = 0;
    for (int k = 0; k < 2; ++k) {
        const int c = kids[k];
        if (c >= n - 1) {
            wide_fill(out.c[slot++], nodes[c], nodes[c].left);
            continue;
        }
        const int g[2] = {nodes[c].left, nodes[c].right};
        for (int j = 0; j < 2; ++j) {
            const int gc = g[j];
            wide_fill(out.c[slot++], nodes[gc], gc >= n - 1 ? nodes[gc].left : wide_id[gc]);
        }
    }
}

// Small-subtree code of internal node g as its parent's traversal node keeps it (0 for the
// root, whose subtree is never one leaf slot).
__device__ __forceinline__ int own_small_code(const Node* __restrict__ nodes,
                                              const BNode* __restrict__ bn,
                                              const int* __restrict__ parent, int g) {
    const int p = parent[g];
    if (p < 0) return 0;
    const float4 v3 = bn[p].v3;
    return __float_as_int(nodes[p].left == g ? v3.z : v3.w);
}

// 4-wide node of binary node i in the leaf-size-4 form (no quarry counterpart; quarry keeps
// `pad` zero): as wide_node_of, except that a child or grandchild whose subtree holds 2..4
// leaves on contiguous slots takes ONE slot as a leaf range -- child = ~first slot (the leaf
// code of its first slot), pad = its primitive count -- and a single leaf slot has pad = 1.
// Internal slots keep pad = 0, so a traversal reads max(pad, 1) primitives at every leaf slot
// of either form.  The wide nodes are the even-depth internal nodes that are not inside such a
// range (the root always).
__device__ __forceinline__ void wide4_slot(WideEntry& e, const Node* __restrict__ nodes, int n,
                                           const int* __restrict__ wide_id, int c, int code) {
    if (c >= n - 1) {
        wide_fill(e, nodes[c], nodes[c].left);
        e.pad = 1;
    } else if (code != 0) {
        wide_fill(e, nodes[c], ~(code >> 2));
        e.pad = (code & 3) + 1;
    } else {
        wide_fill(e, nodes[c], wide_id[c]);
    }
}

__device__ __forceinline__ void wide4_node_of(const Node* __restrict__ nodes,
                                              const BNode* __restrict__ bn, int n,
                                              const int* __restrict__ wide_id, int i,
                                              WideNode& out) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        out.c[s].mn[0] = out.c[s].mn[1] = out.c[s].mn[2] = kInf;
        out.c[s].mx[0] = out.c[s].mx[1] = out.c[s].mx[2] = -kInf;
        out.c[s].child = kEmptySlot;
        out.c[s].pad = 0;
    }
    const int kids[2] = {nodes[i].left, nodes[i].right};
    const float4 v3 = bn[i].v3;
    const int codes[2] = {__float_as_int(v3.z), __float_as_int(v3.w)};
    int slot = 0;
    for (int k = 0; k < 2; ++k) {
        const int c = kids[k];
        if (c >= n - 1 || codes[k] != 0) {
            wide4_slot(out.c[slot++], nodes, n, wide_id, c, codes[k]);
            continue;
        }
        const float4 w3 = bn[c].v3;
        const int g[2] = {nodes[c].left, nodes[c].right};
        const int gcodes[2] = {__float_as_int(w3.z), __float_as_int(w3.w)};
        for (int j = 0; j < 2; ++j) wide4_slot(out.c[slot++], nodes, n, wide_id, g[j], gcodes[j]);
    }
}

}  // namespace qk
