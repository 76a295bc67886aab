// qk_build.cu -- LBVH build, topology-frozen refit, 4-wide collapse and structural checks.
//
// LBVH (Karras 2012, as quarry's src/gpu/lbvh.cu:213-514 and 1954-2041 define it):
//   1. centroid bounds: grid-stride min/max, warp shuffles, one ordered-uint atomic per block
//   2. 30-bit Morton code of the quantized centroid, value = scene index
//   3. stable radix sort on the code (equal codes keep index order = the reference's
//      64-bit (code << 32 | index) key order)
//   4. emit: one thread per slot writes the leaf (payload, canonical leaf node, prim id,
//      inverse map) and, for slot < n-1, the internal node found by the Karras split
//      search over the 64-bit keys
//   5. bottom-up boxes in ONE launch: each leaf thread climbs its parent chain; an atomic
//      visit counter per internal node lets the second arriving child compute the union
//      (both children final) and carry on, the first one stops.  min/max is exact, so the
//      boxes equal the reference's level-by-level refit bit for bit.  The same pass writes
//      the 64-byte traversal node (both child boxes inline).
//   6. depth of every node by walking its parent chain; the maximum is read back once.
#include <algorithm>
#include <cstdio>

#include "qk_internal.cuh"
#include "qk_build.cuh"

namespace qk {

namespace {

__global__ void k_header_init(Header* h) {
    if (threadIdx.x < 3) {
        h->lo[threadIdx.x] = ord_f(kInf);
        h->hi[threadIdx.x] = ord_f(-kInf);
    }
    if (threadIdx.x == 0) {
        h->max_depth = 0;
        h->counter = 0;
        h->overflow = 0;
        h->error = 0;
        h->list_count[0] = 0;
        h->list_count[1] = 0;
    }
}

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <class Ops>
__global__ __launch_bounds__(kBlock) void k_centroid_bounds(const float* __restrict__ items,
                                                            int n, Header* __restrict__ h) {
    float lo0 = kInf, lo1 = kInf, lo2 = kInf, hi0 = -kInf, hi1 = -kInf, hi2 = -kInf;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += kBlock * gridDim.x) {
        const float3 c = Ops::centroid(items + static_cast<size_t>(i) * Ops::kFloats);
        lo0 = fminf(lo0, c.x);
        lo1 = fminf(lo1, c.y);
        lo2 = fminf(lo2, c.z);
        hi0 = fmaxf(hi0, c.x);
        hi1 = fmaxf(hi1, c.y);
        hi2 = fmaxf(hi2, c.z);
    }
    __shared__ float s[6][kBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    lo0 = warp_min(lo0);
    lo1 = warp_min(lo1);
    lo2 = warp_min(lo2);
    hi0 = warp_max(hi0);
    hi1 = warp_max(hi1);
    hi2 = warp_max(hi2);
    if (lane == 0) {
        s[0][warp] = lo0;
        s[1][warp] = lo1;
        s[2][warp] = lo2;
        s[3][warp] = hi0;
        s[4][warp] = hi1;
        s[5][warp] = hi2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        float v = kInf;
        for (int w = 0; w < kBlock / 32; ++w) v = fminf(v, s[threadIdx.x][w]);
        atomicMin(&h->lo[threadIdx.x], ord_f(v));
    } else if (threadIdx.x < 6) {
        float v = -kInf;
        for (int w = 0; w < kBlock / 32; ++w) v = fmaxf(v, s[threadIdx.x][w]);
        atomicMax(&h->hi[threadIdx.x - 3], ord_f(v));
    }
}

template <class Ops>
__global__ __launch_bounds__(kBlock) void k_morton(const float* __restrict__ items, int n,
                                                   const Header* __restrict__ h,
                                                   uint32_t* __restrict__ codes,
                                                   uint32_t* __restrict__ idx) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= n) return;
    const float lx = unord_f(h->lo[0]), ly = unord_f(h->lo[1]), lz = unord_f(h->lo[2]);
    const float hx = unord_f(h->hi[0]), hy = unord_f(h->hi[1]), hz = unord_f(h->hi[2]);
    const float3 c = Ops::centroid(items + static_cast<size_t>(i) * Ops::kFloats);
    codes[i] = spread10(quant(c.x, lx, hx - lx)) | (spread10(quant(c.y, ly, hy - ly)) << 1) |
               (spread10(quant(c.z, lz, hz - lz)) << 2);
    idx[i] = static_cast<uint32_t>(i);
}

template <class Ops>
__global__ __launch_bounds__(kBlock) void k_emit(
    const float* __restrict__ items, int n, const uint32_t* __restrict__ codes,
    const uint32_t* __restrict__ ids, Node* __restrict__ nodes, float* __restrict__ sorted,
    int* __restrict__ prim_ids, int* __restrict__ slot_of, int* __restrict__ parent,
    BNode* __restrict__ bnodes, float4* __restrict__ leaves, int* __restrict__ flags,
    int2* __restrict__ ranges) {
    __shared__ __align__(16) float stage[kBlock / 32][emit_stage_floats<Ops>()];
    const int k0 = blockIdx.x * kBlock + (threadIdx.x & ~31);
    if (k0 >= n) return;  // whole warps
    emit_leaves_warp<Ops>(items, n, ids, nodes, sorted, prim_ids, slot_of, leaves, k0,
                          min(32, n - k0), stage[threadIdx.x >> 5]);
    const int k = k0 + (threadIdx.x & 31);
    if (k < n) emit_internal(n, codes, ids, nodes, parent, bnodes, flags, k, ranges);
}

// (first slot, leaves) of every internal node of a tree whose subtrees cover ordered
// contiguous slot runs (every builder here emits them so): leftmost and rightmost leaf.
__global__ __launch_bounds__(kBlock) void k_ranges_descent(const Node* __restrict__ nodes, int n,
                                                          int2* __restrict__ ranges) {
    const int v = blockIdx.x * kBlock + threadIdx.x;
    if (v >= n - 1) return;
    int a = v, b = v;
    for (int guard = 0; a < n - 1 && guard < 4096; ++guard) a = nodes[a].left;
    for (int guard = 0; b < n - 1 && guard < 4096; ++guard) b = nodes[b].right;
    const int first = a - (n - 1), last = b - (n - 1);
    ranges[v] = make_int2(first, last >= first ? last - first + 1 : 0);
}

// Bottom-up boxes with known slot ranges: block b's threads start at the leaves of slots
// [kUpSpan b, kUpSpan b + kUpSpan) (climb_ranged in qk_build.cuh).  Blocks of 512 and 1,024
// leaves keep more of each climb in shared memory but built no faster (city LBVH 0.567 and
// 0.585-0.595 ms against 0.561-0.564 ms).
constexpr int kUpSpan = 256;  // leaves (and threads) per block of the ranged bottom-up
template <int kSpan>
__global__ __launch_bounds__(kSpan) void k_bottom_up_ranged(Node* __restrict__ nodes,
                                                           BNode* __restrict__ bnodes,
                                                           const int* __restrict__ parent,
                                                           int* __restrict__ flags, int n,
                                                           const int2* __restrict__ ranges) {
    __shared__ int arrivals[kSpan];
    const int base = blockIdx.x * kSpan;
    arrivals[threadIdx.x] = 0;
    __syncthreads();
    const int k = base + threadIdx.x;
    if (k >= n) return;
    climb_ranged<kSpan>(nodes, bnodes, parent, flags, n, k, base, arrivals, ranges);
}

// Refit: one thread per leaf climbs toward the root (climb_refit in qk_build.cuh).
__global__ __launch_bounds__(kBlock) void k_bottom_up(Node* __restrict__ nodes,
                                                     BNode* __restrict__ bnodes,
                                                     const int* __restrict__ parent,
                                                     int* __restrict__ flags, int n) {
    const int k = blockIdx.x * kBlock + threadIdx.x;
    if (k >= n) return;
    climb_refit(nodes, bnodes, parent, flags, n, k);
}

// depth = length of the parent chain (lbvh.cu:419-431), bounded by the node count: the
// anchors' first (anchored_depth in qk_build.cuh), then every other node's and the maximum
__global__ __launch_bounds__(kBlock) void k_depth_anchors(const int* __restrict__ parent,
                                                         const int2* __restrict__ ranges, int n,
                                                         int* __restrict__ depth) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < n - 1 && depth_anchor(ranges, i, n)) depth[i] = chain_depth(parent, i, 2 * n - 1);
}

__global__ __launch_bounds__(kBlock) void k_depth(const int* __restrict__ parent,
                                                 const int2* __restrict__ ranges, int n,
                                                 int* __restrict__ depth, Header* __restrict__ h) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    const int count = 2 * n - 1;
    int d = 0;
    if (i < count) {
        if (depth_anchor(ranges, i, n)) {
            d = depth[i];
        } else {
            d = anchored_depth(parent, ranges, depth, n, i, count);
            depth[i] = d;
        }
    }
    block_max_to(d, &h->max_depth);
}

// ---- refit ----
template <class Ops>
__global__ __launch_bounds__(kBlock) void k_refit_leaves(const float* __restrict__ items, int n,
                                                         const int* __restrict__ prim_ids,
                                                         Node* __restrict__ nodes,
                                                         float* __restrict__ sorted,
                                                         float4* __restrict__ leaves) {
    const int k = blockIdx.x * kBlock + threadIdx.x;
    if (k >= n) return;
    const int src = prim_ids[k];
    float it[Ops::kFloats];
#pragma unroll
    for (int j = 0; j < Ops::kFloats; ++j) it[j] = items[static_cast<size_t>(src) * Ops::kFloats + j];
#pragma unroll
    for (int j = 0; j < Ops::kFloats; ++j) sorted[static_cast<size_t>(k) * Ops::kFloats + j] = it[j];
    write_box(nodes + (n - 1 + k), Ops::bounds(it));
    float4 pay[Ops::kVec4];
    Ops::pack(it, src, pay);
#pragma unroll
    for (int j = 0; j < Ops::kVec4; ++j) leaves[static_cast<size_t>(k) * Ops::kVec4 + j] = pay[j];
}

// Dirty refit, pass 1: write the moved leaves and mark ancestors.  flags[p] bit 0 / bit 1
// record a dirty left / right child; a thread stops climbing at the first node another
// thread already marked.  A repeated id (same leaf twice) is dropped via skip[].
template <class Ops>
__global__ __launch_bounds__(kBlock) void k_dirty_mark(
    const int* __restrict__ ids, const float* __restrict__ items, int count, int n,
    const int* __restrict__ slot_of, const int* __restrict__ parent, Node* __restrict__ nodes,
    float* __restrict__ sorted, float4* __restrict__ leaves, int* __restrict__ flags,
    int* __restrict__ skip, Header* __restrict__ h) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= count) return;
    const int id = ids[i];
    if (id < 0 || id >= n) {
        skip[i] = 1;
        atomicAdd(&h->error, 1);
        return;
    }
    const int slot = slot_of[id];
    int node = n - 1 + slot;
    int p = parent[node];
    // claim the leaf: the first thread to set the child bit of its parent owns it
    const int bit0 = nodes[p].left == node ? 1 : 2;
    const int old0 = atomicOr(&flags[p], bit0);
    if (old0 & bit0) {
        skip[i] = 1;
        return;
    }
    skip[i] = 0;
    float it[Ops::kFloats];
#pragma unroll
    for (int j = 0; j < Ops::kFloats; ++j) it[j] = items[static_cast<size_t>(i) * Ops::kFloats + j];
#pragma unroll
    for (int j = 0; j < Ops::kFloats; ++j) sorted[static_cast<size_t>(slot) * Ops::kFloats + j] = it[j];
    write_box(nodes + node, Ops::bounds(it));
    float4 pay[Ops::kVec4];
    Ops::pack(it, id, pay);
#pragma unroll
    for (int j = 0; j < Ops::kVec4; ++j) leaves[static_cast<size_t>(slot) * Ops::kVec4 + j] = pay[j];
    if (old0 != 0) return;  // parent already marked by the sibling
    int guard = 0;
    while (guard++ < 4096) {
        node = p;
        p = parent[node];
        if (p < 0) return;
        const int bit = nodes[p].left == node ? 1 : 2;
        if (atomicOr(&flags[p], bit) != 0) return;
    }
}

// Dirty refit, pass 2: climb again; arrivals are counted in flags[p] >> 2 and the last of
// the popcount(flags[p] & 3) dirty children finishes p, clears the word and continues.
__global__ __launch_bounds__(kBlock) void k_dirty_merge(const int* __restrict__ ids, int count,
                                                       int n, const int* __restrict__ slot_of,
                                                       const int* __restrict__ parent,
                                                       Node* __restrict__ nodes,
                                                       BNode* __restrict__ bnodes,
                                                       int* __restrict__ flags,
                                                       const int* __restrict__ skip) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= count || skip[i]) return;
    auto links = [&](int v) { return *reinterpret_cast<const int2*>(&nodes[v].left); };
    int p = parent[n - 1 + slot_of[ids[i]]];
    if (p < 0) return;
    int2 lr = links(p);
    int pn = parent[p];
    const int2 none = make_int2(0, 0);
    for (int guard = 0; guard < 4096; ++guard) {
        // the next level's parent and links (static) load while this arrival and box wait
        int2 lrn = none;
        int pnn = -1;
        if (pn >= 0) {
            lrn = links(pn);
            pnn = parent[pn];
        }
        const int old = arrive_add(&flags[p], 4);
        const int need = __popc(old & 3);
        if ((old >> 2) + 1 < need) return;
        finish_node_links<false, false>(nodes, bnodes, p, n, lr, none, none);
        flags[p] = 0;
        if (pn < 0) return;
        p = pn;
        lr = lrn;
        pn = pnn;
    }
}

// ---- 4-wide collapse (lbvh.cu:731-825): even-depth internal nodes ----
__global__ __launch_bounds__(kBlock) void k_wide_flags(const int* __restrict__ depth, int m,
                                                      int* __restrict__ flags) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < m) flags[i] = (depth[i] & 1) == 0 ? 1 : 0;
}

__global__ __launch_bounds__(kBlock) void k_wide_emit(const Node* __restrict__ nodes, int n,
                                                     const int* __restrict__ depth,
                                                     const int* __restrict__ wide_id,
                                                     WideNode* __restrict__ wide) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= n - 1 || (depth[i] & 1) != 0) return;
    WideNode out;
    wide_node_of(nodes, n, wide_id, i, out);
    wide[wide_id[i]] = out;
}

// ---- 4-wide collapse, leaf-size-4 form (wide4_node_of) ----
__global__ __launch_bounds__(kBlock) void k_wide4_flags(const Node* __restrict__ nodes,
                                                       const BNode* __restrict__ bn,
                                                       const int* __restrict__ parent,
                                                       const int* __restrict__ depth, int m,
                                                       int* __restrict__ flags) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < m) flags[i] = ((depth[i] & 1) == 0 && own_small_code(nodes, bn, parent, i) == 0) ? 1 : 0;
}

__global__ __launch_bounds__(kBlock) void k_wide4_emit(const Node* __restrict__ nodes,
                                                      const BNode* __restrict__ bn,
                                                      const int* __restrict__ parent, int n,
                                                      const int* __restrict__ depth,
                                                      const int* __restrict__ wide_id,
                                                      WideNode* __restrict__ wide) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= n - 1 || (depth[i] & 1) != 0 || own_small_code(nodes, bn, parent, i) != 0) return;
    WideNode out;
    wide4_node_of(nodes, bn, n, wide_id, i, out);
    wide[wide_id[i]] = out;
}

// ---- validation (lbvh.cu:613-729) ----
__device__ __forceinline__ bool same_box(const Node& a, Box b) {
    return a.mn[0] == b.lo.x && a.mn[1] == b.lo.y && a.mn[2] == b.lo.z && a.mx[0] == b.hi.x &&
           a.mx[1] == b.hi.y && a.mx[2] == b.hi.z;
}

template <class Ops>
__global__ __launch_bounds__(kBlock) void k_check_nodes(
    const Node* __restrict__ nodes, const BNode* __restrict__ bnodes,
    const float* __restrict__ sorted, int n, int* __restrict__ visited, int* __restrict__ err) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    const int count = 2 * n - 1;
    if (i >= count) return;
    const Node nd = nodes[i];
    if (i < n - 1) {
        if (nd.left < 0 || nd.left >= count || nd.right < 0 || nd.right >= count) {
            atomicAdd(&err[0], 1);
            return;
        }
        atomicAdd(&visited[nd.left], 1);
        atomicAdd(&visited[nd.right], 1);
        const Node l = nodes[nd.left], r = nodes[nd.right];
        Box u;
        u.lo = f3(fmin_t(l.mn[0], r.mn[0]), fmin_t(l.mn[1], r.mn[1]), fmin_t(l.mn[2], r.mn[2]));
        u.hi = f3(fmax_t(l.mx[0], r.mx[0]), fmax_t(l.mx[1], r.mx[1]), fmax_t(l.mx[2], r.mx[2]));
        if (!same_box(nd, u)) atomicAdd(&err[0], 1);
        // the traversal node must mirror the canonical children
        const BNode b = bnodes[i];
        const int lref = nd.left >= n - 1 ? ~(nd.left - (n - 1)) : nd.left;
        const int rref = nd.right >= n - 1 ? ~(nd.right - (n - 1)) : nd.right;
        const bool ok = b.v0.x == l.mn[0] && b.v0.y == l.mn[1] && b.v0.z == l.mn[2] &&
                        b.v0.w == l.mx[0] && b.v1.x == l.mx[1] && b.v1.y == l.mx[2] &&
                        b.v1.z == r.mn[0] && b.v1.w == r.mn[1] && b.v2.x == r.mn[2] &&
                        b.v2.y == r.mx[0] && b.v2.z == r.mx[1] && b.v2.w == r.mx[2] &&
                        __float_as_int(b.v3.x) == lref && __float_as_int(b.v3.y) == rref;
        if (!ok) atomicAdd(&err[0], 1);
    } else {
        const int slot = -nd.left - 1;
        if (slot < 0 || slot >= n) {
            atomicAdd(&err[0], 1);
            return;
        }
        if (i != n - 1 + slot || nd.right != 1) atomicAdd(&err[3], 1);
        if (!same_box(nd, Ops::bounds(sorted + static_cast<size_t>(slot) * Ops::kFloats)))
            atomicAdd(&err[1], 1);
    }
}

__global__ __launch_bounds__(kBlock) void k_check_refs(const int* __restrict__ visited, int count,
                                                      int* __restrict__ err) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < count && visited[i] != (i == 0 ? 0 : 1)) atomicAdd(&err[2], 1);
}

template <class Ops>
__global__ __launch_bounds__(kBlock) void k_check_perm(const int* __restrict__ prim_ids,
                                                      const int* __restrict__ slot_of,
                                                      const float* __restrict__ sorted,
                                                      const float4* __restrict__ leaves,
                                                      const float* __restrict__ items, int n,
                                                      int* __restrict__ hist,
                                                      int* __restrict__ err) {
    const int s = blockIdx.x * kBlock + threadIdx.x;
    if (s >= n) return;
    const int id = prim_ids[s];
    if (id < 0 || id >= n) {
        atomicAdd(&err[4], 1);
        return;
    }
    atomicAdd(&hist[id], 1);
    int bad = slot_of[id] != s;
    float it[Ops::kFloats];
    for (int j = 0; j < Ops::kFloats; ++j) {
        it[j] = sorted[static_cast<size_t>(s) * Ops::kFloats + j];
        bad |= __float_as_uint(it[j]) != __float_as_uint(items[static_cast<size_t>(id) * Ops::kFloats + j]);
    }
    float4 pay[Ops::kVec4];
    Ops::pack(it, id, pay);
    for (int j = 0; j < Ops::kVec4; ++j) {
        const float4 v = leaves[static_cast<size_t>(s) * Ops::kVec4 + j];
        bad |= __float_as_uint(v.x) != __float_as_uint(pay[j].x) ||
               __float_as_uint(v.y) != __float_as_uint(pay[j].y) ||
               __float_as_uint(v.z) != __float_as_uint(pay[j].z) ||
               __float_as_uint(v.w) != __float_as_uint(pay[j].w);
    }
    if (bad) atomicAdd(&err[4], 1);
}

__global__ __launch_bounds__(kBlock) void k_check_hist(const int* __restrict__ hist, int n,
                                                      int* __restrict__ err) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < n && hist[i] != 1) atomicAdd(&err[4], 1);
}

__global__ __launch_bounds__(kBlock) void k_check_depth(const Node* __restrict__ nodes,
                                                       const int* __restrict__ depth, int n,
                                                       int* __restrict__ err) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    const int count = 2 * n - 1;
    if (i >= count) return;
    if (i == 0 && depth[0] != 0) atomicAdd(&err[5], 1);
    if (i < n - 1) {
        const int l = nodes[i].left, r = nodes[i].right;
        if (l >= 0 && l < count && depth[l] != depth[i] + 1) atomicAdd(&err[5], 1);
        if (r >= 0 && r < count && depth[r] != depth[i] + 1) atomicAdd(&err[5], 1);
    }
    if (depth[i] >= kStack) atomicAdd(&err[5], 1);
}

// wide node of every even-depth internal node against a fresh collapse; leaf4: the leaf-size-4
// form (nodes inside a leaf range have none)
__global__ __launch_bounds__(kBlock) void k_check_wide(const Node* __restrict__ nodes,
                                                      const BNode* __restrict__ bn,
                                                      const int* __restrict__ parent, int n,
                                                      const int* __restrict__ depth,
                                                      const int* __restrict__ wide_id,
                                                      const WideNode* __restrict__ wide,
                                                      int leaf4, int* __restrict__ err) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= n - 1 || (depth[i] & 1) != 0) return;
    if (leaf4 && own_small_code(nodes, bn, parent, i) != 0) return;
    WideNode want;
    if (leaf4) wide4_node_of(nodes, bn, n, wide_id, i, want);
    else wide_node_of(nodes, n, wide_id, i, want);
    const WideNode got = wide[wide_id[i]];
    const unsigned* a = reinterpret_cast<const unsigned*>(&want);
    const unsigned* b = reinterpret_cast<const unsigned*>(&got);
    int bad = 0;
    for (int j = 0; j < 32; ++j) bad |= a[j] != b[j];
    if (bad) atomicAdd(&err[6], 1);
}

// Boxes (bottom-up), traversal nodes and depths of a tree whose links and leaves are set;
// shared by the LBVH and SAH builders and topology edits.  `ranges` (one int2 per internal
// node) holds the slot ranges when ranges_ready (the LBVH emit writes them), else they are
// derived first.  Reads the maximum depth back (syncs).
int finish_tree(qk_tree* t, Header* h, int2* ranges, bool ranges_ready, cudaStream_t s) {
    const int n = t->n;
    Node* nodes = static_cast<Node*>(t->nodes);
    if (!ranges_ready) k_ranges_descent<<<blocks_for(n - 1), kBlock, 0, s>>>(nodes, n, ranges);
    k_bottom_up_ranged<kUpSpan><<<blocks_for(n, kUpSpan), kUpSpan, 0, s>>>(nodes, static_cast<BNode*>(t->bnodes),
                                                        t->parent, t->flags, n, ranges);
    stage_mark(kMarkBoxes, s);
    cudaMemsetAsync(&h->max_depth, 0, sizeof(int), s);
    k_depth_anchors<<<blocks_for(n - 1), kBlock, 0, s>>>(t->parent, ranges, n, t->depth_arr);
    k_depth<<<blocks_for(2 * n - 1), kBlock, 0, s>>>(t->parent, ranges, n, t->depth_arr, h);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "tree boxes");
    int depth = 0;
    e = cudaMemcpyAsync(&depth, &h->max_depth, sizeof(int), cudaMemcpyDeviceToHost, s);
    stage_mark(kMarkEnd, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "build depth readback");
    t->depth = depth;
    t->wide_count = 0;
    t->wide_leaf = 0;
    if (depth >= kStack) return fail(QK_ERR_DEPTH, "tree depth %d exceeds %d", depth, kStack - 1);
    return QK_OK;
}

template <class Ops>
int build_lbvh(qk_tree* t, const void* items_v, void* ws, cudaStream_t s) {
    const int n = t->n;
    const float* items = static_cast<const float*>(items_v);
    Carve c{static_cast<char*>(ws)};
    Header* h = c.take<Header>(1);
    uint32_t* codes = c.take<uint32_t>(n);
    uint32_t* idx = c.take<uint32_t>(n);
    uint32_t* codes_s = c.take<uint32_t>(n);
    uint32_t* idx_s = c.take<uint32_t>(n);
    void* sort_ws = c.take<char>(sort_ws_bytes(n));
    Node* nodes = static_cast<Node*>(t->nodes);
    BNode* bn = static_cast<BNode*>(t->bnodes);

    k_header_init<<<1, 32, 0, s>>>(h);
    const int grid = min(blocks_for(n), 148 * 8);
    k_centroid_bounds<Ops><<<grid, kBlock, 0, s>>>(items, n, h);
    k_morton<Ops><<<blocks_for(n), kBlock, 0, s>>>(items, n, h, codes, idx);
    stage_mark(kMarkMorton, s);
    cudaError_t e = sort_pairs(codes, idx, codes_s, idx_s, n, 30, sort_ws, s);
    if (e != cudaSuccess) return cuda_status(e, "build sort");
    stage_mark(kMarkSort, s);
    int2* ranges = build_ranges(ws, t->kind, n, QK_BUILD_LBVH);
    // leaves (the scatter into leaf order) and internal nodes in one pass
    k_emit<Ops><<<blocks_for(n), kBlock, 0, s>>>(items, n, codes_s, idx_s, nodes,
                                                  static_cast<float*>(t->items), t->prim_ids,
                                                  t->slot_of, t->parent, bn,
                                                  static_cast<float4*>(t->leaves), t->flags, ranges);
    stage_mark(kMarkTopo, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "build kernels");
    return finish_tree(t, h, ranges, true, s);
}

template <class Ops>
int refit_impl(qk_tree* t, const void* items, cudaStream_t s) {
    const int n = t->n;
    stage_mark(kMarkStart, s);
    k_refit_leaves<Ops><<<blocks_for(n), kBlock, 0, s>>>(
        static_cast<const float*>(items), n, t->prim_ids, static_cast<Node*>(t->nodes),
        static_cast<float*>(t->items), static_cast<float4*>(t->leaves));
    stage_mark(kMarkScatter, s);
    k_bottom_up<<<blocks_for(n), kBlock, 0, s>>>(static_cast<Node*>(t->nodes),
                                                 static_cast<BNode*>(t->bnodes), t->parent,
                                                 t->flags, n);
    stage_mark(kMarkBoxes, s);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "refit");
    const int st = (t->wide_count > 0 && t->wide) ? wide_emit_all(t, s) : QK_OK;
    stage_mark(kMarkEnd, s);
    return st;
}

template <class Ops>
int refit_dirty_impl(qk_tree* t, const int* ids, const void* items, int count, void* ws,
                     cudaStream_t s) {
    const int n = t->n;
    if (count <= 0) return QK_OK;
    Carve c{static_cast<char*>(ws)};
    Header* h = c.take<Header>(1);
    int* skip = c.take<int>(count);
    stage_mark(kMarkStart, s);
    k_header_init<<<1, 32, 0, s>>>(h);
    k_dirty_mark<Ops><<<blocks_for(count), kBlock, 0, s>>>(
        ids, static_cast<const float*>(items), count, n, t->slot_of, t->parent,
        static_cast<Node*>(t->nodes), static_cast<float*>(t->items),
        static_cast<float4*>(t->leaves), t->flags, skip, h);
    stage_mark(kMarkScatter, s);
    k_dirty_merge<<<blocks_for(count), kBlock, 0, s>>>(ids, count, n, t->slot_of, t->parent,
                                                       static_cast<Node*>(t->nodes),
                                                       static_cast<BNode*>(t->bnodes), t->flags,
                                                       skip);
    stage_mark(kMarkBoxes, s);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "refit dirty");
    const int st = (t->wide_count > 0 && t->wide) ? wide_emit_all(t, s) : QK_OK;
    stage_mark(kMarkEnd, s);
    return st;
}

template <class Ops>
int validate_impl(const qk_tree* t, const void* items, int* err, void* ws, cudaStream_t s) {
    const int n = t->n, count = 2 * n - 1;
    Carve c{static_cast<char*>(ws)};
    int* visited = c.take<int>(count);
    int* hist = c.take<int>(n);
    cudaMemsetAsync(err, 0, 8 * sizeof(int), s);
    cudaMemsetAsync(visited, 0, sizeof(int) * count, s);
    cudaMemsetAsync(hist, 0, sizeof(int) * n, s);
    const Node* nodes = static_cast<const Node*>(t->nodes);
    k_check_nodes<Ops><<<blocks_for(count), kBlock, 0, s>>>(
        nodes, static_cast<const BNode*>(t->bnodes), static_cast<const float*>(t->items), n,
        visited, err);
    k_check_refs<<<blocks_for(count), kBlock, 0, s>>>(visited, count, err);
    k_check_perm<Ops><<<blocks_for(n), kBlock, 0, s>>>(
        t->prim_ids, t->slot_of, static_cast<const float*>(t->items),
        static_cast<const float4*>(t->leaves), static_cast<const float*>(items), n, hist, err);
    k_check_hist<<<blocks_for(n), kBlock, 0, s>>>(hist, n, err);
    k_check_depth<<<blocks_for(count), kBlock, 0, s>>>(nodes, t->depth_arr, n, err);
    if (t->wide_count > 0 && t->wide) {
        k_check_wide<<<blocks_for(n - 1), kBlock, 0, s>>>(
            nodes, static_cast<const BNode*>(t->bnodes), t->parent, n, t->depth_arr, t->wide_id,
            static_cast<const WideNode*>(t->wide), t->wide_leaf == 4 ? 1 : 0, err);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "validate");
}

}  // namespace

int finish_tree_boxes(qk_tree* t, Header* h, int2* ranges, cudaStream_t s) {
    return finish_tree(t, h, ranges, false, s);
}

// workspace of the builders themselves; the bottom-up ranges follow it
size_t build_core_bytes(int kind, int n, int builder) {
    (void)kind;
    Carve c;
    c.take<Header>(1);
    c.take<uint32_t>(n);
    c.take<uint32_t>(n);
    c.take<uint32_t>(n);
    c.take<uint32_t>(n);
    c.take<char>(sort_ws_bytes(n));
    size_t need = c.used;
    // refit_dirty and wide_build share the build workspace
    Carve d;
    d.take<Header>(1);
    d.take<int>(n);
    if (d.used > need) need = d.used;
    Carve w;
    w.take<char>(scan_ws_bytes(n));
    if (w.used > need) need = w.used;
    if (builder == QK_BUILD_SAH || builder == QK_BUILD_SAH4) need = std::max(need, sah_ws_bytes(n));
    return need;
}

size_t build_ws_bytes(int kind, int n, int builder) {
    return (build_core_bytes(kind, n, builder) + 255) / 256 * 256 + sizeof(int2) * static_cast<size_t>(n);
}

// the int2 per internal node the bottom-up pass records leaf-slot ranges in
int2* build_ranges(void* ws, int kind, int n, int builder) {
    return reinterpret_cast<int2*>(static_cast<char*>(ws) +
                                   (build_core_bytes(kind, n, builder) + 255) / 256 * 256);
}

int build_tree(qk_tree* t, int builder, int bins, const void* items, void* ws, size_t ws_bytes,
               cudaStream_t s) {
    (void)ws_bytes;
    stage_mark(kMarkStart, s);
    if (builder == QK_BUILD_SAH || builder == QK_BUILD_SAH4) {
        cudaMemsetAsync(t->flags, 0, sizeof(int) * static_cast<size_t>(t->n - 1), s);
        const int st = build_sah(t, bins, builder == QK_BUILD_SAH4 ? 4 : 1, items, ws, s);
        if (st != QK_OK) return st;
        return finish_tree(t, static_cast<Header*>(ws), build_ranges(ws, t->kind, t->n, builder),
                           false, s);
    }
    switch (t->kind) {
        case kTri: return build_lbvh<TriOps>(t, items, ws, s);
        case kPoint: return build_lbvh<PointOps>(t, items, ws, s);
        case kGauss: return build_lbvh<GaussOps>(t, items, ws, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", t->kind);
    }
}

int refit_tree(qk_tree* t, const void* items, cudaStream_t s) {
    switch (t->kind) {
        case kTri: return refit_impl<TriOps>(t, items, s);
        case kPoint: return refit_impl<PointOps>(t, items, s);
        case kGauss: return refit_impl<GaussOps>(t, items, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", t->kind);
    }
}

int refit_tree_dirty(qk_tree* t, const int* ids, const void* items, int count, void* ws,
                     cudaStream_t s) {
    switch (t->kind) {
        case kTri: return refit_dirty_impl<TriOps>(t, ids, items, count, ws, s);
        case kPoint: return refit_dirty_impl<PointOps>(t, ids, items, count, ws, s);
        case kGauss: return refit_dirty_impl<GaussOps>(t, ids, items, count, ws, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", t->kind);
    }
}

// re-emits the wide nodes in the form tree->wide_leaf records (after a refit)
int wide_emit_all(qk_tree* t, cudaStream_t s) {
    const int n = t->n;
    if (t->wide_leaf == 4) {
        k_wide4_emit<<<blocks_for(n - 1), kBlock, 0, s>>>(
            static_cast<const Node*>(t->nodes), static_cast<const BNode*>(t->bnodes), t->parent, n,
            t->depth_arr, t->wide_id, static_cast<WideNode*>(t->wide));
    } else {
        k_wide_emit<<<blocks_for(n - 1), kBlock, 0, s>>>(static_cast<const Node*>(t->nodes), n,
                                                         t->depth_arr, t->wide_id,
                                                         static_cast<WideNode*>(t->wide));
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "wide emit");
}

int wide_build(qk_tree* t, int leaf, void* ws, size_t ws_bytes, cudaStream_t s) {
    (void)ws_bytes;
    const int n = t->n, m = n - 1;
    if (leaf == 4) {
        k_wide4_flags<<<blocks_for(m), kBlock, 0, s>>>(static_cast<const Node*>(t->nodes),
                                                       static_cast<const BNode*>(t->bnodes),
                                                       t->parent, t->depth_arr, m, t->flags);
    } else {
        k_wide_flags<<<blocks_for(m), kBlock, 0, s>>>(t->depth_arr, m, t->flags);
    }
    // wide_id = exclusive scan of the flags; count = last prefix + last flag
    cudaError_t e = scan_exclusive(t->flags, t->wide_id, m, false, ws, s);
    if (e != cudaSuccess) return cuda_status(e, "wide scan");
    int tail[2] = {0, 0};
    e = cudaMemcpyAsync(&tail[0], t->wide_id + (m - 1), sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&tail[1], t->flags + (m - 1), sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "wide count readback");
    // the flags are scratch of the bottom-up pass, which expects zeros
    cudaMemsetAsync(t->flags, 0, sizeof(int) * static_cast<size_t>(m), s);
    t->wide_count = tail[0] + tail[1];
    t->wide_leaf = leaf == 4 ? 4 : 1;
    if (t->wide_count <= 0) return fail(QK_ERR_INVALID, "no wide nodes");
    // first call without a node buffer only sizes it
    if (t->wide == nullptr) return QK_OK;
    return wide_emit_all(t, s);
}

size_t validate_ws_bytes(int n) {
    Carve c;
    c.take<int>(2 * static_cast<size_t>(n));
    c.take<int>(n);
    return c.used;
}

int validate_tree(const qk_tree* t, const void* items, int* errors, void* ws, cudaStream_t s) {
    switch (t->kind) {
        case kTri: return validate_impl<TriOps>(t, items, errors, ws, s);
        case kPoint: return validate_impl<PointOps>(t, items, errors, ws, s);
        case kGauss: return validate_impl<GaussOps>(t, items, errors, ws, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", t->kind);
    }
}

}  // namespace qk
