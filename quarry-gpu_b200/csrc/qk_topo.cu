// qk_topo.cu -- topology edits of a built tree: quarry's updateBVHGPU / updatePointBVHGPU /
// updateGaussianBVHGPU (src/gpu/gpu_bvh.h:182-213, src/gpu/lbvh.cu:2543-3099) with the same
// edit script (deleted old indices, inserted new indices, appended tail, moved new indices),
// done by rebuilding only the small subtrees the edit touches.
//
// Every subtree of the engine's trees covers a contiguous run of leaf slots (LBVH and SAH
// both emit them that way, and this pass keeps it so).  Plan, one host synchronisation:
//   * every old internal node's (first slot, leaf count) comes from its leftmost and rightmost
//     leaves;
//   * a cut is a maximal subtree of at most S leaves (its parent holds more), so the cuts
//     partition the leaves.  A deleted leaf rebuilds its cut.  A new primitive descends from
//     the root toward the child whose box grows least and joins the cut it reaches: new
//     geometry lands next to its neighbours instead of at the end of the slot order;
//   * one exclusive scan over the old slots, weighted by survival plus the new primitives a
//     cut receives (counted at the cut's first slot), gives every surviving leaf its new slot
//     and every cut its block of new slots, so subtrees stay contiguous;
//   * one exclusive scan over the old nodes gives the new numbering: a kept internal node
//     (outside the cuts, both sides non-empty) takes one id, a cut of m >= 2 primitives takes
//     m - 1 (its root and forest), and a node left with one non-empty side is spliced out.
//     The root keeps id 0 because it comes first.
// Emit: kept nodes are relinked through spliced nodes; kept leaves move to their new slots
// with their new scene indices; each cut's primitives are staged in its slot block and built
// by the SAH block builder (one thread block per cut, qk_sah.cu); moved primitives are
// rewritten; boxes, traversal nodes, small-subtree codes and depths then come from the
// shared bottom-up pass over the whole new tree.  Queries are tree-invariant, so results
// equal a fresh build's.  The plan declines (the caller rebuilds) when the root is a cut or
// would be spliced, a cut would exceed 1024 primitives, the cuts hold more than a quarter of
// the new leaves, or a forest could pass the depth limit.
#include <algorithm>

#include "qk_build.cuh"

namespace qk {
namespace {

constexpr int kForestMax = 1024;  // the SAH block builder's largest range
constexpr int kDepthLimit = 62;   // the builders' depth cap (traversal stacks hold 64)

struct TopoPlan {
    int error;       // bit 0 deleted, 1 inserted, 2 moved: out of order or range
    int cuts;        // cut count
    int max_new;     // largest cut after the edit
    int old_leaves;  // leaves under the cuts before the edit
    int new_leaves;  // ... after it
    int ids;         // internal ids handed out (must be n_new - 1)
    int root;        // 0 fine; 1 the root is a cut; 2 the root loses a side or empties
    int depth_need;  // deepest forest bound: cut depth + ceil(log2(m))
    int spliced;     // internal nodes spliced out
    int slots;       // new slot total (must be n_new)
    int emit_err;    // out-of-range writes skipped by the emit
    int emit_site;   // which checks fired (EmitSite bits); must follow emit_err
    int forest_err;  // errors reported by the forest builders
    int noncontig;   // old subtrees whose slots are not contiguous
    int pad[2];
};

// The emit checks, one bit each in TopoPlan::emit_site (reported with the error).
enum EmitSite {
    kSiteNodes = 1,        // a kept node's new id or relinked child out of range
    kSiteKeptLeaf = 2,     // a surviving leaf outside the cuts: slot or index out of range
    kSiteStageCut = 4,     // a cut survivor's staging position out of range
    kSiteStageExtra = 8,   // a new primitive's staging position out of range
    kSiteCutOrder = 16,    // a forest position whose staged entry is out of range
    kSiteCutLeaf = 32,     // a forest leaf: slot or index out of range
    kSiteMovedId = 64,     // a moved index out of range
    kSiteMovedLeaf = 128,  // a moved primitive's slot out of range
};

// Counts a failed emit check at `err` (TopoPlan::emit_err) and records its site.
__device__ __forceinline__ void emit_fault(int* err, int site) {
    atomicAdd(err, 1);
    atomicOr(err + 1, site);
}

struct TopoWs {
    TopoPlan* plan;
    Header* h;
    int* del_flag;     // n_old: old scene index deleted
    int2* range;       // n_old - 1: (first slot, leaves) of every old internal node
    int* wslot;        // n_old + 1: slot weights, then new slot starts (exclusive scan)
    int* cut_mark;     // 2 n_old: 1 for a cut node; then the cut list index (scan)
    int* cut_extra;    // 2 n_old - 1: new primitives per cut node
    int* cut_list;     // cut node ids, ascending
    int* cut_of_slot;  // n_old: the cut node holding the slot, or -1
    int* wnode;        // 2 n_old: node weights, then new internal ids (scan)
    int* shifts;       // n_inserted: inserted[k] - k
    uint32_t* ext_key;
    uint32_t* ext_val;
    uint32_t* ext_key_s;
    uint32_t* ext_val_s;
    int4* tasks;       // one forest task per cut
    int* id_base;
    float4* cen;       // n_new staged centroids / boxes, indexed by new slot
    float4* plo;
    float4* phi;
    float* st_items;   // n_new staged records
    int* st_id;        // n_new staged new scene indices
    int* order;        // n_new
    int* tmp;          // n_new: partition scratch of the forest builders
    int2* new_range;   // n_new - 1: bottom-up ranges of the new tree
    void* sort_ws;
    void* scan_ws;
};

TopoWs carve_topo(Carve& c, int kind, int n_old, int n_new, int n_extra) {
    const int fl = qk_stride_floats(kind);
    const int max_cuts = n_old + n_extra + 1;
    TopoWs w;
    w.plan = c.take<TopoPlan>(1);
    w.h = c.take<Header>(1);
    w.del_flag = c.take<int>(n_old);
    w.range = c.take<int2>(n_old);
    w.wslot = c.take<int>(n_old + 1);
    w.cut_mark = c.take<int>(2 * static_cast<size_t>(n_old));
    w.cut_extra = c.take<int>(2 * static_cast<size_t>(n_old));
    w.cut_list = c.take<int>(max_cuts);
    w.cut_of_slot = c.take<int>(n_old);
    w.wnode = c.take<int>(2 * static_cast<size_t>(n_old));
    w.shifts = c.take<int>(n_extra + 1);
    w.ext_key = c.take<uint32_t>(n_extra + 1);
    w.ext_val = c.take<uint32_t>(n_extra + 1);
    w.ext_key_s = c.take<uint32_t>(n_extra + 1);
    w.ext_val_s = c.take<uint32_t>(n_extra + 1);
    w.tasks = c.take<int4>(max_cuts);
    w.id_base = c.take<int>(max_cuts);
    w.cen = c.take<float4>(n_new);
    w.plo = c.take<float4>(n_new);
    w.phi = c.take<float4>(n_new);
    w.st_items = c.take<float>(static_cast<size_t>(n_new) * fl);
    w.st_id = c.take<int>(n_new);
    w.order = c.take<int>(n_new);
    w.tmp = c.take<int>(n_new);
    w.new_range = c.take<int2>(n_new);
    w.sort_ws = c.take<char>(sort_ws_bytes(n_extra + 1));
    w.scan_ws = c.take<char>(scan_ws_bytes(2 * n_old + 1));
    return w;
}

// ---------------------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int2 node_range(const int2* __restrict__ range, int v, int n) {
    return v >= n - 1 ? make_int2(v - (n - 1), 1) : range[v];
}

// primitives under old node v after the edit (new slots it spans)
__device__ __forceinline__ int new_count(const int2* __restrict__ range,
                                         const int* __restrict__ xs, int v, int n) {
    const int2 r = node_range(range, v, n);
    return xs[r.x + r.y] - xs[r.x];
}

// number of entries of the ascending array a[0..m) below x / at most x
__device__ __forceinline__ int count_below(const int* __restrict__ a, int m, int x) {
    int lo = 0, hi = m;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ int count_at_most(const int* __restrict__ a, int m, int x) {
    int lo = 0, hi = m;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

struct EditDev {
    const int* deleted;
    int n_del;
    const int* inserted;
    int n_ins;
    int appended;
    const int* moved;
    int n_mov;
    const float* extra;
    const float* moved_items;
    int n_old, n_new;
};

// new scene index of surviving old scene index j: its survivor rank r, pushed right by every
// insertion that lands at or before it (shifts[k] = inserted[k] - k survivors precede it)
__device__ __forceinline__ int remap_id(const EditDev& e, const int* __restrict__ shifts, int j) {
    const int r = j - count_below(e.deleted, e.n_del, j);
    return r + count_at_most(shifts, e.n_ins, r);
}

__device__ __forceinline__ int extra_id(const EditDev& e, int k) {
    return k < e.n_ins ? e.inserted[k] : e.n_new - e.appended + (k - e.n_ins);
}

__device__ __forceinline__ float half_area(const Box& b) {
    const float dx = b.hi.x - b.lo.x, dy = b.hi.y - b.lo.y, dz = b.hi.z - b.lo.z;
    return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ Box join(const Box& a, const Box& b) {
    Box u;
    u.lo = f3(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y), fminf(a.lo.z, b.lo.z));
    u.hi = f3(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y), fmaxf(a.hi.z, b.hi.z));
    return u;
}

// Every emit write is bounds-checked: a slot or index outside the new tree is counted in
// `err` (read back as an error before the tree is used) and skipped.
template <class Ops>
__device__ __forceinline__ void write_leaf(const qk_tree& t, int slot, const float* it, int id,
                                           int* err, int site) {
    const int n = t.n;
    if (slot < 0 || slot >= n || id < 0 || id >= n) {
        emit_fault(err, site);
        return;
    }
    float* dst = static_cast<float*>(t.items) + static_cast<size_t>(slot) * Ops::kFloats;
#pragma unroll
    for (int j = 0; j < Ops::kFloats; ++j) dst[j] = it[j];
    t.prim_ids[slot] = id;
    t.slot_of[id] = slot;
    const Box b = Ops::bounds(it);
    float4* leaf = reinterpret_cast<float4*>(static_cast<Node*>(t.nodes) + (n - 1 + slot));
    leaf[0] = make_float4(b.lo.x, b.lo.y, b.lo.z, b.hi.x);
    leaf[1] = make_float4(b.hi.y, b.hi.z, __int_as_float(-(slot + 1)), __int_as_float(1));
    float4 pay[Ops::kVec4];
    Ops::pack(it, id, pay);
    float4* lv = static_cast<float4*>(t.leaves) + static_cast<size_t>(slot) * Ops::kVec4;
#pragma unroll
    for (int j = 0; j < Ops::kVec4; ++j) lv[j] = pay[j];
}

// ---------------------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------------------
// the edit script's order and range rules (src/gpu/lbvh.cu:2556-2590); deleted flags; shifts
__global__ __launch_bounds__(kBlock) void k_topo_check(EditDev e, int* __restrict__ del_flag,
                                                      int* __restrict__ shifts,
                                                      TopoPlan* __restrict__ plan) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < e.n_del) {
        const int j = e.deleted[i];
        if (j < 0 || j >= e.n_old || (i > 0 && j <= e.deleted[i - 1])) atomicOr(&plan->error, 1);
        else del_flag[j] = 1;
    }
    if (i < e.n_ins) {
        const int j = e.inserted[i];
        if (j < 0 || j >= e.n_new - e.appended || (i > 0 && j <= e.inserted[i - 1]))
            atomicOr(&plan->error, 2);
        shifts[i] = j - i;
    }
    if (i < e.n_mov) {
        const int j = e.moved[i];
        if (j < 0 || j >= e.n_new) atomicOr(&plan->error, 4);
    }
}

// (first slot, leaves) of every old internal node.  Every subtree covers an ordered
// contiguous run of slots (left child's run first), so its run is [leftmost leaf, rightmost
// leaf]: two descents, no atomics.  k_topo_weights verifies the assumption node by node; a
// run that comes out inverted is recorded as empty and reported.
__global__ __launch_bounds__(kBlock) void k_topo_ranges(const Node* __restrict__ nodes,
                                                       int2* __restrict__ range, int n,
                                                       TopoPlan* __restrict__ plan) {
    const int v = blockIdx.x * kBlock + threadIdx.x;
    if (v >= n - 1) return;
    int a = v, b = v;
    for (int guard = 0; a < n - 1 && guard < 4096; ++guard) a = nodes[a].left;
    for (int guard = 0; b < n - 1 && guard < 4096; ++guard) b = nodes[b].right;
    const int first = a - (n - 1), last = b - (n - 1);
    if (a < n - 1 || b < n - 1 || last < first) {
        atomicAdd(&plan->noncontig, 1);
        range[v] = make_int2(0, 0);
        return;
    }
    range[v] = make_int2(first, last - first + 1);
}

__global__ __launch_bounds__(kBlock) void k_topo_kept(const int* __restrict__ prim_ids,
                                                     const int* __restrict__ del_flag, int n,
                                                     int* __restrict__ wslot) {
    const int s = blockIdx.x * kBlock + threadIdx.x;
    if (s < n) wslot[s] = del_flag[prim_ids[s]] ? 0 : 1;
    if (s == n) wslot[n] = 0;
}

// the cut of a deleted leaf: its highest ancestor of at most S leaves
__global__ __launch_bounds__(kBlock) void k_topo_cut_deleted(EditDev e,
                                                            const int* __restrict__ slot_of,
                                                            const int* __restrict__ parent,
                                                            const int2* __restrict__ range,
                                                            int S, int* __restrict__ cut_mark) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= e.n_del) return;
    const int j = e.deleted[i];
    if (j < 0 || j >= e.n_old) return;
    const int n = e.n_old;
    int v = n - 1 + slot_of[j];
    for (int guard = 0; guard < 4096; ++guard) {
        const int p = parent[v];
        if (p < 0 || range[p].y > S) break;
        v = p;
    }
    cut_mark[v] = 1;
}

// the cut a new primitive joins: descend from the root toward the child whose box grows
// least (ties to the left) until a subtree of at most S leaves
template <class Ops>
__global__ __launch_bounds__(kBlock) void k_topo_cut_extra(EditDev e, const BNode* __restrict__ bn,
                                                          const int2* __restrict__ range, int S,
                                                          int* __restrict__ cut_mark,
                                                          int* __restrict__ cut_extra,
                                                          uint32_t* __restrict__ key,
                                                          uint32_t* __restrict__ val) {
    const int k = blockIdx.x * kBlock + threadIdx.x;
    const int n_extra = e.n_ins + e.appended;
    if (k >= n_extra) return;
    const int n = e.n_old;
    const Box b = Ops::bounds(e.extra + static_cast<size_t>(k) * Ops::kFloats);
    int v = 0;
    for (int guard = 0; guard < 4096 && range[v].y > S; ++guard) {
        const float4* p = reinterpret_cast<const float4*>(bn + v);
        const float4 a = p[0], bb = p[1], c = p[2], d = p[3];
        Box lb, rb;
        lb.lo = f3(a.x, a.y, a.z);
        lb.hi = f3(a.w, bb.x, bb.y);
        rb.lo = f3(bb.z, bb.w, c.x);
        rb.hi = f3(c.y, c.z, c.w);
        const float gl = half_area(join(lb, b)) - half_area(lb);
        const float gr = half_area(join(rb, b)) - half_area(rb);
        const int ref = gr < gl ? __float_as_int(d.y) : __float_as_int(d.x);
        v = ref >= 0 ? ref : n - 1 + ~ref;
        if (v >= n - 1) break;
    }
    cut_mark[v] = 1;
    atomicAdd(&cut_extra[v], 1);
    key[k] = static_cast<uint32_t>(v);
    val[k] = static_cast<uint32_t>(k);
}

// new primitives of a cut counted at its first slot
__global__ __launch_bounds__(kBlock) void k_topo_extra_slots(const int* __restrict__ cut_mark,
                                                            const int* __restrict__ cut_extra,
                                                            const int2* __restrict__ range, int n,
                                                            int* __restrict__ wslot) {
    const int v = blockIdx.x * kBlock + threadIdx.x;
    if (v >= 2 * n - 1 || !cut_mark[v] || cut_extra[v] == 0) return;
    atomicAdd(&wslot[node_range(range, v, n).x], cut_extra[v]);
}

__global__ __launch_bounds__(kBlock) void k_topo_cut_list(const int* __restrict__ rank, int n,
                                                         int* __restrict__ list) {
    const int v = blockIdx.x * kBlock + threadIdx.x;
    if (v < 2 * n - 1 && rank[v + 1] != rank[v]) list[rank[v]] = v;
}

// per cut (one block each): mark its slots, plan statistics
__global__ __launch_bounds__(kBlock) void k_topo_cuts(const int* __restrict__ list,
                                                     const int* __restrict__ ncut_p,
                                                     const int2* __restrict__ range,
                                                     const int* __restrict__ xs,
                                                     const int* __restrict__ depth, int n,
                                                     int* __restrict__ cut_of_slot,
                                                     TopoPlan* __restrict__ plan) {
    const int ncut = *ncut_p;
    for (int ti = blockIdx.x; ti < ncut; ti += gridDim.x) {
        const int c = list[ti];
        const int2 r = node_range(range, c, n);
        for (int s = r.x + threadIdx.x; s < r.x + r.y; s += kBlock) cut_of_slot[s] = c;
        if (threadIdx.x == 0) {
            const int m = xs[r.x + r.y] - xs[r.x];
            atomicMax(&plan->max_new, m);
            atomicAdd(&plan->old_leaves, r.y);
            atomicAdd(&plan->new_leaves, m);
            const int lg = m <= 1 ? 0 : 32 - __clz(m - 1);
            atomicMax(&plan->depth_need, depth[c] + lg);
            if (c == 0) plan->root = 1;
        }
    }
}

// ids per old node: a kept internal node 1, a cut of m primitives m - 1, otherwise 0
__global__ __launch_bounds__(kBlock) void k_topo_weights(const Node* __restrict__ nodes,
                                                        const int* __restrict__ cut_rank,
                                                        const int2* __restrict__ range,
                                                        const int* __restrict__ xs,
                                                        const int* __restrict__ cut_of_slot,
                                                        int n, int* __restrict__ w,
                                                        TopoPlan* __restrict__ plan) {
    const int v = blockIdx.x * kBlock + threadIdx.x;
    if (v >= 2 * n - 1) return;
    const bool is_cut = cut_rank[v + 1] != cut_rank[v];
    const int m = new_count(range, xs, v, n);
    if (v < n - 1) {
        const int2 r = range[v];
        const int2 rl = node_range(range, nodes[v].left, n);
        const int2 rr = node_range(range, nodes[v].right, n);
        if (rl.x != r.x || rr.x != rl.x + rl.y || rl.y + rr.y != r.y) atomicAdd(&plan->noncontig, 1);
    }
    int wt = 0;
    if (is_cut) {
        wt = m > 1 ? m - 1 : 0;
    } else if (v < n - 1) {
        const int2 r = range[v];
        const int c = cut_of_slot[r.x];
        const bool inside = c >= 0 && r.y < node_range(range, c, n).y;
        if (!inside) {
            const int ml = new_count(range, xs, nodes[v].left, n);
            const int mr = new_count(range, xs, nodes[v].right, n);
            const bool split = ml > 0 && mr > 0;
            wt = split ? 1 : 0;
            if (!split && m > 0) atomicAdd(&plan->spliced, 1);
            if (v == 0 && !split) plan->root = 2;
        }
    }
    w[v] = wt;
}

__global__ void k_topo_totals(TopoPlan* __restrict__ plan, const int* __restrict__ xs, int n_old,
                              const int* __restrict__ rank, const int* __restrict__ ids) {
    plan->slots = xs[n_old];
    plan->cuts = rank[2 * n_old - 1];
    plan->ids = ids[2 * n_old - 1];
}

// ---------------------------------------------------------------------------------------
// emit
// ---------------------------------------------------------------------------------------
struct Relink {
    const Node* nodes;
    const int* rank;   // cut marks, scanned
    const int2* range;
    const int* xs;
    const int* ids;    // new internal ids, scanned
    int n_old, n_new;
};

// new reference of old child c of a kept node: through spliced nodes to what survives
__device__ __forceinline__ int relink(const Relink& R, int c) {
    for (int guard = 0; guard < 4096; ++guard) {
        const int2 r = node_range(R.range, c, R.n_old);
        if (R.rank[c + 1] != R.rank[c]) {
            const int m = R.xs[r.x + r.y] - R.xs[r.x];
            return m == 1 ? R.n_new - 1 + R.xs[r.x] : R.ids[c];
        }
        if (c >= R.n_old - 1) return R.n_new - 1 + R.xs[r.x];
        const int l = R.nodes[c].left, rr = R.nodes[c].right;
        const int ml = new_count(R.range, R.xs, l, R.n_old);
        const int mr = new_count(R.range, R.xs, rr, R.n_old);
        if (ml == 0) c = rr;
        else if (mr == 0) c = l;
        else return R.ids[c];
    }
    return -1;
}

__global__ __launch_bounds__(kBlock) void k_topo_nodes(Relink R, qk_tree t, int* err) {
    const int v = blockIdx.x * kBlock + threadIdx.x;
    if (v >= R.n_old - 1) return;
    if (R.rank[v + 1] != R.rank[v] || R.ids[v + 1] - R.ids[v] != 1) return;  // not kept
    const int id = R.ids[v];
    const int l = relink(R, R.nodes[v].left);
    const int r = relink(R, R.nodes[v].right);
    const int n = R.n_new;
    if (id < 0 || id >= n - 1 || l < 0 || l >= 2 * n - 1 || r < 0 || r >= 2 * n - 1) {
        emit_fault(err, kSiteNodes);
        return;
    }
    Node* nodes = static_cast<Node*>(t.nodes);
    nodes[id].left = l;
    nodes[id].right = r;
    t.parent[l] = id;
    t.parent[r] = id;
    const int lref = l >= n - 1 ? ~(l - (n - 1)) : l;
    const int rref = r >= n - 1 ? ~(r - (n - 1)) : r;
    static_cast<BNode*>(t.bnodes)[id].v3 =
        make_float4(__int_as_float(lref), __int_as_float(rref), 0.0f, 0.0f);
}

// surviving leaves outside the cuts: to their new slots with their new scene indices
template <class Ops>
__global__ __launch_bounds__(kBlock) void k_topo_kept_leaves(EditDev e, const qk_tree old_t,
                                                            qk_tree t,
                                                            const int* __restrict__ del_flag,
                                                            const int* __restrict__ cut_of_slot,
                                                            const int* __restrict__ xs,
                                                            const int* __restrict__ shifts,
                                                            int* err) {
    __shared__ __align__(16) float stage[kBlock / 32][emit_stage_floats<Ops>()];
    const int s = blockIdx.x * kBlock + threadIdx.x;
    const int lane = threadIdx.x & 31;
    if ((s & ~31) >= e.n_old) return;  // whole warps
    int j = 0;
    bool mine = s < e.n_old;
    if (mine) {
        j = old_t.prim_ids[s];
        mine = !del_flag[j] && cut_of_slot[s] < 0;
    }
    float buf[Ops::kFloats];
    const float* it = static_cast<const float*>(old_t.items) + static_cast<size_t>(mine ? s : 0) * Ops::kFloats;
#pragma unroll
    for (int q = 0; q < Ops::kFloats; ++q) buf[q] = mine ? it[q] : 0.0f;
    const int slot = mine ? xs[s] : -1;
    const int id = mine ? remap_id(e, shifts, j) : 0;
    // a warp whose 32 slots all survive into 32 consecutive in-range new slots (most of them,
    // for small edits) writes through the emit's staged leaf writer; any other lane alone,
    // with the bounds checks
    const int slot0 = __shfl_sync(0xffffffffu, slot, 0);
    const bool run = __all_sync(0xffffffffu, mine && slot == slot0 + lane && id >= 0 && id < t.n) &&
                     slot0 >= 0 && slot0 + 32 <= t.n;
    if (run) {
        store_leaves_warp<Ops>(buf, id, t.n, static_cast<Node*>(t.nodes),
                               static_cast<float*>(t.items), t.prim_ids, t.slot_of,
                               static_cast<float4*>(t.leaves), slot0, 32, stage[threadIdx.x >> 5]);
    } else if (mine) {
        write_leaf<Ops>(t, slot, buf, id, err, kSiteKeptLeaf);
    }
}

template <class Ops>
__device__ __forceinline__ void stage(const float* it, int pos, int id, float* st_items,
                                      int* st_id, float4* cen, float4* plo, float4* phi,
                                      int* order, int n, int* err, int site) {
    if (pos < 0 || pos >= n) {
        emit_fault(err, site);
        return;
    }
    float buf[Ops::kFloats];
#pragma unroll
    for (int q = 0; q < Ops::kFloats; ++q) buf[q] = it[q];
#pragma unroll
    for (int q = 0; q < Ops::kFloats; ++q) st_items[static_cast<size_t>(pos) * Ops::kFloats + q] = buf[q];
    st_id[pos] = id;
    const float3 c = Ops::centroid(buf);
    const Box b = Ops::bounds(buf);
    cen[pos] = make_float4(c.x, c.y, c.z, 0.0f);
    plo[pos] = make_float4(b.lo.x, b.lo.y, b.lo.z, 0.0f);
    phi[pos] = make_float4(b.hi.x, b.hi.y, b.hi.z, 0.0f);
    order[pos] = pos;
}

// per cut (one block each): its survivors staged at their new slots; its forest task
template <class Ops>
__global__ __launch_bounds__(kBlock) void k_topo_stage_cuts(
    EditDev e, const qk_tree old_t, const int* __restrict__ list, const int* __restrict__ ncut_p,
    const int2* __restrict__ range, const int* __restrict__ xs, const int* __restrict__ del_flag,
    const int* __restrict__ shifts, const int* __restrict__ ids, float* st_items, int* st_id,
    float4* cen, float4* plo, float4* phi, int* order, int4* __restrict__ tasks,
    int* __restrict__ id_base, int* err) {
    const int ncut = *ncut_p;
    const int n = e.n_old;
    for (int ti = blockIdx.x; ti < ncut; ti += gridDim.x) {
        const int c = list[ti];
        const int2 r = node_range(range, c, n);
        for (int s = r.x + threadIdx.x; s < r.x + r.y; s += kBlock) {
            const int j = old_t.prim_ids[s];
            if (del_flag[j]) continue;
            stage<Ops>(static_cast<const float*>(old_t.items) + static_cast<size_t>(s) * Ops::kFloats,
                       xs[s], remap_id(e, shifts, j), st_items, st_id, cen, plo, phi, order,
                       e.n_new, err, kSiteStageCut);
        }
        if (threadIdx.x == 0) {
            const int B = xs[r.x], m = xs[r.x + r.y] - B;
            tasks[ti] = make_int4(B, B + m, m >= 2 ? ids[c] : -1, old_t.depth_arr[c]);
            id_base[ti] = ids[c] + 1;
        }
    }
}

// cut node of every new primitive -> its cut's rank in the cut list
__global__ __launch_bounds__(kBlock) void k_topo_extra_rank(const int* __restrict__ cut_rank,
                                                           int n_extra, uint32_t* __restrict__ key) {
    const int k = blockIdx.x * kBlock + threadIdx.x;
    if (k < n_extra) key[k] = static_cast<uint32_t>(cut_rank[key[k]]);
}

// new primitives, sorted by cut rank: after the cut's first-slot survivor (when it survives)
template <class Ops>
__global__ __launch_bounds__(kBlock) void k_topo_stage_extra(
    EditDev e, const qk_tree old_t, const uint32_t* __restrict__ key, const uint32_t* __restrict__ val,
    const int* __restrict__ list, const int2* __restrict__ range, const int* __restrict__ xs,
    const int* __restrict__ del_flag, float* st_items, int* st_id, float4* cen, float4* plo,
    float4* phi, int* order, int* err) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    const int n_extra = e.n_ins + e.appended;
    if (i >= n_extra) return;
    const int ck = static_cast<int>(key[i]);
    int lo = 0, hi = i;  // first sorted entry of this cut
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (static_cast<int>(key[mid]) < ck) lo = mid + 1;
        else hi = mid;
    }
    const int c = list[ck];
    const int2 r = node_range(range, c, e.n_old);
    const int first_kept = del_flag[old_t.prim_ids[r.x]] ? 0 : 1;
    const int k = static_cast<int>(val[i]);
    stage<Ops>(e.extra + static_cast<size_t>(k) * Ops::kFloats, xs[r.x] + first_kept + (i - lo),
               extra_id(e, k), st_items, st_id, cen, plo, phi, order, e.n_new, err,
               kSiteStageExtra);
}

// per cut: the built order's primitives into the new tree's leaves
template <class Ops>
__global__ __launch_bounds__(kBlock) void k_topo_cut_leaves(const int4* __restrict__ tasks,
                                                           const int* __restrict__ ncut_p,
                                                           const int* __restrict__ order,
                                                           const float* __restrict__ st_items,
                                                           const int* __restrict__ st_id,
                                                           qk_tree t, int* err) {
    const int ncut = *ncut_p;
    for (int ti = blockIdx.x; ti < ncut; ti += gridDim.x) {
        const int4 tk = tasks[ti];
        for (int pos = tk.x + threadIdx.x; pos < tk.y; pos += kBlock) {
            const int src = order[pos];
            if (src < 0 || src >= t.n) {
                emit_fault(err, kSiteCutOrder);
                continue;
            }
            write_leaf<Ops>(t, pos, st_items + static_cast<size_t>(src) * Ops::kFloats, st_id[src],
                            err, kSiteCutLeaf);
        }
    }
}

template <class Ops>
__global__ __launch_bounds__(kBlock) void k_topo_moved(EditDev e, qk_tree t, int* err) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= e.n_mov) return;
    const int id = e.moved[i];
    if (id < 0 || id >= t.n) {
        emit_fault(err, kSiteMovedId);
        return;
    }
    write_leaf<Ops>(t, t.slot_of[id], e.moved_items + static_cast<size_t>(i) * Ops::kFloats, id,
                    err, kSiteMovedLeaf);
}

template <class Ops>
int update_impl(const qk_tree* old_t, qk_tree* new_t, const qk_topo_edit* ed, int S, int bins,
                qk_topo_info* info, void* ws, cudaStream_t s) {
    const int n_old = old_t->n;
    const int n_new = new_t->n;
    const int n_extra = ed->n_inserted + ed->appended;
    Carve c{static_cast<char*>(ws)};
    TopoWs w = carve_topo(c, old_t->kind, n_old, n_new, n_extra);
    EditDev e{ed->deleted, ed->n_deleted, ed->inserted, ed->n_inserted, ed->appended, ed->moved,
              ed->n_moved, static_cast<const float*>(ed->extra_items),
              static_cast<const float*>(ed->moved_items), n_old, n_new};
    const int nn = 2 * n_old - 1;

    stage_mark(kMarkStart, s);
    cudaMemsetAsync(w.plan, 0, sizeof(TopoPlan), s);
    cudaMemsetAsync(w.del_flag, 0, sizeof(int) * n_old, s);
    cudaMemsetAsync(w.cut_mark, 0, sizeof(int) * 2 * static_cast<size_t>(n_old), s);
    cudaMemsetAsync(w.cut_extra, 0, sizeof(int) * 2 * static_cast<size_t>(n_old), s);
    cudaMemsetAsync(w.cut_of_slot, 0xff, sizeof(int) * n_old, s);
    const int checks = std::max(std::max(e.n_del, e.n_ins), std::max(e.n_mov, 1));
    k_topo_check<<<blocks_for(checks), kBlock, 0, s>>>(e, w.del_flag, w.shifts, w.plan);
    k_topo_ranges<<<blocks_for(n_old - 1), kBlock, 0, s>>>(static_cast<const Node*>(old_t->nodes),
                                                           w.range, n_old, w.plan);
    k_topo_kept<<<blocks_for(n_old + 1), kBlock, 0, s>>>(old_t->prim_ids, w.del_flag, n_old,
                                                         w.wslot);
    if (e.n_del > 0)
        k_topo_cut_deleted<<<blocks_for(e.n_del), kBlock, 0, s>>>(e, old_t->slot_of, old_t->parent,
                                                                  w.range, S, w.cut_mark);
    if (n_extra > 0) {
        k_topo_cut_extra<Ops><<<blocks_for(n_extra), kBlock, 0, s>>>(
            e, static_cast<const BNode*>(old_t->bnodes), w.range, S, w.cut_mark, w.cut_extra,
            w.ext_key, w.ext_val);
        k_topo_extra_slots<<<blocks_for(nn), kBlock, 0, s>>>(w.cut_mark, w.cut_extra, w.range,
                                                             n_old, w.wslot);
    }
    cudaError_t err = scan_exclusive(w.wslot, w.wslot, n_old, true, w.scan_ws, s);
    // cut_mark -> its exclusive scan (cut list index), total at [2 n_old - 1]
    if (err == cudaSuccess) err = scan_exclusive(w.cut_mark, w.cut_mark, nn, true, w.scan_ws, s);
    if (err != cudaSuccess) return cuda_status(err, "topology scans");
    k_topo_cut_list<<<blocks_for(nn), kBlock, 0, s>>>(w.cut_mark, n_old, w.cut_list);
    const int* ncut_p = w.cut_mark + nn;
    const int cut_grid = 148 * 4;
    k_topo_cuts<<<cut_grid, kBlock, 0, s>>>(w.cut_list, ncut_p, w.range, w.wslot,
                                            old_t->depth_arr, n_old, w.cut_of_slot, w.plan);
    k_topo_weights<<<blocks_for(nn), kBlock, 0, s>>>(static_cast<const Node*>(old_t->nodes),
                                                     w.cut_mark, w.range, w.wslot, w.cut_of_slot,
                                                     n_old, w.wnode, w.plan);
    err = scan_exclusive(w.wnode, w.wnode, nn, true, w.scan_ws, s);
    if (err != cudaSuccess) return cuda_status(err, "topology id scan");
    k_topo_totals<<<1, 1, 0, s>>>(w.plan, w.wslot, n_old, w.cut_mark, w.wnode);
    stage_mark(kMarkPlan, s);
    TopoPlan plan{};
    err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaMemcpyAsync(&plan, w.plan, sizeof(plan), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_status(err, "topology plan");

    if (plan.error)
        return fail(QK_ERR_INVALID, "edit script: %s%s%s", (plan.error & 1) ? "deleted " : "",
                    (plan.error & 2) ? "inserted " : "", (plan.error & 4) ? "moved " : "");
    if (plan.noncontig)
        return fail(QK_ERR_INVALID, "tree has %d subtrees over non-contiguous slots", plan.noncontig);
    if (plan.slots != n_new)
        return fail(QK_ERR_INVALID, "edit leaves %d primitives, new tree has %d", plan.slots, n_new);
    info->cuts = plan.cuts;
    info->old_leaves = plan.old_leaves;
    info->new_leaves = plan.new_leaves;
    info->max_cut = plan.max_new;
    info->spliced = plan.spliced;
    int reason = 0;
    if (plan.root == 1) reason = 1;
    else if (plan.root == 2) reason = 2;
    else if (plan.max_new > kForestMax) reason = 3;
    else if (static_cast<long long>(plan.old_leaves) * 4 > n_new) reason = 4;
    else if (plan.depth_need > kDepthLimit) reason = 5;
    if (reason) {
        info->rebuild = 1;
        info->reason = reason;
        return QK_OK;
    }
    if (plan.ids != n_new - 1)
        return fail(QK_ERR_INVALID, "topology node accounting: %d ids for %d", plan.ids, n_new - 1);

    // ---- emit ----
    cudaMemsetAsync(new_t->parent, 0xff, sizeof(int) * (2 * static_cast<size_t>(n_new) - 1), s);
    cudaMemsetAsync(new_t->flags, 0, sizeof(int) * static_cast<size_t>(n_new - 1), s);
    int* eerr = &w.plan->emit_err;
    Relink R{static_cast<const Node*>(old_t->nodes), w.cut_mark, w.range, w.wslot, w.wnode,
             n_old, n_new};
    k_topo_nodes<<<blocks_for(n_old - 1), kBlock, 0, s>>>(R, *new_t, eerr);
    k_topo_kept_leaves<Ops><<<blocks_for(n_old), kBlock, 0, s>>>(e, *old_t, *new_t, w.del_flag,
                                                                 w.cut_of_slot, w.wslot, w.shifts,
                                                                 eerr);
    const int grid = std::min(plan.cuts, cut_grid);
    if (plan.cuts > 0) {
        k_topo_stage_cuts<Ops><<<grid, kBlock, 0, s>>>(e, *old_t, w.cut_list, ncut_p, w.range,
                                                       w.wslot, w.del_flag, w.shifts, w.wnode,
                                                       w.st_items, w.st_id, w.cen, w.plo, w.phi,
                                                       w.order, w.tasks, w.id_base, eerr);
    }
    if (n_extra > 0) {
        // new primitives grouped by cut (dense cut rank as the key) in index order (stable),
        // so the forest is deterministic
        k_topo_extra_rank<<<blocks_for(n_extra), kBlock, 0, s>>>(w.cut_mark, n_extra, w.ext_key);
        int bits = 1;
        while (bits < 32 && (1ll << bits) < plan.cuts) ++bits;
        err = sort_pairs(w.ext_key, w.ext_val, w.ext_key_s, w.ext_val_s, n_extra, bits, w.sort_ws, s);
        if (err != cudaSuccess) return cuda_status(err, "topology extra sort");
        k_topo_stage_extra<Ops><<<blocks_for(n_extra), kBlock, 0, s>>>(
            e, *old_t, w.ext_key_s, w.ext_val_s, w.cut_list, w.range, w.wslot, w.del_flag,
            w.st_items, w.st_id, w.cen, w.plo, w.phi, w.order, eerr);
    }
    stage_mark(kMarkRelayout, s);
    if (plan.cuts > 0) {
        const int st = sah_forest(w.tasks, plan.cuts, plan.max_new, w.id_base, w.order, w.tmp,
                                  w.cen, w.plo, w.phi, new_t, bins, &w.plan->forest_err, s);
        if (st != QK_OK) return st;
        k_topo_cut_leaves<Ops><<<grid, kBlock, 0, s>>>(w.tasks, ncut_p, w.order, w.st_items,
                                                       w.st_id, *new_t, eerr);
    }
    if (e.n_mov > 0) k_topo_moved<Ops><<<blocks_for(e.n_mov), kBlock, 0, s>>>(e, *new_t, eerr);
    stage_mark(kMarkTopo, s);
    err = cudaGetLastError();
    // every emit write was checked; the bottom-up pass only runs over a fully linked tree
    int emit[3] = {0, 0, 0};  // emit_err, emit_site, forest_err
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(emit, eerr, sizeof(emit), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_status(err, "topology emit");
    if (emit[0] || emit[2])
        return fail(QK_ERR_OVERFLOW,
                    "topology emit reported %d failed checks (sites 0x%x) and %d forest builder "
                    "errors (%d cuts, largest %d primitives)",
                    emit[0], emit[1], emit[2], plan.cuts, plan.max_new);
    const int st = finish_tree_boxes(new_t, w.h, w.new_range, s);
    if (st != QK_OK) return st;
    info->depth = new_t->depth;
    return QK_OK;
}

}  // namespace

size_t update_ws_bytes(int kind, int n_old, int n_new, int n_extra) {
    Carve c;
    carve_topo(c, kind, n_old, n_new, n_extra);
    return c.used;
}

int update_topology(const qk_tree* old_t, qk_tree* new_t, const qk_topo_edit* edit, int cut_size,
                    int bins, qk_topo_info* info, void* ws, cudaStream_t s) {
    *info = qk_topo_info{};
    // default cut size: the touched subtrees together hold about an eighth of the tree
    int S = cut_size;
    if (S <= 0) {
        const long long edits = std::max(1, edit->n_deleted + edit->n_inserted + edit->appended);
        S = static_cast<int>(std::min<long long>(256, std::max<long long>(8, old_t->n / (8 * edits))));
    }
    if (S < 2 || S > kForestMax) return fail(QK_ERR_INVALID, "cut_size must be in [2, 1024]");
    switch (old_t->kind) {
        case kTri: return update_impl<TriOps>(old_t, new_t, edit, S, bins, info, ws, s);
        case kPoint: return update_impl<PointOps>(old_t, new_t, edit, S, bins, info, ws, s);
        case kGauss: return update_impl<GaussOps>(old_t, new_t, edit, S, bins, info, ws, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", old_t->kind);
    }
}

}  // namespace qk
