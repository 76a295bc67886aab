// qk_batch.cu -- many scenes of uneven size built and queried together.
//
// Layout.  One caller-allocated arena holds every scene's tree as an ordinary qk_tree: each
// tree array is one field of the arena in which the scenes follow each other (each scene's
// part rounded up to 256 bytes), so a field can also be scanned as one array -- the 4-wide
// node ids of all scenes come from ONE exclusive scan over the flags field.  A device table
// of BScene entries gives the kernels each scene's tree and input pointers.
//
// Build (LBVH, bit-identical to qk_build's per scene).  Every phase is one launch over all
// scenes; a block takes one 1024-primitive chunk of one scene, so per-scene values (bounds,
// depth) reduce in the block before one atomic per block:
//   reset headers -> centroid bounds -> 30-bit Morton codes (each in its scene's bounds)
//   -> radix sort on the code (4 passes), then a stable sort on the scene index (1 pass):
//      the scenes' slots come out contiguous, each in (code, index) order
//   -> code / local-index gather -> Karras emit -> bottom-up boxes with atomic visit flags
//   -> depths -> [4-wide: even-depth flags, one scan, per-scene rebase, emit]
//
// Queries.  Persistent kernels: a grid of SMs x blocks_per_sm blocks whose warps take
// `chunks_per_fetch` 32-query chunks at a time from a global counter until the chunk table
// (built at plan time, scene by scene) is exhausted.  Each lane runs one query through its
// scene's tree with the same traversal as the single-tree kernels (qk_traverse.cuh); the top
// `short_stack` entries of its stack live in shared memory.  Morton order, when asked for,
// sorts the queries by (scene, 3-axis code inside the scene's root box) in one radix sort.
//
// The loop schedule runs the same work through the single-tree launchers scene by scene.
#include <algorithm>
#include <cstring>
#include <vector>

#include "qk_build.cuh"
#include "qk_internal.cuh"
#include "qk_traverse.cuh"

namespace qk {
namespace {

constexpr int kBuildChunk = 1024;  // primitives per block in the build phases
constexpr int kQueryChunk = 32;    // queries per chunk-table entry (one per lane)
constexpr int kMaxShortStack = 32;

struct BScene {
    qk_tree t;        // the scene's arrays (device pointers) and size
    const float* in;  // the scene's input items
    int prim_off;     // first primitive in the concatenated build arrays
    int pad[3];
};

size_t a256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

constexpr int kFields = 11;

void field_sizes(int kind, int n, size_t f[kFields]) {
    qk_tree_sizes z;
    std::memset(&z, 0, sizeof(z));
    qk_tree_bytes(kind, n, &z);
    const size_t v[kFields] = {z.nodes, z.items, z.prim_ids, z.parent, z.depth_arr, z.bnodes,
                               z.leaves, z.slot_of, z.flags, z.wide, z.wide_id};
    for (int i = 0; i < kFields; ++i) f[i] = a256(v[i]);
}

int scene_bits_for(int scenes) {
    int b = 1;
    while ((1 << b) < scenes) ++b;
    return b;
}

// ---------------------------------------------------------------------------------------
// build kernels (block = one chunk of one scene)
// ---------------------------------------------------------------------------------------
__global__ void k_bt_reset(Header* __restrict__ hdr, int scenes) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= scenes) return;
    Header& h = hdr[s];
    for (int a = 0; a < 3; ++a) {
        h.lo[a] = ord_f(kInf);
        h.hi[a] = ord_f(-kInf);
    }
    h.max_depth = 0;
    h.counter = 0;
    h.overflow = 0;
    h.error = 0;
    h.list_count[0] = 0;
    h.list_count[1] = 0;
}

__device__ __forceinline__ float bwarp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float bwarp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <class Ops>
__global__ __launch_bounds__(kBlock) void k_bt_bounds(const BScene* __restrict__ tab,
                                                      const int2* __restrict__ chunks,
                                                      Header* __restrict__ hdr) {
    const int2 ch = chunks[blockIdx.x];
    const BScene& sc = tab[ch.x];
    const int end = min(sc.t.n, ch.y + kBuildChunk);
    float v[6] = {kInf, kInf, kInf, -kInf, -kInf, -kInf};
    for (int i = ch.y + threadIdx.x; i < end; i += kBlock) {
        const float3 c = Ops::centroid(sc.in + static_cast<size_t>(i) * Ops::kFloats);
        v[0] = fminf(v[0], c.x);
        v[1] = fminf(v[1], c.y);
        v[2] = fminf(v[2], c.z);
        v[3] = fmaxf(v[3], c.x);
        v[4] = fmaxf(v[4], c.y);
        v[5] = fmaxf(v[5], c.z);
    }
    __shared__ float sm[6][kBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int a = 0; a < 3; ++a) {
        v[a] = bwarp_min(v[a]);
        v[a + 3] = bwarp_max(v[a + 3]);
    }
    if (lane == 0)
        for (int a = 0; a < 6; ++a) sm[a][warp] = v[a];
    __syncthreads();
    if (threadIdx.x < 6) {
        const int a = threadIdx.x;
        float r = a < 3 ? kInf : -kInf;
        for (int w = 0; w < kBlock / 32; ++w) r = a < 3 ? fminf(r, sm[a][w]) : fmaxf(r, sm[a][w]);
        if (a < 3) atomicMin(&hdr[ch.x].lo[a], ord_f(r));
        else atomicMax(&hdr[ch.x].hi[a - 3], ord_f(r));
    }
}

template <class Ops>
__global__ __launch_bounds__(kBlock) void k_bt_morton(const BScene* __restrict__ tab,
                                                      const int2* __restrict__ chunks,
                                                      const Header* __restrict__ hdr,
                                                      uint32_t* __restrict__ codes,
                                                      uint32_t* __restrict__ keep,
                                                      uint32_t* __restrict__ idx) {
    const int2 ch = chunks[blockIdx.x];
    const BScene& sc = tab[ch.x];
    const Header& h = hdr[ch.x];
    const float lx = unord_f(h.lo[0]), ly = unord_f(h.lo[1]), lz = unord_f(h.lo[2]);
    const float hx = unord_f(h.hi[0]), hy = unord_f(h.hi[1]), hz = unord_f(h.hi[2]);
    const int end = min(sc.t.n, ch.y + kBuildChunk);
    for (int i = ch.y + threadIdx.x; i < end; i += kBlock) {
        const float3 c = Ops::centroid(sc.in + static_cast<size_t>(i) * Ops::kFloats);
        const uint32_t code = spread10(quant(c.x, lx, hx - lx)) |
                              (spread10(quant(c.y, ly, hy - ly)) << 1) |
                              (spread10(quant(c.z, lz, hz - lz)) << 2);
        const int j = sc.prim_off + i;
        codes[j] = code;
        keep[j] = code;
        idx[j] = static_cast<uint32_t>(j);
    }
}

// scene of every sorted slot's primitive: the last s with prim_off[s] <= index
__global__ __launch_bounds__(kBlock) void k_bt_scene_key(const int* __restrict__ prim_off,
                                                         int scenes,
                                                         const uint32_t* __restrict__ idx,
                                                         int total, uint32_t* __restrict__ key) {
    const int j = blockIdx.x * kBlock + threadIdx.x;
    if (j >= total) return;
    const int g = static_cast<int>(idx[j]);
    int lo = 0, hi = scenes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prim_off + mid) <= g) lo = mid;
        else hi = mid - 1;
    }
    key[j] = static_cast<uint32_t>(lo);
}

__global__ __launch_bounds__(kBlock) void k_bt_gather(const BScene* __restrict__ tab,
                                                      const int2* __restrict__ chunks,
                                                      const uint32_t* __restrict__ keep,
                                                      const uint32_t* __restrict__ idx_f,
                                                      uint32_t* __restrict__ codes_f,
                                                      uint32_t* __restrict__ ids_f) {
    const int2 ch = chunks[blockIdx.x];
    const BScene& sc = tab[ch.x];
    const int end = min(sc.t.n, ch.y + kBuildChunk);
    for (int i = ch.y + threadIdx.x; i < end; i += kBlock) {
        const int j = sc.prim_off + i;
        const uint32_t g = idx_f[j];
        codes_f[j] = keep[g];
        ids_f[j] = g - static_cast<uint32_t>(sc.prim_off);
    }
}

// ranges: one int2 per primitive of the batch (scene s's internal nodes at prim_off(s)); the
// emit writes every internal node's slot range (first, count)
template <class Ops>
__global__ __launch_bounds__(kBlock) void k_bt_emit(const BScene* __restrict__ tab,
                                                    const int2* __restrict__ chunks,
                                                    const uint32_t* __restrict__ codes_f,
                                                    const uint32_t* __restrict__ ids_f,
                                                    int2* __restrict__ ranges) {
    __shared__ __align__(16) float stage[kBlock / 32][emit_stage_floats<Ops>()];
    const int2 ch = chunks[blockIdx.x];
    const BScene& sc = tab[ch.x];
    const qk_tree& t = sc.t;
    const int n = t.n;
    const int end = min(n, ch.y + kBuildChunk);
    const uint32_t* codes = codes_f + sc.prim_off;
    const uint32_t* ids = ids_f + sc.prim_off;
    for (int k0 = ch.y + (threadIdx.x & ~31); k0 < end; k0 += kBlock) {  // whole warps
        emit_leaves_warp<Ops>(sc.in, n, ids, static_cast<Node*>(t.nodes),
                              static_cast<float*>(t.items), t.prim_ids, t.slot_of,
                              static_cast<float4*>(t.leaves), k0, min(32, end - k0),
                              stage[threadIdx.x >> 5]);
        const int k = k0 + (threadIdx.x & 31);
        if (k < end)
            emit_internal(n, codes, ids, static_cast<Node*>(t.nodes), t.parent,
                          static_cast<BNode*>(t.bnodes), t.flags, k, ranges + sc.prim_off);
    }
}

// Bottom-up boxes of every scene: a chunk's block starts the climbs at its kBuildChunk leaf
// slots, and nodes whose range lies inside the chunk meet in shared memory (climb_ranged).
__global__ __launch_bounds__(kBlock) void k_bt_bottom_up(const BScene* __restrict__ tab,
                                                         const int2* __restrict__ chunks,
                                                         const int2* __restrict__ ranges) {
    __shared__ int arrivals[kBuildChunk];
    const int2 ch = chunks[blockIdx.x];
    const BScene& sc = tab[ch.x];
    const qk_tree& t = sc.t;
    const int n = t.n;
    const int end = min(n, ch.y + kBuildChunk);
    for (int i = threadIdx.x; i < kBuildChunk; i += kBlock) arrivals[i] = 0;
    __syncthreads();
    for (int k = ch.y + threadIdx.x; k < end; k += kBlock)
        climb_ranged<kBuildChunk>(static_cast<Node*>(t.nodes), static_cast<BNode*>(t.bnodes),
                                  t.parent, t.flags, n, k, ch.y, arrivals, ranges + sc.prim_off);
}

// depths in two passes, as the single-tree build (anchored_depth in qk_build.cuh): the
// anchors of every chunk's internal nodes, then every other node and each scene's maximum
__global__ __launch_bounds__(kBlock) void k_bt_depth_anchors(const BScene* __restrict__ tab,
                                                             const int2* __restrict__ chunks,
                                                             const int2* __restrict__ ranges_all) {
    const int2 ch = chunks[blockIdx.x];
    const BScene& sc = tab[ch.x];
    const qk_tree& t = sc.t;
    const int n = t.n;
    const int2* ranges = ranges_all + sc.prim_off;
    const int end = min(n - 1, ch.y + kBuildChunk);
    for (int k = ch.y + threadIdx.x; k < end; k += kBlock)
        if (depth_anchor(ranges, k, n)) t.depth_arr[k] = chain_depth(t.parent, k, 2 * n - 1);
}

__global__ __launch_bounds__(kBlock) void k_bt_depth(const BScene* __restrict__ tab,
                                                     const int2* __restrict__ chunks,
                                                     const int2* __restrict__ ranges_all,
                                                     Header* __restrict__ hdr) {
    const int2 ch = chunks[blockIdx.x];
    const BScene& sc = tab[ch.x];
    const qk_tree& t = sc.t;
    const int n = t.n;
    const int m = 2 * n - 1;
    const int2* ranges = ranges_all + sc.prim_off;
    const int end = min(n, ch.y + kBuildChunk);
    int dmax = 0;
    for (int k = ch.y + threadIdx.x; k < end; k += kBlock) {
        if (k < n - 1) {
            int d;
            if (depth_anchor(ranges, k, n)) {
                d = t.depth_arr[k];
            } else {
                d = anchored_depth(t.parent, ranges, t.depth_arr, n, k, m);
                t.depth_arr[k] = d;
            }
            dmax = max(dmax, d);
        }
        const int d = anchored_depth(t.parent, ranges, t.depth_arr, n, n - 1 + k, m);
        t.depth_arr[n - 1 + k] = d;
        dmax = max(dmax, d);
    }
    block_max_to(dmax, &hdr[ch.x].max_depth);
}

__global__ __launch_bounds__(kBlock) void k_bt_wide_flags(const BScene* __restrict__ tab,
                                                          const int2* __restrict__ chunks) {
    const int2 ch = chunks[blockIdx.x];
    const qk_tree& t = tab[ch.x].t;
    const int end = min(t.n - 1, ch.y + kBuildChunk);
    for (int k = ch.y + threadIdx.x; k < end; k += kBlock)
        t.flags[k] = (t.depth_arr[k] & 1) == 0 ? 1 : 0;
}

// the scan over the whole flags field is global; a scene's ids start at its first entry
__global__ void k_bt_wide_base(const BScene* __restrict__ tab, int scenes,
                               Header* __restrict__ hdr) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < scenes) hdr[s].counter = tab[s].t.wide_id[0];
}

__global__ __launch_bounds__(kBlock) void k_bt_wide_fix(const BScene* __restrict__ tab,
                                                        const int2* __restrict__ chunks,
                                                        Header* __restrict__ hdr) {
    const int2 ch = chunks[blockIdx.x];
    const qk_tree& t = tab[ch.x].t;
    const int m = t.n - 1;
    const int base = hdr[ch.x].counter;
    const int end = min(m, ch.y + kBuildChunk);
    for (int k = ch.y + threadIdx.x; k < end; k += kBlock) {
        const int id = t.wide_id[k] - base;
        const int f = t.flags[k];
        t.wide_id[k] = id;
        t.flags[k] = 0;  // the bottom-up pass of the next build expects zeros
        if (k == m - 1) hdr[ch.x].list_count[0] = id + f;
    }
}

__global__ __launch_bounds__(kBlock) void k_bt_wide_emit(const BScene* __restrict__ tab,
                                                         const int2* __restrict__ chunks) {
    const int2 ch = chunks[blockIdx.x];
    const qk_tree& t = tab[ch.x].t;
    const int n = t.n;
    const int end = min(n - 1, ch.y + kBuildChunk);
    const Node* nodes = static_cast<const Node*>(t.nodes);
    WideNode* wide = static_cast<WideNode*>(t.wide);
    for (int k = ch.y + threadIdx.x; k < end; k += kBlock) {
        if ((t.depth_arr[k] & 1) != 0) continue;
        WideNode out;
        wide_node_of(nodes, n, t.wide_id, k, out);
        wide[t.wide_id[k]] = out;
    }
}

// ---------------------------------------------------------------------------------------
// persistent query kernels
// ---------------------------------------------------------------------------------------
struct QArgs {
    const BScene* tab;
    const int2* chunks;
    int nchunks;
    const int* q_off;
    const uint32_t* order;
    int* counter;
    int per_fetch;
    int short_stack;
    unsigned long long* stats;  // [2] counts traversals stopped by a limit
};

template <class Q>
__global__ __launch_bounds__(256) void k_bq(Q q, QArgs a) {
    extern __shared__ int bq_smem[];
    if (!q.enabled()) return;
    using St = typename Q::Stack;
    St st;
    st.sh = a.short_stack;
    st.stride = blockDim.x;
    st.snode = bq_smem + threadIdx.x;
    st.skey = reinterpret_cast<float*>(bq_smem + a.short_stack * blockDim.x) + threadIdx.x;
    Trav tv;
    const int lane = threadIdx.x & 31;
    for (;;) {
        int c0 = 0;
        if (lane == 0) c0 = atomicAdd(a.counter, a.per_fetch);
        c0 = __shfl_sync(0xffffffffu, c0, 0);
        if (c0 >= a.nchunks) break;
        const int c1 = min(c0 + a.per_fetch, a.nchunks);
        for (int c = c0; c < c1; ++c) {
            const int2 ch = __ldg(a.chunks + c);
            const int s = ch.x;
            const int base = __ldg(a.q_off + s);
            const int local = ch.y + lane;
            if (local < __ldg(a.q_off + s + 1) - base) {
                const int pos = base + local;
                const int qi = a.order ? static_cast<int>(__ldg(a.order + pos)) : pos;
                q.run(a.tab[s], s, qi, st, tv);
            }
        }
    }
    flush_stats<false>(true, 0, 0, tv.overflow, a.stats);
}

__device__ __forceinline__ int max_iter_of(const qk_tree& t) { return t.n * 2 + 64; }

// Split schedule of the persistent kernel: a warp takes chunks the same way, then answers
// their queries one after another with the whole warp (qk_traverse.cuh *_split_one).
template <class Q>
__global__ __launch_bounds__(256) void k_bq_split(Q q, QArgs a) {
    if (!q.enabled()) return;
    Trav tv;
    const int lane = threadIdx.x & 31;
    for (;;) {
        int c0 = 0;
        if (lane == 0) c0 = atomicAdd(a.counter, a.per_fetch);
        c0 = __shfl_sync(0xffffffffu, c0, 0);
        if (c0 >= a.nchunks) break;
        const int c1 = min(c0 + a.per_fetch, a.nchunks);
        for (int c = c0; c < c1; ++c) {
            const int2 ch = __ldg(a.chunks + c);
            const int s = ch.x;
            const int base = __ldg(a.q_off + s);
            const int m = min(32, __ldg(a.q_off + s + 1) - base - ch.y);
            for (int j = 0; j < m; ++j) {
                const int pos = base + ch.y + j;
                const int qi = a.order ? static_cast<int>(__ldg(a.order + pos)) : pos;
                q.run_split(a.tab[s], s, qi, lane, tv);
            }
        }
    }
    flush_stats<false>(true, 0, 0, tv.overflow, a.stats);
}

template <class Ops>
struct QClosestSplit {
    const float* pts;
    uint2* out;
    __device__ bool enabled() const { return true; }
    __device__ __forceinline__ void run_split(const BScene& sc, int, int q, int lane, Trav& tv) const {
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        const uint2 r = closest_split_one<Ops>(static_cast<const BNode*>(sc.t.bnodes),
                                               static_cast<const float4*>(sc.t.leaves), p, lane,
                                               max_iter_of(sc.t), tv);
        if (lane == 0) out[q] = r;
    }
};

template <class Ops>
struct QKnnSplit {
    const float* pts;
    uint2* out;
    int k;
    __device__ bool enabled() const { return true; }
    __device__ __forceinline__ void run_split(const BScene& sc, int, int q, int lane, Trav& tv) const {
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        WarpTable tab;
        knn_split_one<Ops>(static_cast<const BNode*>(sc.t.bnodes),
                           static_cast<const float4*>(sc.t.leaves), p, k, lane,
                           max_iter_of(sc.t), tv, tab);
        if (lane < k) out[static_cast<size_t>(q) * k + lane] = warp_table_entry(tab);
    }
};

template <class Ops, bool kFill>
struct QRadiusSplit {
    const float* pts;
    const float* radius;
    int* counts;
    int* lane_counts;  // queries x 32
    const int* offsets;
    unsigned long long* keys;
    const int* total;
    long long cap;
    __device__ bool enabled() const { return !kFill || static_cast<long long>(*total) <= cap; }
    __device__ __forceinline__ void run_split(const BScene& sc, int s, int q, int lane, Trav& tv) const {
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        const float r = __ldg(radius + s);
        const float r2 = r * r;
        int write = 0, end = 0;
        if (kFill) {
            const int mine = lane_counts[static_cast<size_t>(q) * 32 + lane];
            write = offsets[q] + warp_exclusive(mine, lane);
            end = min(write + mine, offsets[q + 1]);
        }
        const int found = radius_split_one<Ops, kFill>(static_cast<const BNode*>(sc.t.bnodes),
                                                       static_cast<const float4*>(sc.t.leaves),
                                                       p, r2, lane, write, end, keys,
                                                       max_iter_of(sc.t), tv);
        if (!kFill) {
            lane_counts[static_cast<size_t>(q) * 32 + lane] = found;
            const int t = __reduce_add_sync(0xffffffffu, found);
            if (lane == 0) counts[q] = t;
        }
    }
};

template <bool kWide>
struct QRay {
    using Stack = SplitStack<kWide ? kStackWide : kStack>;
    const float4* rays;
    unsigned long long* out;
    __device__ bool enabled() const { return true; }
    __device__ __forceinline__ void run(const BScene& sc, int, int q, Stack& st, Trav& tv) const {
        const RayPre R = prepare_ray(__ldg(rays + 2 * q), __ldg(rays + 2 * q + 1));
        int best_id;
        // rays with no parallel axis and vertical rays take traversals compiled for their
        // RayPre::mode; others the general one
        const WideNode* wn = static_cast<const WideNode*>(sc.t.wide);
        const BNode* bn = static_cast<const BNode*>(sc.t.bnodes);
        const float4* lv = static_cast<const float4*>(sc.t.leaves);
        if (kWide) {
            out[q] = R.mode == 0 ? ray_wide_one<false, 0>(wn, lv, R, max_iter_of(sc.t), st, tv, best_id)
                   : R.mode == 3 ? ray_wide_one<false, 3>(wn, lv, R, max_iter_of(sc.t), st, tv, best_id)
                                 : ray_wide_one<false, -1>(wn, lv, R, max_iter_of(sc.t), st, tv, best_id);
        } else {
            const Box rb = root_box(static_cast<const Node*>(sc.t.nodes));
            out[q] = R.mode == 0
                         ? ray_bin_one<Stack, false, 0>(bn, lv, rb, R, max_iter_of(sc.t), st, tv, best_id)
                     : R.mode == 3
                         ? ray_bin_one<Stack, false, 3>(bn, lv, rb, R, max_iter_of(sc.t), st, tv, best_id)
                         : ray_bin_one<Stack, false, -1>(bn, lv, rb, R, max_iter_of(sc.t), st, tv, best_id);
        }
    }
};

template <class Ops, bool kWide>
struct QClosest {
    using Stack = SplitStack<kWide ? kStackWide : kStack>;
    const float* pts;
    uint2* out;
    __device__ bool enabled() const { return true; }
    __device__ __forceinline__ void run(const BScene& sc, int, int q, Stack& st, Trav& tv) const {
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        if (kWide)
            out[q] = closest_wide_one<Ops>(static_cast<const WideNode*>(sc.t.wide),
                                           static_cast<const float4*>(sc.t.leaves), p,
                                           max_iter_of(sc.t), st, tv);
        else
            out[q] = closest_bin_one<Ops>(static_cast<const BNode*>(sc.t.bnodes),
                                          static_cast<const float4*>(sc.t.leaves), p,
                                          max_iter_of(sc.t), st, tv);
    }
};

template <class Ops, int K, bool kWide>
struct QKnn {
    using Stack = SplitStack<kWide ? kStackWide : kStack>;
    const float* pts;
    uint2* out;
    int k;
    __device__ bool enabled() const { return true; }
    __device__ __forceinline__ void run(const BScene& sc, int, int q, Stack& st, Trav& tv) const {
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        KnnTable<K> tab;
        if (kWide)
            knn_wide_one<Ops, K>(static_cast<const WideNode*>(sc.t.wide),
                                 static_cast<const float4*>(sc.t.leaves), p, k, max_iter_of(sc.t),
                                 st, tv, tab);
        else
            knn_bin_one<Ops, K>(static_cast<const BNode*>(sc.t.bnodes),
                                static_cast<const float4*>(sc.t.leaves), p, k, max_iter_of(sc.t),
                                st, tv, tab);
        write_knn<K>(tab, k, out + static_cast<size_t>(q) * k);
    }
};

template <class Ops, bool kFill, bool kWide>
struct QRadius {
    using Stack = SplitStack<kWide ? kStackWide : kStack>;
    const float* pts;
    const float* radius;   // per scene
    int* counts;           // count pass
    const int* offsets;    // fill pass (global CSR)
    unsigned long long* keys;
    const int* total;      // offsets + queries
    long long cap;
    const int* pool_first = nullptr;  // fill pass after a single-pass count: only the queries
                                      // whose keys did not fit the pool
    __device__ bool enabled() const { return !kFill || static_cast<long long>(*total) <= cap; }
    __device__ __forceinline__ void run(const BScene& sc, int s, int q, Stack& st, Trav& tv) const {
        if (kFill && pool_first != nullptr &&
            (offsets[q + 1] - offsets[q] <= kRadiusStash || pool_first[q] != kPoolLost))
            return;
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        const float r = __ldg(radius + s);
        const float r2 = r * r;
        const int write = kFill ? offsets[q] : 0;
        const int end = kFill ? offsets[q + 1] : 0;
        int found;
        if (kWide)
            found = radius_wide_one<Ops, kFill>(static_cast<const WideNode*>(sc.t.wide),
                                                static_cast<const float4*>(sc.t.leaves), p, r2,
                                                write, end, keys, max_iter_of(sc.t), st, tv);
        else
            found = radius_bin_one<Ops, kFill>(static_cast<const BNode*>(sc.t.bnodes),
                                               static_cast<const float4*>(sc.t.leaves),
                                               root_box(static_cast<const Node*>(sc.t.nodes)), p,
                                               r2, write, end, keys, max_iter_of(sc.t), st, tv);
        if (!kFill) counts[q] = found;
    }
};

// Single-pass radius count (QK_TUNE_STASH): every key found goes to the query's stash slots
// and pool chain (PoolSink), so the fill only copies.
template <class Ops, bool kWide>
struct QRadiusPool {
    using Stack = SplitStack<kWide ? kStackWide : kStack>;
    const float* pts;
    const float* radius;   // per scene
    int* counts;
    RadiusPool pool;
    __device__ bool enabled() const { return true; }
    __device__ __forceinline__ void run(const BScene& sc, int s, int q, Stack& st, Trav& tv) const {
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        const float r = __ldg(radius + s);
        const float r2 = r * r;
        pool.first[q] = -1;
        PoolSink sink{pool.stash + static_cast<size_t>(q) * kRadiusStash, pool.keys, pool.next,
                      pool.taken, pool.chunks, pool.first + q, 0, -1};
        int found;
        if (kWide)
            found = radius_wide_visit<Ops, true>(static_cast<const WideNode*>(sc.t.wide),
                                                 static_cast<const float4*>(sc.t.leaves), p, r2,
                                                 sink, max_iter_of(sc.t), st, tv);
        else
            found = radius_bin_visit<Ops, true, Stack, false>(
                static_cast<const BNode*>(sc.t.bnodes), static_cast<const float4*>(sc.t.leaves),
                root_box(static_cast<const Node*>(sc.t.nodes)), p, r2, sink, max_iter_of(sc.t), st,
                tv);
        counts[q] = found;
    }
};

// scene-major Morton keys of the query positions inside each scene's root box; one warp per
// chunk-table entry
__global__ __launch_bounds__(kBlock) void k_bq_keys(const BScene* __restrict__ tab,
                                                    const int2* __restrict__ chunks, int nchunks,
                                                    const int* __restrict__ q_off,
                                                    const float* __restrict__ pos, int stride,
                                                    int scene_bits, int axis_bits,
                                                    uint32_t* __restrict__ keys,
                                                    uint32_t* __restrict__ idx) {
    const int c = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    if (c >= nchunks) return;
    const int2 ch = chunks[c];
    const int s = ch.x;
    const int base = q_off[s];
    const int local = ch.y + (threadIdx.x & 31);
    if (local >= q_off[s + 1] - base) return;
    const int i = base + local;
    const Box rb = root_box(static_cast<const Node*>(tab[s].t.nodes));
    const float* p = pos + static_cast<size_t>(i) * stride;
    const float cells = static_cast<float>((1u << axis_bits) - 1u);
    const float v[3] = {p[0], p[1], p[2]};
    const float lo[3] = {rb.lo.x, rb.lo.y, rb.lo.z};
    const float hi[3] = {rb.hi.x, rb.hi.y, rb.hi.z};
    uint32_t code = 0;
    uint32_t q3[3];
    for (int a = 0; a < 3; ++a) {
        float f = hi[a] > lo[a] ? (v[a] - lo[a]) / (hi[a] - lo[a]) : 0.0f;
        f = fminf(fmaxf(f, 0.0f), 1.0f);  // NaN -> 0
        q3[a] = static_cast<uint32_t>(f * cells + 0.5f);
    }
    for (int b = axis_bits - 1; b >= 0; --b)
        code = (code << 3) | (((q3[2] >> b) & 1u) << 2) | (((q3[1] >> b) & 1u) << 1) | ((q3[0] >> b) & 1u);
    keys[i] = (static_cast<uint32_t>(s) << (3 * axis_bits)) | code;
    idx[i] = static_cast<uint32_t>(i);
}

}  // namespace
}  // namespace qk

// ---------------------------------------------------------------------------------------
// host objects
// ---------------------------------------------------------------------------------------
struct qk_batch {
    int kind = 0;
    int scenes = 0;
    int total = 0;
    int max_n = 0;
    unsigned flags = 0;
    const float* items = nullptr;
    std::vector<qk_tree> trees;
    std::vector<int> prim_off;
    int nchunks = 0;
    qk::BScene* d_tab = nullptr;
    int2* d_chunks = nullptr;
    qk::Header* d_hdr = nullptr;
    int* d_prim_off = nullptr;
    uint32_t* bufs[5] = {};
    void* sort_ws = nullptr;
    int* flags_field = nullptr;
    int* wide_id_field = nullptr;
    long long flag_span = 0;
    void* scan_ws = nullptr;
    void* single_ws = nullptr;
    size_t single_ws_bytes = 0;
    bool built_by_loop = false;
};

struct qk_batch_plan {
    const qk_batch* b = nullptr;
    int op = 0;
    unsigned flags = 0;
    int total = 0;
    int max_q = 0;
    int nchunks = 0;
    std::vector<int> q_off;
    std::vector<float> params;
    int* d_qoff = nullptr;
    int2* d_chunks = nullptr;
    int* d_counter = nullptr;
    float* d_params = nullptr;
    unsigned long long* d_stats = nullptr;
    qk::Header* d_hdr = nullptr;
    uint32_t *keys = nullptr, *idx = nullptr, *keys_s = nullptr, *idx_s = nullptr;
    void* sort_ws = nullptr;
    int* counts = nullptr;
    void* scan_ws = nullptr;
    int* medium = nullptr;
    int* large = nullptr;
    int* lane_counts = nullptr;
    qk::RadiusPool pool{};  // single-pass radius (QK_TUNE_STASH)
    void* loop_ws = nullptr;
    size_t loop_ws_bytes = 0;
    int sms = 148;
    long long radius_total = -1;
    bool radius_overrun = false;
    int32_t* last_offsets = nullptr;
    long long last_cap = -1;
    bool last_loop = false;
};

namespace qk {
namespace {

struct BatchLayout {
    size_t field_base[kFields];
    size_t field_bytes[kFields];
    size_t tab, chunks, hdr, prim_off, bufs, sort_ws, scan_ws, single_ws, single_ws_bytes, total;
    int nchunks;
};

int check_counts(int kind, const int32_t* counts, int scenes, long long* total, int* max_n) {
    if (kind < 0 || kind > 2) return fail(QK_ERR_INVALID, "unknown primitive kind %d", kind);
    if (scenes < 1 || !counts) return fail(QK_ERR_INVALID, "a batch needs at least one scene");
    long long t = 0;
    int mx = 0;
    for (int s = 0; s < scenes; ++s) {
        if (counts[s] < 2)
            return fail(QK_ERR_INVALID, "scene %d has %d primitives (at least 2 required)", s,
                        counts[s]);
        t += counts[s];
        mx = std::max(mx, static_cast<int>(counts[s]));
    }
    if (t > (1ll << 30)) return fail(QK_ERR_INVALID, "batch of %lld primitives is too large", t);
    *total = t;
    *max_n = mx;
    return QK_OK;
}

// uint32 elements between the five build buffers: 64-aligned, so each starts on 256 bytes
size_t buf_stride(long long total) {
    return (static_cast<size_t>(total) + 63) & ~static_cast<size_t>(63);
}

BatchLayout batch_layout(int kind, const int32_t* counts, int scenes, unsigned flags) {
    BatchLayout L;
    std::memset(&L, 0, sizeof(L));
    long long total = 0;
    int max_n = 0;
    int nchunks = 0;
    for (int s = 0; s < scenes; ++s) {
        size_t f[kFields];
        field_sizes(kind, counts[s], f);
        const bool wide = (flags & QK_WIDE) != 0;
        for (int i = 0; i < kFields; ++i) {
            if (!wide && (i == 9 || i == 10)) continue;
            L.field_bytes[i] += f[i];
        }
        total += counts[s];
        max_n = std::max(max_n, static_cast<int>(counts[s]));
        nchunks += (counts[s] + kBuildChunk - 1) / kBuildChunk;
    }
    size_t off = 0;
    for (int i = 0; i < kFields; ++i) {
        L.field_base[i] = off;
        off += a256(L.field_bytes[i]);
    }
    Carve c;
    c.used = off;
    auto take = [&](size_t bytes) {
        c.take<char>(bytes);
        return c.used - bytes;
    };
    const size_t n = static_cast<size_t>(total);
    L.tab = take(sizeof(BScene) * scenes);
    L.chunks = take(sizeof(int2) * nchunks);
    L.hdr = take(sizeof(Header) * scenes);
    L.prim_off = take(sizeof(int) * (scenes + 1));
    L.bufs = take(sizeof(uint32_t) * buf_stride(n) * 5);
    L.sort_ws = take(sort_ws_bytes(static_cast<int>(n)));
    const long long span = static_cast<long long>(L.field_bytes[8] / sizeof(int));
    L.scan_ws = take((flags & QK_WIDE) ? scan_ws_bytes(static_cast<int>(span)) : 0);
    L.single_ws_bytes = std::max(build_ws_bytes(kind, max_n, QK_BUILD_SAH),
                                 scan_ws_bytes(max_n));
    L.single_ws = take(L.single_ws_bytes);
    L.total = c.used;
    L.nchunks = nchunks;
    return L;
}

template <class Ops>
int batch_build_impl(qk_batch* b, cudaStream_t s) {
    const int S = b->scenes, C = b->nchunks, N = b->total;
    uint32_t* codes = b->bufs[0];
    uint32_t* keep = b->bufs[1];
    uint32_t* idx = b->bufs[2];
    uint32_t* codes_s = b->bufs[3];
    uint32_t* idx_s = b->bufs[4];
    k_bt_reset<<<blocks_for(S, 128), 128, 0, s>>>(b->d_hdr, S);
    k_bt_bounds<Ops><<<C, kBlock, 0, s>>>(b->d_tab, b->d_chunks, b->d_hdr);
    k_bt_morton<Ops><<<C, kBlock, 0, s>>>(b->d_tab, b->d_chunks, b->d_hdr, codes, keep, idx);
    cudaError_t e = sort_pairs(codes, idx, codes_s, idx_s, N, 30, b->sort_ws, s);
    if (e != cudaSuccess) return cuda_status(e, "batch code sort");
    // second, stable pass on the scene: sorted (code, index) stays in order inside a scene
    k_bt_scene_key<<<blocks_for(N), kBlock, 0, s>>>(b->d_prim_off, S, idx_s, N, codes);
    e = sort_pairs(codes, idx_s, idx, codes_s, N, scene_bits_for(S), b->sort_ws, s);
    if (e != cudaSuccess) return cuda_status(e, "batch scene sort");
    // idx_f = codes_s; gather codes into codes, local ids into idx_s
    k_bt_gather<<<C, kBlock, 0, s>>>(b->d_tab, b->d_chunks, keep, codes_s, codes, idx_s);
    // keep and idx are free after the gather: their 2N uint32 (adjacent, 256-byte aligned) hold
    // the N int2 slot ranges
    int2* ranges = reinterpret_cast<int2*>(keep);
    k_bt_emit<Ops><<<C, kBlock, 0, s>>>(b->d_tab, b->d_chunks, codes, idx_s, ranges);
    k_bt_bottom_up<<<C, kBlock, 0, s>>>(b->d_tab, b->d_chunks, ranges);
    k_bt_depth_anchors<<<C, kBlock, 0, s>>>(b->d_tab, b->d_chunks, ranges);
    k_bt_depth<<<C, kBlock, 0, s>>>(b->d_tab, b->d_chunks, ranges, b->d_hdr);
    if (b->flags & QK_WIDE) {
        k_bt_wide_flags<<<C, kBlock, 0, s>>>(b->d_tab, b->d_chunks);
        e = scan_exclusive(b->flags_field, b->wide_id_field, static_cast<int>(b->flag_span), false,
                           b->scan_ws, s);
        if (e != cudaSuccess) return cuda_status(e, "batch wide scan");
        k_bt_wide_base<<<blocks_for(S, 128), 128, 0, s>>>(b->d_tab, S, b->d_hdr);
        k_bt_wide_fix<<<C, kBlock, 0, s>>>(b->d_tab, b->d_chunks, b->d_hdr);
        k_bt_wide_emit<<<C, kBlock, 0, s>>>(b->d_tab, b->d_chunks);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "batch build");
}

int batch_build_loop(qk_batch* b, int builder, int bins, cudaStream_t s) {
    for (int i = 0; i < b->scenes; ++i) {
        qk_tree& t = b->trees[i];
        const float* in = b->items + static_cast<size_t>(b->prim_off[i]) * qk_stride_floats(b->kind);
        int st = build_tree(&t, builder, bins, in, b->single_ws, b->single_ws_bytes, s);
        if (st != QK_OK) return st;
        if (b->flags & QK_WIDE) {
            st = wide_build(&t, 1, b->single_ws, b->single_ws_bytes, s);
            if (st != QK_OK) return st;
        }
    }
    return QK_OK;
}

// ---- queries ----
// Key pool of a batched single-pass radius plan, in keys per query on average (shared by all
// queries of the plan).  Larger than the single-tree default: a plan is built once for many
// replays, and a batch's terrain radius averages about 420 keys per query, so a smaller pool
// sends most of its keys back through the second traversal.  The plan grows by about 4.3 KB
// per query (1.3 GB for 300 K queries).
constexpr int kBatchPoolPerQuery = 512;

struct PlanLayout {
    size_t qoff, chunks, counter, params, stats, hdr, keys, idx, keys_s, idx_s, sort_ws, counts,
        scan_ws, medium, large, lane_counts, pool, loop_ws, loop_ws_bytes, total;
    int nchunks;
};

PlanLayout plan_layout(int op, const int32_t* counts, int scenes, unsigned flags) {
    PlanLayout L;
    std::memset(&L, 0, sizeof(L));
    long long total = 0;
    int max_q = 0, nchunks = 0;
    for (int s = 0; s < scenes; ++s) {
        total += counts[s];
        max_q = std::max(max_q, static_cast<int>(counts[s]));
        nchunks += (counts[s] + kQueryChunk - 1) / kQueryChunk;
    }
    const int n = static_cast<int>(total);
    Carve c;
    auto take = [&](size_t bytes) {
        c.take<char>(bytes);
        return c.used - bytes;
    };
    L.qoff = take(sizeof(int) * (scenes + 1));
    L.chunks = take(sizeof(int2) * std::max(nchunks, 1));
    L.counter = take(sizeof(int) * 4);
    L.params = take(sizeof(float) * scenes);
    L.stats = take(sizeof(unsigned long long) * 4);
    L.hdr = take(sizeof(Header));
    if (flags & QK_ORDER_MORTON) {
        L.keys = take(sizeof(uint32_t) * n);
        L.idx = take(sizeof(uint32_t) * n);
        L.keys_s = take(sizeof(uint32_t) * n);
        L.idx_s = take(sizeof(uint32_t) * n);
        L.sort_ws = take(sort_ws_bytes(n));
    }
    if (op == QK_OP_RADIUS) {
        L.counts = take(sizeof(int) * n);
        L.scan_ws = take(scan_ws_bytes(n));
        L.medium = take(sizeof(int) * n);
        L.large = take(sizeof(int) * n);
        L.lane_counts = take(sizeof(int) * static_cast<size_t>(n) * 32);
        if (flags & QK_TUNE_STASH) {
            // the single-pass radius's stash and key pool, carved at the plan creation
            Carve pc;
            carve_pool(pc, n, kBatchPoolPerQuery);
            L.pool = take(pc.used);
        }
    }
    L.loop_ws_bytes = op == QK_OP_RADIUS ? radius_ws_bytes(max_q, flags) : order_ws_bytes(max_q);
    L.loop_ws = take(L.loop_ws_bytes);
    L.total = c.used;
    L.nchunks = nchunks;
    return L;
}

int device_sms() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 148;
    return sms;
}

template <class Q>
int launch_bq(const Q& q, const qk_batch_plan* p, const qk_batch_tune& tune, cudaStream_t s) {
    QArgs a;
    a.tab = p->b->d_tab;
    a.chunks = p->d_chunks;
    a.nchunks = p->nchunks;
    a.q_off = p->d_qoff;
    a.order = (p->flags & QK_ORDER_MORTON) ? p->idx_s : nullptr;
    a.counter = p->d_counter;
    a.per_fetch = tune.chunks_per_fetch;
    a.short_stack = tune.short_stack;
    a.stats = p->d_stats;
    const size_t smem = static_cast<size_t>(tune.short_stack) * tune.block * 8;
    const int grid = p->sms * tune.blocks_per_sm;
    cudaMemsetAsync(p->d_counter, 0, sizeof(int), s);
    k_bq<Q><<<grid, tune.block, smem, s>>>(q, a);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "batched query");
}

template <class Q>
int launch_bq_split(const Q& q, const qk_batch_plan* p, const qk_batch_tune& tune,
                    cudaStream_t s) {
    QArgs a;
    a.tab = p->b->d_tab;
    a.chunks = p->d_chunks;
    a.nchunks = p->nchunks;
    a.q_off = p->d_qoff;
    a.order = (p->flags & QK_ORDER_MORTON) ? p->idx_s : nullptr;
    a.counter = p->d_counter;
    a.per_fetch = tune.chunks_per_fetch;
    a.short_stack = 0;
    a.stats = p->d_stats;
    const int grid = p->sms * tune.blocks_per_sm;
    cudaMemsetAsync(p->d_counter, 0, sizeof(int), s);
    k_bq_split<Q><<<grid, tune.block, 0, s>>>(q, a);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "batched split query");
}

// closest / kNN / radius with one warp per query (binary nodes)
template <class Ops>
int batch_query_split(qk_batch_plan* p, const qk_batch_io& io, const qk_batch_tune& tune,
                      cudaStream_t s) {
    const int N = p->total;
    const float* pts = static_cast<const float*>(io.input);
    switch (p->op) {
        case QK_OP_CLOSEST:
            return launch_bq_split(QClosestSplit<Ops>{pts, static_cast<uint2*>(io.out)}, p, tune, s);
        case QK_OP_KNN:
            return launch_bq_split(QKnnSplit<Ops>{pts, static_cast<uint2*>(io.out), io.k}, p, tune, s);
        case QK_OP_RADIUS: {
            auto* keys = static_cast<unsigned long long*>(io.out);
            QRadiusSplit<Ops, false> qc{pts, p->d_params, p->counts, p->lane_counts, nullptr,
                                        nullptr, nullptr, -1};
            int st = launch_bq_split(qc, p, tune, s);
            if (st != QK_OK) return st;
            const cudaError_t e = scan_exclusive(p->counts, io.offsets, N, true, p->scan_ws, s);
            if (e != cudaSuccess) return cuda_status(e, "batched radius scan");
            QRadiusSplit<Ops, true> qf{pts, p->d_params, nullptr, p->lane_counts, io.offsets, keys,
                                       io.offsets + N, io.capacity};
            st = launch_bq_split(qf, p, tune, s);
            if (st != QK_OK) return st;
            return radius_sort_segments(io.offsets, N, static_cast<uint64_t*>(io.out), p->medium,
                                        p->large, p->d_hdr, io.capacity, s);
        }
        default:
            return fail(QK_ERR_INVALID, "the split schedule serves closest, kNN and radius");
    }
}

template <class Ops, bool kWide>
int batch_query_kind(qk_batch_plan* p, const qk_batch_io& io, const qk_batch_tune& tune,
                     cudaStream_t s) {
    const int N = p->total;
    switch (p->op) {
        case QK_OP_RAY: {
            QRay<kWide> q{static_cast<const float4*>(io.input),
                          static_cast<unsigned long long*>(io.out)};
            return launch_bq(q, p, tune, s);
        }
        case QK_OP_CLOSEST: {
            QClosest<Ops, kWide> q{static_cast<const float*>(io.input), static_cast<uint2*>(io.out)};
            return launch_bq(q, p, tune, s);
        }
        case QK_OP_KNN: {
            const float* pts = static_cast<const float*>(io.input);
            uint2* out = static_cast<uint2*>(io.out);
            if (io.k <= 4) return launch_bq(QKnn<Ops, 4, kWide>{pts, out, io.k}, p, tune, s);
            if (io.k <= 8) return launch_bq(QKnn<Ops, 8, kWide>{pts, out, io.k}, p, tune, s);
            if (io.k <= 16) return launch_bq(QKnn<Ops, 16, kWide>{pts, out, io.k}, p, tune, s);
            return launch_bq(QKnn<Ops, 32, kWide>{pts, out, io.k}, p, tune, s);
        }
        case QK_OP_RADIUS: {
            const float* pts = static_cast<const float*>(io.input);
            auto* keys = static_cast<unsigned long long*>(io.out);
            if (p->flags & QK_TUNE_STASH) {
                // single pass: count + keep every key, scan, copy; traverse again only the
                // queries whose keys did not fit the pool
                cudaMemsetAsync(p->pool.taken, 0, sizeof(int), s);
                QRadiusPool<Ops, kWide> qc{pts, p->d_params, p->counts, p->pool};
                int st = launch_bq(qc, p, tune, s);
                if (st != QK_OK) return st;
                const cudaError_t e = scan_exclusive(p->counts, io.offsets, N, true, p->scan_ws, s);
                if (e != cudaSuccess) return cuda_status(e, "batched radius scan");
                k_radius_gather<<<blocks_for(static_cast<long long>(N) * 32), kBlock, 0, s>>>(
                    p->pool, io.offsets, N, keys, io.capacity);
                QRadius<Ops, true, kWide> qf{pts, p->d_params, nullptr, io.offsets, keys,
                                             io.offsets + N, io.capacity, p->pool.first};
                st = launch_bq(qf, p, tune, s);
                if (st != QK_OK) return st;
                return radius_sort_segments(io.offsets, N, io.out ? static_cast<uint64_t*>(io.out) : nullptr,
                                            p->medium, p->large, p->d_hdr, io.capacity, s);
            }
            QRadius<Ops, false, kWide> qc{pts, p->d_params, p->counts, nullptr, nullptr, nullptr, -1};
            int st = launch_bq(qc, p, tune, s);
            if (st != QK_OK) return st;
            const cudaError_t e = scan_exclusive(p->counts, io.offsets, N, true, p->scan_ws, s);
            if (e != cudaSuccess) return cuda_status(e, "batched radius scan");
            QRadius<Ops, true, kWide> qf{pts, p->d_params, nullptr, io.offsets, keys,
                                         io.offsets + N, io.capacity};
            st = launch_bq(qf, p, tune, s);
            if (st != QK_OK) return st;
            return radius_sort_segments(io.offsets, N, io.out ? static_cast<uint64_t*>(io.out) : nullptr,
                                        p->medium, p->large, p->d_hdr, io.capacity, s);
        }
        default:
            return fail(QK_ERR_INVALID, "unknown batch operation %d", p->op);
    }
}

int batch_query_loop(qk_batch_plan* p, const qk_batch_io& io, cudaStream_t s) {
    const qk_batch* b = p->b;
    // the same layout, order and radius algorithm as the batched schedule
    const unsigned f = p->flags & (QK_ORDER_MORTON | QK_WIDE | QK_TUNE_STASH);
    long long base = 0;
    for (int i = 0; i < b->scenes; ++i) {
        const int count = p->q_off[i + 1] - p->q_off[i];
        if (count == 0) continue;
        const qk_tree* t = &b->trees[i];
        const size_t q0 = static_cast<size_t>(p->q_off[i]);
        int st = QK_OK;
        switch (p->op) {
            case QK_OP_RAY:
                st = ray_query(t, static_cast<const float*>(io.input) + q0 * 8, count,
                               static_cast<uint64_t*>(io.out) + q0, nullptr, f, nullptr, p->loop_ws, s);
                break;
            case QK_OP_CLOSEST:
                st = closest_query(t, static_cast<const float*>(io.input) + q0 * 3, count,
                                   static_cast<uint2*>(io.out) + q0, f, nullptr, p->loop_ws, s);
                break;
            case QK_OP_KNN:
                st = knn_query(t, static_cast<const float*>(io.input) + q0 * 3, count, io.k, io.k,
                               static_cast<uint2*>(io.out) + q0 * io.k, f, nullptr, p->loop_ws, s);
                break;
            case QK_OP_RADIUS: {
                const float* pts = static_cast<const float*>(io.input) + q0 * 3;
                int32_t* off = io.offsets + q0 + i;
                long long tot = 0;
                st = radius_count(t, pts, count, p->params[i], off, &tot, f, nullptr, p->loop_ws, s);
                if (st != QK_OK) return st;
                if (base + tot > io.capacity) {
                    p->radius_overrun = true;
                    return fail(QK_ERR_WORKSPACE, "radius keys (%lld+) exceed the capacity %lld",
                                base + tot, static_cast<long long>(io.capacity));
                }
                st = radius_fill(t, pts, count, p->params[i], off,
                                 static_cast<uint64_t*>(io.out) + base, f, p->loop_ws, s);
                base += tot;
                break;
            }
            default:
                return fail(QK_ERR_INVALID, "unknown batch operation %d", p->op);
        }
        if (st != QK_OK) return st;
    }
    if (p->op == QK_OP_RADIUS) p->radius_total = base;
    return QK_OK;
}

}  // namespace
}  // namespace qk

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
using namespace qk;

extern "C" {

size_t qk_batch_arena_bytes(int kind, const int32_t* counts, int scenes, unsigned flags) {
    long long total = 0;
    int max_n = 0;
    if (check_counts(kind, counts, scenes, &total, &max_n) != QK_OK) return 0;
    return batch_layout(kind, counts, scenes, flags).total;
}

int qk_batch_create(qk_batch** out, int kind, const int32_t* counts, int scenes,
                    const void* items, void* arena, size_t arena_bytes, unsigned flags,
                    void* stream) {
    if (!out) return fail(QK_ERR_INVALID, "out is NULL");
    *out = nullptr;
    long long total = 0;
    int max_n = 0;
    int st = check_counts(kind, counts, scenes, &total, &max_n);
    if (st) return st;
    if (!items || !arena) return fail(QK_ERR_INVALID, "items or arena is NULL");
    if (reinterpret_cast<uintptr_t>(arena) % 256 != 0)
        return fail(QK_ERR_INVALID, "arena must be 256-byte aligned");
    if (flags & ~QK_WIDE) return fail(QK_ERR_INVALID, "unknown batch flags 0x%x", flags);
    const BatchLayout L = batch_layout(kind, counts, scenes, flags);
    if (arena_bytes < L.total)
        return fail(QK_ERR_WORKSPACE, "arena of %zu bytes is smaller than the %zu required",
                    arena_bytes, L.total);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(arena);
    auto* b = new qk_batch;
    b->kind = kind;
    b->scenes = scenes;
    b->total = static_cast<int>(total);
    b->max_n = max_n;
    b->flags = flags;
    b->items = static_cast<const float*>(items);
    b->trees.resize(scenes);
    b->prim_off.resize(scenes + 1);
    b->nchunks = L.nchunks;
    b->d_tab = reinterpret_cast<BScene*>(base + L.tab);
    b->d_chunks = reinterpret_cast<int2*>(base + L.chunks);
    b->d_hdr = reinterpret_cast<Header*>(base + L.hdr);
    b->d_prim_off = reinterpret_cast<int*>(base + L.prim_off);
    for (int i = 0; i < 5; ++i)
        b->bufs[i] = reinterpret_cast<uint32_t*>(base + L.bufs) +
                     static_cast<size_t>(i) * buf_stride(total);
    b->sort_ws = base + L.sort_ws;
    b->scan_ws = base + L.scan_ws;
    b->single_ws = base + L.single_ws;
    b->single_ws_bytes = L.single_ws_bytes;
    b->flags_field = reinterpret_cast<int*>(base + L.field_base[8]);
    b->wide_id_field = (flags & QK_WIDE) ? reinterpret_cast<int*>(base + L.field_base[10]) : nullptr;
    b->flag_span = static_cast<long long>(L.field_bytes[8] / sizeof(int));

    std::vector<BScene> tab(scenes);
    std::vector<int2> chunks;
    chunks.reserve(L.nchunks);
    size_t run[kFields] = {};
    int off = 0;
    const int fl = qk_stride_floats(kind);
    for (int i = 0; i < scenes; ++i) {
        size_t f[kFields];
        field_sizes(kind, counts[i], f);
        void* ptr[kFields];
        for (int k = 0; k < kFields; ++k) {
            const bool absent = !(flags & QK_WIDE) && (k == 9 || k == 10);
            ptr[k] = absent ? nullptr : base + L.field_base[k] + run[k];
            if (!absent) run[k] += f[k];
        }
        qk_tree& t = b->trees[i];
        std::memset(&t, 0, sizeof(t));
        t.kind = kind;
        t.n = counts[i];
        t.nodes = ptr[0];
        t.items = ptr[1];
        t.prim_ids = static_cast<int32_t*>(ptr[2]);
        t.parent = static_cast<int32_t*>(ptr[3]);
        t.depth_arr = static_cast<int32_t*>(ptr[4]);
        t.bnodes = ptr[5];
        t.leaves = ptr[6];
        t.slot_of = static_cast<int32_t*>(ptr[7]);
        t.flags = static_cast<int32_t*>(ptr[8]);
        t.wide = ptr[9];
        t.wide_id = static_cast<int32_t*>(ptr[10]);
        tab[i].t = t;
        tab[i].in = b->items + static_cast<size_t>(off) * fl;
        tab[i].prim_off = off;
        b->prim_off[i] = off;
        for (int c = 0; c < counts[i]; c += kBuildChunk) chunks.push_back(make_int2(i, c));
        off += counts[i];
    }
    b->prim_off[scenes] = off;
    cudaError_t e = cudaMemsetAsync(base + L.field_base[8], 0, L.field_bytes[8], s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_tab, tab.data(), sizeof(BScene) * scenes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_chunks, chunks.data(), sizeof(int2) * chunks.size(),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_prim_off, b->prim_off.data(), sizeof(int) * (scenes + 1),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        delete b;
        return cuda_status(e, "batch table upload");
    }
    *out = b;
    return QK_OK;
}

int qk_batch_build(qk_batch* b, unsigned schedule, void* stream) {
    if (!b) return fail(QK_ERR_INVALID, "batch is NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (schedule == QK_SCHEDULE_LOOP) {
        b->built_by_loop = true;
        return batch_build_loop(b, QK_BUILD_LBVH, 0, s);
    }
    if (schedule != QK_SCHEDULE_BATCHED) return fail(QK_ERR_INVALID, "unknown schedule %u", schedule);
    b->built_by_loop = false;
    switch (b->kind) {
        case kTri: return batch_build_impl<TriOps>(b, s);
        case kPoint: return batch_build_impl<PointOps>(b, s);
        case kGauss: return batch_build_impl<GaussOps>(b, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", b->kind);
    }
}

int qk_batch_build_sah(qk_batch* b, int sah_bins, void* stream) {
    if (!b) return fail(QK_ERR_INVALID, "batch is NULL");
    if (sah_bins < 4 || sah_bins > 64) return fail(QK_ERR_INVALID, "sah_bins must be in [4, 64]");
    b->built_by_loop = true;
    return batch_build_loop(b, QK_BUILD_SAH, sah_bins, static_cast<cudaStream_t>(stream));
}

int qk_batch_sync(qk_batch* b, void* stream) {
    if (!b) return fail(QK_ERR_INVALID, "batch is NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::vector<Header> h(b->scenes);
    cudaError_t e = cudaSuccess;
    // the loop schedule's single-tree calls set depth and wide counts on the host already
    if (!b->built_by_loop)
        e = cudaMemcpyAsync(h.data(), b->d_hdr, sizeof(Header) * b->scenes,
                            cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "batch header readback");
    if (!b->built_by_loop) {
        for (int i = 0; i < b->scenes; ++i) {
            b->trees[i].depth = h[i].max_depth;
            b->trees[i].wide_count = (b->flags & QK_WIDE) ? h[i].list_count[0] : 0;
        }
    }
    for (int i = 0; i < b->scenes; ++i)
        if (b->trees[i].depth >= kStack)
            return fail(QK_ERR_DEPTH, "scene %d: tree depth %d exceeds %d", i, b->trees[i].depth,
                        kStack - 1);
    return QK_OK;
}

int qk_batch_tree(const qk_batch* b, int scene, qk_tree* out) {
    if (!b || !out) return fail(QK_ERR_INVALID, "batch or out is NULL");
    if (scene < 0 || scene >= b->scenes) return fail(QK_ERR_INVALID, "scene %d out of range", scene);
    *out = b->trees[scene];
    return QK_OK;
}

int qk_batch_scenes(const qk_batch* b) { return b ? b->scenes : 0; }

void qk_batch_destroy(qk_batch* b) { delete b; }

size_t qk_batch_plan_bytes(const qk_batch* b, int op, const int32_t* counts, unsigned flags) {
    if (!b || !counts) return 0;
    return plan_layout(op, counts, b->scenes, flags).total;
}

int qk_batch_plan_create(qk_batch_plan** out, const qk_batch* b, int op, const int32_t* counts,
                         const float* params, void* mem, size_t bytes, unsigned flags,
                         void* stream) {
    if (!out) return fail(QK_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!b || !counts || !mem) return fail(QK_ERR_INVALID, "batch, counts or memory is NULL");
    if (op < QK_OP_RAY || op > QK_OP_RADIUS) return fail(QK_ERR_INVALID, "unknown batch operation %d", op);
    if (op == QK_OP_RAY && b->kind != kTri) return fail(QK_ERR_INVALID, "rays need triangle scenes");
    if (op == QK_OP_RADIUS && !params) return fail(QK_ERR_INVALID, "radius queries need per-scene radii");
    if (flags & ~(QK_ORDER_MORTON | QK_WIDE | QK_TUNE_STASH))
        return fail(QK_ERR_INVALID, "unknown plan flags 0x%x", flags);
    if ((flags & QK_TUNE_STASH) && op != QK_OP_RADIUS)
        return fail(QK_ERR_INVALID, "QK_TUNE_STASH applies to radius plans");
    if ((flags & QK_WIDE) && !(b->flags & QK_WIDE))
        return fail(QK_ERR_INVALID, "the batch was created without 4-wide nodes");
    if (reinterpret_cast<uintptr_t>(mem) % 256 != 0)
        return fail(QK_ERR_INVALID, "plan memory must be 256-byte aligned");
    long long total = 0;
    int max_q = 0;
    for (int s = 0; s < b->scenes; ++s) {
        if (counts[s] < 0) return fail(QK_ERR_INVALID, "scene %d: negative query count", s);
        total += counts[s];
        max_q = std::max(max_q, static_cast<int>(counts[s]));
    }
    if (total > (1ll << 30)) return fail(QK_ERR_INVALID, "too many queries (%lld)", total);
    const PlanLayout L = plan_layout(op, counts, b->scenes, flags);
    if (bytes < L.total)
        return fail(QK_ERR_WORKSPACE, "plan memory of %zu bytes is smaller than the %zu required",
                    bytes, L.total);
    char* base = static_cast<char*>(mem);
    auto* p = new qk_batch_plan;
    p->b = b;
    p->op = op;
    p->flags = flags;
    p->total = static_cast<int>(total);
    p->max_q = max_q;
    p->nchunks = L.nchunks;
    p->q_off.resize(b->scenes + 1);
    p->params.assign(b->scenes, 0.0f);
    if (params) p->params.assign(params, params + b->scenes);
    p->d_qoff = reinterpret_cast<int*>(base + L.qoff);
    p->d_chunks = reinterpret_cast<int2*>(base + L.chunks);
    p->d_counter = reinterpret_cast<int*>(base + L.counter);
    p->d_params = reinterpret_cast<float*>(base + L.params);
    p->d_stats = reinterpret_cast<unsigned long long*>(base + L.stats);
    p->d_hdr = reinterpret_cast<Header*>(base + L.hdr);
    if (flags & QK_ORDER_MORTON) {
        p->keys = reinterpret_cast<uint32_t*>(base + L.keys);
        p->idx = reinterpret_cast<uint32_t*>(base + L.idx);
        p->keys_s = reinterpret_cast<uint32_t*>(base + L.keys_s);
        p->idx_s = reinterpret_cast<uint32_t*>(base + L.idx_s);
        p->sort_ws = base + L.sort_ws;
    }
    if (op == QK_OP_RADIUS) {
        p->counts = reinterpret_cast<int*>(base + L.counts);
        p->scan_ws = base + L.scan_ws;
        p->medium = reinterpret_cast<int*>(base + L.medium);
        p->large = reinterpret_cast<int*>(base + L.large);
        p->lane_counts = reinterpret_cast<int*>(base + L.lane_counts);
        if (flags & QK_TUNE_STASH) {
            Carve pc{base + L.pool};
            p->pool = carve_pool(pc, static_cast<int>(total), kBatchPoolPerQuery);
        }
    }
    p->loop_ws = base + L.loop_ws;
    p->loop_ws_bytes = L.loop_ws_bytes;
    p->sms = device_sms();
    std::vector<int2> chunks;
    chunks.reserve(L.nchunks);
    int off = 0;
    for (int s = 0; s < b->scenes; ++s) {
        p->q_off[s] = off;
        for (int c = 0; c < counts[s]; c += kQueryChunk) chunks.push_back(make_int2(s, c));
        off += counts[s];
    }
    p->q_off[b->scenes] = off;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(p->d_qoff, p->q_off.data(), sizeof(int) * (b->scenes + 1),
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !chunks.empty())
        e = cudaMemcpyAsync(p->d_chunks, chunks.data(), sizeof(int2) * chunks.size(),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->d_params, p->params.data(), sizeof(float) * b->scenes,
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->d_stats, 0, sizeof(unsigned long long) * 4, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        delete p;
        return cuda_status(e, "plan upload");
    }
    *out = p;
    return QK_OK;
}

int qk_batch_query(qk_batch_plan* p, const qk_batch_io* io, const qk_batch_tune* tune,
                   unsigned schedule, void* stream) {
    if (!p || !io) return fail(QK_ERR_INVALID, "plan or io is NULL");
    if (p->total > 0 && (!io->input || !io->out)) return fail(QK_ERR_INVALID, "input or out is NULL");
    if (p->op == QK_OP_KNN && (io->k < 1 || io->k > kMaxKnn))
        return fail(QK_ERR_INVALID, "k=%d outside [1, %d]", io->k, kMaxKnn);
    if (p->op == QK_OP_RADIUS && (!io->offsets || io->capacity < 0))
        return fail(QK_ERR_INVALID, "radius queries need offsets and a capacity");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    p->last_offsets = io->offsets;
    p->last_cap = io->capacity;
    p->last_loop = schedule == QK_SCHEDULE_LOOP;
    p->radius_overrun = false;
    p->radius_total = -1;
    if (schedule == QK_SCHEDULE_LOOP) return batch_query_loop(p, *io, s);
    if (schedule != QK_SCHEDULE_BATCHED) return fail(QK_ERR_INVALID, "unknown schedule %u", schedule);
    qk_batch_tune t = {128, 4, 8, 4, 0};
    if (tune) t = *tune;
    if (t.split && (p->op == QK_OP_RAY || (p->flags & QK_WIDE)))
        return fail(QK_ERR_INVALID, "the split schedule serves closest, kNN and radius on binary nodes");
    if ((t.block != 64 && t.block != 128 && t.block != 256) || t.blocks_per_sm < 1 ||
        t.blocks_per_sm > 16 || t.short_stack < 0 || t.short_stack > kMaxShortStack ||
        t.chunks_per_fetch < 1 || t.chunks_per_fetch > 64)
        return fail(QK_ERR_INVALID, "tune {block %d, blocks/SM %d, short stack %d, chunks %d} out of range",
                    t.block, t.blocks_per_sm, t.short_stack, t.chunks_per_fetch);
    if (static_cast<size_t>(t.short_stack) * t.block * 8 > 48 * 1024)
        return fail(QK_ERR_INVALID, "short stack of %d x %d threads exceeds 48 KB", t.short_stack, t.block);
    if (p->total == 0) return QK_OK;
    cudaError_t e0 = cudaMemsetAsync(p->d_stats, 0, sizeof(unsigned long long) * 4, s);
    if (e0 != cudaSuccess) return cuda_status(e0, "batched query stats");
    if (p->flags & QK_ORDER_MORTON) {
        const int sb = scene_bits_for(p->b->scenes);
        const int ab = std::min(10, (32 - sb) / 3);
        const int stride = p->op == QK_OP_RAY ? 8 : 3;
        k_bq_keys<<<blocks_for(p->nchunks, kBlock / 32), kBlock, 0, s>>>(
            p->b->d_tab, p->d_chunks, p->nchunks, p->d_qoff, static_cast<const float*>(io->input),
            stride, sb, ab, p->keys, p->idx);
        const cudaError_t e = sort_pairs(p->keys, p->idx, p->keys_s, p->idx_s, p->total,
                                         sb + 3 * ab, p->sort_ws, s);
        if (e != cudaSuccess) return cuda_status(e, "batched query order");
    }
    const bool wide = (p->flags & QK_WIDE) != 0;
    if (t.split) {
        switch (p->b->kind) {
            case kTri: return batch_query_split<TriOps>(p, *io, t, s);
            case kPoint: return batch_query_split<PointOps>(p, *io, t, s);
            case kGauss: return batch_query_split<GaussOps>(p, *io, t, s);
            default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", p->b->kind);
        }
    }
    switch (p->b->kind) {
        case kTri: return wide ? batch_query_kind<TriOps, true>(p, *io, t, s)
                               : batch_query_kind<TriOps, false>(p, *io, t, s);
        case kPoint: return wide ? batch_query_kind<PointOps, true>(p, *io, t, s)
                                 : batch_query_kind<PointOps, false>(p, *io, t, s);
        case kGauss: return wide ? batch_query_kind<GaussOps, true>(p, *io, t, s)
                                 : batch_query_kind<GaussOps, false>(p, *io, t, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", p->b->kind);
    }
}

int qk_batch_plan_status(qk_batch_plan* p, int64_t* radius_total, int64_t* overflows,
                         void* stream) {
    if (!p) return fail(QK_ERR_INVALID, "plan is NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned long long st[4] = {0, 0, 0, 0};
    int tot = 0;
    cudaError_t e = cudaMemcpyAsync(st, p->d_stats, sizeof(st), cudaMemcpyDeviceToHost, s);
    const bool read_total = p->op == QK_OP_RADIUS && !p->last_loop && p->last_offsets;
    if (e == cudaSuccess && read_total)
        e = cudaMemcpyAsync(&tot, p->last_offsets + p->total, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "plan status readback");
    if (read_total) {
        p->radius_total = tot;
        p->radius_overrun = tot > p->last_cap;
    }
    if (radius_total) *radius_total = p->radius_total;
    if (overflows) *overflows = static_cast<int64_t>(st[2]);
    if (p->radius_overrun)
        return fail(QK_ERR_WORKSPACE, "radius keys (%lld) exceed the capacity %lld",
                    p->radius_total, p->last_cap);
    return QK_OK;
}

void qk_batch_plan_destroy(qk_batch_plan* p) { delete p; }

}  // extern "C"
