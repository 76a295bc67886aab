// qk_query.cu -- stack traversals for first-hit rays and closest / kNN / radius queries.
//
// One thread per ray or query point.  Binary traversal reads one 64-byte node (four 16-byte
// vector loads) that holds both child boxes, so each level costs one dependent fetch; leaf
// children are tested as soon as their box passes, near internal children are followed
// directly and far ones pushed together with their entry bound, which is re-checked against
// the current best when popped (the same test the reference's CPU traversal makes at pop
// time, src/cpu/bvh.cpp:147-152, 230-234).  Pruning keeps the reference's rules exactly --
// the slab test with its 1e-6 margins for rays and "bound <= best" for point queries
// (src/gpu/raycast.cu:100-139, src/gpu/query.cu:74-116) -- which is what makes every result
// independent of tree shape and visit order, and so bit-identical to the CPU reference.
//
// Morton ordering (RayOrder::Morton / QueryOrder::Morton) does not gather and scatter copies
// of the inputs: the sorted permutation is handed to the traversal, thread i works on item
// order[i] and writes its result in place.
#include "qk_internal.cuh"
#include "qk_traverse.cuh"

namespace qk {

namespace {

// Launch with programmatic stream serialization: the kernel's blocks may be scheduled while the
// previous kernel of the stream drains, and the kernel calls cudaGridDependencySynchronize()
// before it reads anything that kernel wrote.  Used only where the previous operation in the
// stream is one of this file's own kernels (the chained passes of an ordering and the
// traversal that reads the order); elsewhere the kernels' wait returns at once.
template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s,
                       Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// canonical nodes of the leaves (leaf of slot s at n-1+s): their boxes are the leaf boxes
inline const Node* leaf_nodes(const qk_tree* t) {
    return static_cast<const Node*>(t->nodes) + (t->n - 1);
}

// ---------------------------------------------------------------------------------------
// Morton keys (src/gpu/morton.h:125-146) for query reordering
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t spread10q(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t quantize10(float v, float lo, float hi) {
    if (!(hi > lo)) return 0;
    float f = (v - lo) / (hi - lo);
    f = fminf(fmaxf(f, 0.0f), 1.0f);
    return static_cast<uint32_t>(f * 1023.0f + 0.5f);
}

// bounds of the 3-float positions at `stride` floats apart (origins of rays or points)
__global__ __launch_bounds__(kBlock) void k_pos_bounds(const float* __restrict__ p, int stride,
                                                      int count, Header* __restrict__ h) {
    float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < count; i += kBlock * gridDim.x) {
        for (int a = 0; a < 3; ++a) {
            const float v = p[static_cast<size_t>(i) * stride + a];
            lo[a] = fminf(lo[a], v);
            hi[a] = fmaxf(hi[a], v);
        }
    }
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    // one atomic per block and bound: the warps' partial bounds meet in shared memory first
    // (thousands of warps hitting six words serialise at the L2)
    __shared__ float part[kBlock / 32][6];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        for (int a = 0; a < 3; ++a) {
            part[warp][a] = lo[a];
            part[warp][3 + a] = hi[a];
        }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int a = threadIdx.x % 3;
        float m = part[0][threadIdx.x];
        for (int w = 1; w < kBlock / 32; ++w)
            m = threadIdx.x < 3 ? fminf(m, part[w][threadIdx.x]) : fmaxf(m, part[w][threadIdx.x]);
        if (threadIdx.x < 3) atomicMin(&h->lo[a], ord_f(m));
        else atomicMax(&h->hi[a], ord_f(m));
    }
}

__global__ void k_bounds_reset(Header* h, int fixed_unit) {
    if (threadIdx.x < 3) {
        h->lo[threadIdx.x] = ord_f(fixed_unit ? -1.0f : kInf);
        h->hi[threadIdx.x] = ord_f(fixed_unit ? 1.0f : -kInf);
    }
    if (threadIdx.x == 0) {
        h->overflow = 0;
        h->list_count[0] = 0;
        h->list_count[1] = 0;
    }
}

__global__ __launch_bounds__(kBlock) void k_pos_keys(const float* __restrict__ p, int stride,
                                                    int offset, int count,
                                                    const Header* __restrict__ h,
                                                    uint32_t* __restrict__ keys,
                                                    uint32_t* __restrict__ idx) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= count) return;
    const float* q = p + static_cast<size_t>(i) * stride + offset;
    const float lx = unord_f(h->lo[0]), ly = unord_f(h->lo[1]), lz = unord_f(h->lo[2]);
    const float hx = unord_f(h->hi[0]), hy = unord_f(h->hi[1]), hz = unord_f(h->hi[2]);
    keys[i] = spread10q(quantize10(q[0], lx, hx)) | (spread10q(quantize10(q[1], ly, hy)) << 1) |
              (spread10q(quantize10(q[2], lz, hz)) << 2);
    idx[i] = static_cast<uint32_t>(i);
}

// ---------------------------------------------------------------------------------------
// Coherent order (QK_ORDER_COHERENT): a counting sort of the records on a Morton key over
// the first `dims` floats of each record (origin xyz and direction xyz of a ray, the
// position of a query point).  The key spans the bounds of an evenly spaced sample of the
// records; axes whose bounds are flat or not finite are left out, and the others get b bits
// each, b the largest with b * axes <= log2(bucket count), interleaved most significant bit
// first.  Rays that start close together and point the same way get neighbouring threads,
// so a warp walks fewer distinct nodes.  The key pass takes each record's rank in its bucket
// with one atomic; the order inside a bucket follows the atomics and may differ between
// runs, and results never depend on it (the traversal keeps the lexicographic minimum).
// ---------------------------------------------------------------------------------------
constexpr int kCohMaxBuckets = 1 << 15;  // one block scans them
constexpr int kCohMinCount = 64;         // smaller batches keep input order
constexpr int kCohSample = 4096;         // evenly spaced records whose bounds set the key
constexpr int kCohThreads = 1024;        // the grid and scan blocks
constexpr int kCohItems = 4;             // records per thread in the key and scatter kernels

// key parameters: q_a = min((v_a - lo_a) * scale_a, 2^bits - 1) for the axes in `live`
struct CohGrid {
    float lo[6];
    float scale[6];  // 2^bits / extent
    uint32_t live;   // bit a set for an axis that takes part
    int bits;        // bits per axis
};

// the first D floats of record i: rays are 8-float records (two 16-byte loads), query
// points 3-float records
template <int D>
__device__ __forceinline__ void coh_load(const float* __restrict__ p, int i, float (&v)[6]) {
    if constexpr (D == 6) {
        const float4* r = reinterpret_cast<const float4*>(p) + 2 * static_cast<size_t>(i);
        const float4 a = __ldg(r), b = __ldg(r + 1);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y;
    } else {
        const float* r = p + 3 * static_cast<size_t>(i);
        v[0] = __ldg(r); v[1] = __ldg(r + 1); v[2] = __ldg(r + 2);
        v[3] = v[4] = v[5] = 0.0f;
    }
}

// One block: bounds of kCohSample records spaced count / kCohSample apart (records outside
// them fall into the edge cells), then the key parameters for `key_bits` bits.
template <int D>
__global__ __launch_bounds__(kCohThreads) void k_coh_grid(const float* __restrict__ p, int count,
                                                         int key_bits, CohGrid* __restrict__ g) {
    __shared__ float part[kCohThreads / 32][12];
    __shared__ float bound[12];
    const int samples = min(count, kCohSample);
    const int step = count / samples;  // samples * step <= count
    float lo[6], hi[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        lo[a] = kInf;
        hi[a] = -kInf;
    }
#pragma unroll 4
    for (int j = threadIdx.x; j < samples; j += kCohThreads) {
        float v[6];
        coh_load<D>(p, j * step, v);
#pragma unroll
        for (int a = 0; a < D; ++a) {
            lo[a] = fminf(lo[a], v[a]);
            hi[a] = fmaxf(hi[a], v[a]);
        }
    }
#pragma unroll
    for (int a = 0; a < D; ++a) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 6; ++a) {
            part[warp][a] = lo[a];
            part[warp][6 + a] = hi[a];
        }
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        const bool is_lo = threadIdx.x < 6;
        float m = part[0][threadIdx.x];
        for (int w = 1; w < kCohThreads / 32; ++w)
            m = is_lo ? fminf(m, part[w][threadIdx.x]) : fmaxf(m, part[w][threadIdx.x]);
        bound[threadIdx.x] = m;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    uint32_t live = 0;
    int axes = 0;
    for (int a = 0; a < D; ++a) {
        const float ext = bound[6 + a] - bound[a];
        if (ext > 0.0f && ext < kInf) {
            live |= 1u << a;
            ++axes;
        }
    }
    const int bits = axes ? min(key_bits / axes, 10) : 0;
    for (int a = 0; a < 6; ++a) {
        const bool on = (live >> a) & 1u;
        g->lo[a] = on ? bound[a] : 0.0f;
        g->scale[a] = on ? static_cast<float>(1 << bits) / (bound[6 + a] - bound[a]) : 0.0f;
    }
    g->live = live;
    g->bits = bits;
}

// key of every record and its rank in its bucket (one atomic per record; the kCohItems
// atomics of a thread are issued before any of their results is stored)
template <int D>
__global__ __launch_bounds__(kBlock) void k_coh_keys(const float* __restrict__ p, int count,
                                                    const CohGrid* __restrict__ g,
                                                    uint32_t* __restrict__ keys,
                                                    uint32_t* __restrict__ ranks,
                                                    uint32_t* __restrict__ hist) {
    cudaGridDependencySynchronize();  // the grid of k_coh_grid
    float lo[6], scale[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        lo[a] = g->lo[a];
        scale[a] = g->scale[a];
    }
    const uint32_t live = g->live;
    const int bits = g->bits;
    const float top = static_cast<float>((1 << bits) - 1);
    const int base = blockIdx.x * (kBlock * kCohItems) + threadIdx.x;
    uint32_t key[kCohItems], rank[kCohItems];
#pragma unroll
    for (int k = 0; k < kCohItems; ++k) {
        const int i = base + k * kBlock;
        key[k] = 0;
        rank[k] = 0;
        if (i < count) {
            float v[6];
            coh_load<D>(p, i, v);
            uint32_t q[6];
#pragma unroll
            for (int a = 0; a < 6; ++a) {
                // fmaxf / fminf also send a NaN coordinate to cell 0
                q[a] = a < D ? static_cast<uint32_t>(
                                   fminf(fmaxf((v[a] - lo[a]) * scale[a], 0.0f), top))
                             : 0u;
            }
            uint32_t kk = 0;
            for (int bit = bits - 1; bit >= 0; --bit) {
#pragma unroll
                for (int a = 0; a < D; ++a) {
                    if ((live >> a) & 1u) kk = (kk << 1) | ((q[a] >> bit) & 1u);
                }
            }
            key[k] = kk;
        }
    }
#pragma unroll
    for (int k = 0; k < kCohItems; ++k) {
        if (base + k * kBlock < count) rank[k] = atomicAdd(&hist[key[k]], 1u);
    }
#pragma unroll
    for (int k = 0; k < kCohItems; ++k) {
        const int i = base + k * kBlock;
        if (i < count) {
            keys[i] = key[k];
            ranks[i] = rank[k];
        }
    }
}

// exclusive scan of the bucket counts by one block (buckets <= kCohMaxBuckets): warp w
// scans buckets [1024 w, 1024 w + 1024) in 32 coalesced steps after the warps' totals
// have been scanned
__global__ __launch_bounds__(kCohThreads) void k_coh_scan(uint32_t* __restrict__ hist,
                                                         int buckets) {
    cudaGridDependencySynchronize();  // the histogram of k_coh_keys
    constexpr int kWarps = kCohThreads / 32;
    constexpr int kSteps = kCohMaxBuckets / kCohThreads;
    __shared__ uint32_t warp_base[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg = warp * (kCohMaxBuckets / kWarps);
    uint32_t v[kSteps];
    uint32_t tot = 0;
#pragma unroll
    for (int j = 0; j < kSteps; ++j) {
        const int idx = seg + j * 32 + lane;
        v[j] = idx < buckets ? hist[idx] : 0u;
        tot += v[j];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (lane == 0) warp_base[warp] = tot;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = warp_base[lane];
        uint32_t inc = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        warp_base[lane] = inc - w;
    }
    __syncthreads();
    uint32_t carry = warp_base[warp];
#pragma unroll
    for (int j = 0; j < kSteps; ++j) {
        uint32_t inc = v[j];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        const int idx = seg + j * 32 + lane;
        if (idx < buckets) hist[idx] = carry + inc - v[j];
        carry += __shfl_sync(0xffffffffu, inc, 31);
    }
}

// each record goes to its bucket's start plus its rank
__global__ __launch_bounds__(kBlock) void k_coh_scatter(const uint32_t* __restrict__ keys,
                                                       const uint32_t* __restrict__ ranks,
                                                       int count,
                                                       const uint32_t* __restrict__ start,
                                                       uint32_t* __restrict__ order) {
    cudaGridDependencySynchronize();  // the bucket starts of k_coh_scan
    const int base = blockIdx.x * (kBlock * kCohItems) + threadIdx.x;
#pragma unroll
    for (int k = 0; k < kCohItems; ++k) {
        const int i = base + k * kBlock;
        if (i < count) order[start[keys[i]] + ranks[i]] = static_cast<uint32_t>(i);
    }
}

// ---------------------------------------------------------------------------------------
// single-tree kernels: one thread per ray / query point, bodies in qk_traverse.cuh
// ---------------------------------------------------------------------------------------
template <bool kStats, int kMinBlocks, int kShort = 0, bool kLeaf4 = false>
__global__ __launch_bounds__(kBlock, kMinBlocks) void k_ray_bin(const BNode* __restrict__ bn,
                                                   const float4* __restrict__ leaves,
                                                   const Node* __restrict__ nodes,
                                                   const float4* __restrict__ rays,
                                                   const uint32_t* __restrict__ order, int count,
                                                   unsigned long long* __restrict__ out,
                                                   int* __restrict__ ids,
                                                   int max_iter, unsigned long long* __restrict__ stats,
                                                   const Node* __restrict__ lnodes = nullptr) {
    cudaGridDependencySynchronize();  // the order, when the ordering kernels launched it early
    const int i = blockIdx.x * kBlock + threadIdx.x;
    const bool active = i < count;
    Trav tv;
    if (active) {
        const int r = order ? static_cast<int>(order[i]) : i;
        const RayPre R = prepare_ray(__ldg(rays + 2 * r), __ldg(rays + 2 * r + 1));
        int best_id;
        if constexpr (kShort > 0) {
            // the top kShort entries of every thread's stack in shared memory
            __shared__ int sn[kShort * kBlock];
            __shared__ float sk[kShort * kBlock];
            SplitStack<kStack> st;
            st.snode = sn + threadIdx.x;
            st.skey = sk + threadIdx.x;
            st.sh = kShort;
            st.stride = kBlock;
            out[r] = ray_bin_one(bn, leaves, root_box(nodes), R, max_iter, st, tv, best_id);
        } else {
            LocalStack<kStack> st;
            // rays with no parallel axis and vertical rays (x and y parallel), tmin / tmax not
            // NaN, run traversals compiled for their mode (RayPre::mode); others the general one
            const Box rb = root_box(nodes);
            if (R.mode == 0)
                out[r] = ray_bin_one<LocalStack<kStack>, kLeaf4, 0>(bn, leaves, rb, R, max_iter,
                                                                    st, tv, best_id, lnodes);
            else if (R.mode == 3)
                out[r] = ray_bin_one<LocalStack<kStack>, kLeaf4, 3>(bn, leaves, rb, R, max_iter,
                                                                    st, tv, best_id, lnodes);
            else
                out[r] = ray_bin_one<LocalStack<kStack>, kLeaf4, -1>(bn, leaves, rb, R, max_iter,
                                                                     st, tv, best_id, lnodes);
        }
        if (ids) ids[r] = best_id;
    }
    flush_stats<kStats>(active, tv.nodes, tv.leaves, tv.overflow, stats);
}

// Persistent variant with dynamic ray fetching (Aila & Laine 2009): a fixed grid of warps
// loops; each iteration every lane makes one traversal step, and lanes whose ray finished
// take the next rays from a global counter (one atomic per warp per refill).  Same per-ray
// algorithm and results as k_ray_bin; it removes the idle lanes that wait for the longest
// ray of their warp.
template <bool kStats, int kMinBlocks>
__global__ __launch_bounds__(kBlock, kMinBlocks) void k_ray_bin_dyn(
    const BNode* __restrict__ bn, const float4* __restrict__ leaves, const Node* __restrict__ nodes,
    const float4* __restrict__ rays, const uint32_t* __restrict__ order, int count,
    unsigned long long* __restrict__ out, int* __restrict__ ids, int* __restrict__ counter,
    int max_iter, unsigned long long* __restrict__ stats) {
    const int lane = threadIdx.x & 31;
    const unsigned lower = (1u << lane) - 1u;
    int ntests = 0, ttests = 0;
    bool overflow = false;
    int r = -1;
    bool done = false;
    RayPre R;
    float best = 0.0f, bound = 0.0f;
    bool any = false;
    int best_id = -1;
    int stack[kStack];
    float stackT[kStack];
    int sp = 0, node = 0, iters = 0;
    const Box rb = root_box(nodes);
    for (int guard = 0; guard < (1 << 30); ++guard) {
        const bool need = r < 0 && !done;
        const unsigned needm = __ballot_sync(0xffffffffu, need);
        if (needm) {
            const int leader = __ffs(needm) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(counter, __popc(needm));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                const int k = base + __popc(needm & lower);
                if (k >= count) {
                    done = true;
                } else {
                    r = order ? static_cast<int>(order[k]) : k;
                    R = prepare_ray(__ldg(rays + 2 * r), __ldg(rays + 2 * r + 1));
                    best = R.tmax;
                    bound = best * kMarginMul + kMarginAdd;
                    any = false;
                    best_id = -1;
                    sp = 0;
                    node = 0;
                    iters = 0;
                    float te;
                    if (ray_box(R, rb.lo, rb.hi, bound, te)) {
                        ++ntests;
                    } else {
                        out[r] = 0ull;
                        if (ids) ids[r] = -1;
                        r = -1;
                    }
                }
            }
        }
        if (__all_sync(0xffffffffu, done)) break;
        if (r < 0) continue;
        // one traversal step of this lane's ray
        bool finished = false;
        if (++iters > max_iter) {
            overflow = true;
            finished = true;
        } else {
            float3 llo, lhi, rlo, rhi;
            int lref, rref;
            load_bnode(bn, node, llo, lhi, rlo, rhi, lref, rref);
            float tl, tr;
            bool hl = ray_box(R, llo, lhi, bound, tl);
            bool hr = ray_box(R, rlo, rhi, bound, tr);
            ntests += static_cast<int>(hl) + static_cast<int>(hr);
            if (hl && lref < 0) {
                ++ttests;
                test_tri(R, leaves, ~lref, best, bound, any, best_id);
                hl = false;
            }
            if (hr && rref < 0) {
                ++ttests;
                test_tri(R, leaves, ~rref, best, bound, any, best_id);
                hr = false;
            }
            if (hl && hr) {
                const bool lnear = tl <= tr;
                if (sp >= kStack) {
                    overflow = true;
                    finished = true;
                } else {
                    stack[sp] = lnear ? rref : lref;
                    stackT[sp] = lnear ? tr : tl;
                    ++sp;
                    node = lnear ? lref : rref;
                }
            } else if (hl) {
                node = lref;
            } else if (hr) {
                node = rref;
            } else {
                const float limit = bound * kMarginMul + kMarginAdd;
                node = -1;
                while (sp > 0) {
                    --sp;
                    if (!(stackT[sp] > limit)) {
                        node = stack[sp];
                        break;
                    }
                }
                if (node < 0) finished = true;
            }
        }
        if (finished) {
            out[r] = any ? ((1ull << 32) | static_cast<unsigned long long>(__float_as_uint(best))) : 0ull;
            if (ids) ids[r] = best_id;
            r = -1;
        }
    }
    flush_stats<kStats>(true, ntests, ttests, overflow, stats);
}

// kRange: the tree's wide nodes are the leaf-size-4 form (a leaf slot holds up to 4 primitives)
template <bool kStats, bool kRange = false>
__global__ __launch_bounds__(kBlock) void k_ray_wide(const WideNode* __restrict__ wn,
                                                    const float4* __restrict__ leaves,
                                                    const float4* __restrict__ rays,
                                                    const uint32_t* __restrict__ order, int count,
                                                    unsigned long long* __restrict__ out,
                                                    int* __restrict__ ids,
                                                    int max_iter, unsigned long long* __restrict__ stats) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    const bool active = i < count;
    Trav tv;
    if (active) {
        const int r = order ? static_cast<int>(order[i]) : i;
        const RayPre R = prepare_ray(__ldg(rays + 2 * r), __ldg(rays + 2 * r + 1));
        LocalStack<kStackWide> st;
        int best_id;
        out[r] = R.mode == 0 ? ray_wide_one<kRange, 0>(wn, leaves, R, max_iter, st, tv, best_id)
               : R.mode == 3 ? ray_wide_one<kRange, 3>(wn, leaves, R, max_iter, st, tv, best_id)
                             : ray_wide_one<kRange, -1>(wn, leaves, R, max_iter, st, tv, best_id);
        if (ids) ids[r] = best_id;
    }
    flush_stats<kStats>(active, tv.nodes, tv.leaves, tv.overflow, stats);
}

// Threads per block of the thread-per-query point-query kernels: a few tens of thousands of
// queries in blocks of 256 would occupy only some of the 148 SMs, and these latency-bound
// traversals run faster spread over all of them; large batches keep 256.
inline int query_block(int count) { return count <= 148 * 512 ? 64 : kBlock; }

// ---------------------------------------------------------------------------------------
// heavy-query tail (QK_TUNE_TAIL, point clouds).  A point near the centre of a spherical shell
// has most of the shell at almost the same distance, so its search ball admits most of the
// tree: a few such queries take most of a step while the GPU is nearly idle.  With the flag,
// the binary closest / kNN kernels stop a query after a step budget and list it; the listed
// queries are then answered by one brute-force scan over all points that every listed query
// shares (point tiles x heavy-query batches), merged per query.  The scan computes the same
// dist2 as the leaf test and keeps the same (dist2, id) order, so results are bit-identical.
// ---------------------------------------------------------------------------------------
constexpr int kTailCap = 1024;           // heavy queries per scan round
constexpr int kTailBatch = 256;          // heavy queries per scan block, one per thread
constexpr int kTailCands = 4096;         // candidates kept per heavy query (tiles x K)
constexpr int kTailBudgetThread = 2048;  // traversal steps of a thread-per-query query
constexpr int kTailBudgetLane = 192;     // traversal steps of each lane of a warp-per-query one

struct TailList {
    int* count = nullptr;      // heavy queries listed
    int* list = nullptr;       // their query indices (capacity: every query)
    uint2* partial = nullptr;  // kTailCap x kTailCands candidates (dist2 bits, id)
};

__device__ __forceinline__ void tail_append(const TailList& tail, int q) {
    const int h = atomicAdd(tail.count, 1);
    tail.list[h] = q;
}

template <class Ops, bool kStats, bool kLeaf4 = false>
__global__ __launch_bounds__(kBlock) void k_closest_bin(const BNode* __restrict__ bn,
                                                       const float4* __restrict__ leaves,
                                                       const float* __restrict__ pts,
                                                       const uint32_t* __restrict__ order,
                                                       int count, uint2* __restrict__ out,
                                                       int max_iter, unsigned long long* __restrict__ stats,
                                                       const Node* __restrict__ lnodes = nullptr,
                                                       TailList tail = TailList{}) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < count;
    Trav tv;
    if (active) {
        const int q = order ? static_cast<int>(order[i]) : i;
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        LocalStack<kStack> st;
        out[q] = closest_bin_one<Ops, LocalStack<kStack>, kLeaf4>(bn, leaves, p, max_iter, st, tv,
                                                                  lnodes);
        if (tail.count && tv.overflow) tail_append(tail, q);
    }
    flush_stats<kStats>(active, tv.nodes, tv.leaves, tv.overflow, stats);
}

template <class Ops, bool kStats, bool kRange = false>
__global__ __launch_bounds__(kBlock) void k_closest_wide(const WideNode* __restrict__ wn,
                                                        const float4* __restrict__ leaves,
                                                        const float* __restrict__ pts,
                                                        const uint32_t* __restrict__ order,
                                                        int count, uint2* __restrict__ out,
                                                        int max_iter, unsigned long long* __restrict__ stats) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < count;
    Trav tv;
    if (active) {
        const int q = order ? static_cast<int>(order[i]) : i;
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        LocalStack<kStackWide> st;
        out[q] = closest_wide_one<Ops, kRange>(wn, leaves, p, max_iter, st, tv);
    }
    flush_stats<kStats>(active, tv.nodes, tv.leaves, tv.overflow, stats);
}

template <class Ops, int K, bool kStats, bool kLeaf4 = false>
__global__ __launch_bounds__(kBlock) void k_knn_bin(const BNode* __restrict__ bn,
                                                   const float4* __restrict__ leaves,
                                                   const float* __restrict__ pts,
                                                   const uint32_t* __restrict__ order, int count,
                                                   int k, int stride, uint2* __restrict__ out,
                                                   int max_iter, unsigned long long* __restrict__ stats,
                                                   const Node* __restrict__ lnodes = nullptr,
                                                   TailList tail = TailList{}) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < count;
    Trav tv;
    if (active) {
        const int q = order ? static_cast<int>(order[i]) : i;
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        LocalStack<kStack> st;
        KnnTable<K> tab;
        knn_bin_one<Ops, K, LocalStack<kStack>, kLeaf4>(bn, leaves, p, k, max_iter, st, tv, tab,
                                                        lnodes);
        write_knn<K>(tab, k, out + static_cast<size_t>(q) * stride);
        if (tail.count && tv.overflow) tail_append(tail, q);
    }
    flush_stats<kStats>(active, tv.nodes, tv.leaves, tv.overflow, stats);
}

template <class Ops, int K, bool kStats, bool kRange = false>
__global__ __launch_bounds__(kBlock) void k_knn_wide(const WideNode* __restrict__ wn,
                                                    const float4* __restrict__ leaves,
                                                    const float* __restrict__ pts,
                                                    const uint32_t* __restrict__ order, int count,
                                                    int k, int stride, uint2* __restrict__ out,
                                                    int max_iter, unsigned long long* __restrict__ stats) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < count;
    Trav tv;
    if (active) {
        const int q = order ? static_cast<int>(order[i]) : i;
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        LocalStack<kStackWide> st;
        KnnTable<K> tab;
        knn_wide_one<Ops, K, kRange>(wn, leaves, p, k, max_iter, st, tv, tab);
        write_knn<K>(tab, k, out + static_cast<size_t>(q) * stride);
    }
    flush_stats<kStats>(active, tv.nodes, tv.leaves, tv.overflow, stats);
}

// radius: count, then fill at the scanned offsets, then sort every segment by (dist2, id)
template <class Ops, bool kFill, bool kStats, bool kLeaf4 = false>
__global__ __launch_bounds__(kBlock) void k_radius_bin(
    const BNode* __restrict__ bn, const float4* __restrict__ leaves, const Node* __restrict__ nodes,
    const float* __restrict__ pts, const uint32_t* __restrict__ order, int count, float r2,
    int* __restrict__ counts, const int* __restrict__ offsets,
    unsigned long long* __restrict__ keys, int max_iter, unsigned long long* __restrict__ stats,
    const Node* __restrict__ lnodes = nullptr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < count;
    Trav tv;
    if (active) {
        const int q = order ? static_cast<int>(order[i]) : i;
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        const int write = kFill ? offsets[q] : 0;
        const int end = kFill ? offsets[q + 1] : 0;  // never write past this query's segment
        LocalStack<kStack> st;
        const int found = radius_bin_one<Ops, kFill, LocalStack<kStack>, kLeaf4>(
            bn, leaves, root_box(nodes), p, r2, write, end, keys, max_iter, st, tv, lnodes);
        if (!kFill) counts[q] = found;
    }
    flush_stats<kStats>(active, tv.nodes, tv.leaves, tv.overflow, stats);
}

// Single-pass radius (QK_TUNE_STASH): the count pass stores every key it finds -- the first
// kRadiusStash of a query in its stash slots, the rest in chained chunks of a shared pool
// (PoolSink, qk_traverse.cuh) -- so the fill pass only copies each query's keys into its CSR
// segment.  A query whose keys did not fit the pool is traversed again by the fill pass.  The
// keys are the same either way, and the segment sort orders them.
template <class Ops, bool kStats, bool kLeaf4 = false>
__global__ __launch_bounds__(kBlock) void k_radius_count_pool(
    const BNode* __restrict__ bn, const float4* __restrict__ leaves, const Node* __restrict__ nodes,
    const float* __restrict__ pts, const uint32_t* __restrict__ order, int count, float r2,
    int* __restrict__ counts, RadiusPool pool, int max_iter,
    unsigned long long* __restrict__ stats, const Node* __restrict__ lnodes = nullptr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < count;
    Trav tv;
    if (active) {
        const int q = order ? static_cast<int>(order[i]) : i;
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        pool.first[q] = -1;
        PoolSink sink{pool.stash + static_cast<size_t>(q) * kRadiusStash, pool.keys, pool.next,
                      pool.taken, pool.chunks, pool.first + q, 0, -1};
        LocalStack<kStack> st;
        counts[q] = radius_bin_visit<Ops, true, LocalStack<kStack>, kLeaf4>(
            bn, leaves, root_box(nodes), p, r2, sink, max_iter, st, tv, lnodes);
    }
    flush_stats<kStats>(active, tv.nodes, tv.leaves, tv.overflow, stats);
}

// the single-pass radius's second traversal: only queries whose keys the pool could not hold
template <class Ops, bool kLeaf4 = false>
__global__ __launch_bounds__(kBlock) void k_radius_fill_lost(
    const BNode* __restrict__ bn, const float4* __restrict__ leaves, const Node* __restrict__ nodes,
    const float* __restrict__ pts, int count, float r2, const int* __restrict__ offsets,
    RadiusPool pool, unsigned long long* __restrict__ keys, int max_iter,
    const Node* __restrict__ lnodes = nullptr) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const int begin = offsets[q], end = offsets[q + 1];
    if (end - begin <= kRadiusStash || pool.first[q] != kPoolLost) return;
    const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
    Trav tv;
    LocalStack<kStack> st;
    radius_bin_one<Ops, true, LocalStack<kStack>, kLeaf4>(bn, leaves, root_box(nodes), p, r2, begin,
                                                          end, keys, max_iter, st, tv, lnodes);
}

template <class Ops, bool kFill, bool kStats, bool kRange = false>
__global__ __launch_bounds__(kBlock) void k_radius_wide(
    const WideNode* __restrict__ wn, const float4* __restrict__ leaves,
    const float* __restrict__ pts, const uint32_t* __restrict__ order, int count, float r2,
    int* __restrict__ counts, const int* __restrict__ offsets,
    unsigned long long* __restrict__ keys, int max_iter, unsigned long long* __restrict__ stats,
    const Node* __restrict__ lnodes = nullptr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < count;
    Trav tv;
    if (active) {
        const int q = order ? static_cast<int>(order[i]) : i;
        const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        const int write = kFill ? offsets[q] : 0;
        const int end = kFill ? offsets[q + 1] : 0;
        LocalStack<kStackWide> st;
        const int found = radius_wide_one<Ops, kFill, kRange>(wn, leaves, p, r2, write, end,
                                                              keys, max_iter, st, tv);
        if (!kFill) counts[q] = found;
    }
    flush_stats<kStats>(active, tv.nodes, tv.leaves, tv.overflow, stats);
}

// ---------------------------------------------------------------------------------------
// split mode (QK_TUNE_SPLIT: one warp per query; QK_TUNE_SPLIT8 / 4: groups of 8 / 4 lanes;
// bodies in qk_traverse.cuh)
// ---------------------------------------------------------------------------------------
// G lanes per query (32: a warp); a group past the last query traces query 0, writes nothing
template <int G>
__device__ __forceinline__ int split_query(int count, const uint32_t* order, bool& valid,
                                           int& lane) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int w = static_cast<int>(t / G);
    lane = static_cast<int>(threadIdx.x & (G - 1));
    valid = w < count;
    return valid ? (order ? static_cast<int>(order[w]) : w) : 0;
}

template <class Ops, bool kStats, int G>
__global__ __launch_bounds__(kBlock) void k_closest_split(const BNode* __restrict__ bn,
                                                         const float4* __restrict__ leaves,
                                                         const float* __restrict__ pts,
                                                         const uint32_t* __restrict__ order,
                                                         int count, uint2* __restrict__ out,
                                                         int max_iter,
                                                         unsigned long long* __restrict__ stats,
                                                         TailList tail = TailList{}) {
    if (static_cast<long long>(blockIdx.x * kBlock + (threadIdx.x & ~31u)) / G >= count)
        return;  // whole warps past the last query
    bool valid;
    int lane;
    const int q = split_query<G>(count, order, valid, lane);
    const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
    Trav tv;
    const uint2 r = closest_split_one<Ops, G>(bn, leaves, p, lane, max_iter, tv, valid);
    if (valid && lane == 0) out[q] = r;
    const bool ovf = group_any<G>(tv.overflow);
    if (tail.count && valid && ovf && lane == 0) tail_append(tail, q);
    // a group past the last query traced query 0: it counts nothing
    flush_stats<kStats>(valid, valid ? tv.nodes : 0, valid ? tv.leaves : 0, valid && tv.overflow, stats);
}

template <class Ops, bool kStats, int G>
__global__ __launch_bounds__(kBlock) void k_knn_split(const BNode* __restrict__ bn,
                                                     const float4* __restrict__ leaves,
                                                     const float* __restrict__ pts,
                                                     const uint32_t* __restrict__ order,
                                                     int count, int k, int stride,
                                                     uint2* __restrict__ out, int max_iter,
                                                     unsigned long long* __restrict__ stats,
                                                     TailList tail = TailList{}) {
    if (static_cast<long long>(blockIdx.x * kBlock + (threadIdx.x & ~31u)) / G >= count)
        return;  // whole warps past the last query
    bool valid;
    int lane;
    const int q = split_query<G>(count, order, valid, lane);
    const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
    Trav tv;
    WarpTable tab;
    knn_split_one<Ops, G>(bn, leaves, p, k, lane, max_iter, tv, tab, valid);
    if (valid && lane < k) out[static_cast<size_t>(q) * stride + lane] = warp_table_entry(tab);
    const bool ovf = group_any<G>(tv.overflow);
    if (tail.count && valid && ovf && lane == 0) tail_append(tail, q);
    // a group past the last query traced query 0: it counts nothing
    flush_stats<kStats>(valid, valid ? tv.nodes : 0, valid ? tv.leaves : 0, valid && tv.overflow, stats);
}

// The tail scan: block (tile, batch) runs heavy query base + batch x kTailBatch + t of the
// current round over the tile's points and keeps the K nearest (dist2, id); the whole block
// reads the same point at a time, so every load is one broadcast per warp.
template <class Ops, int K>
__global__ __launch_bounds__(kTailBatch) void k_tail_scan(const float4* __restrict__ leaves, int n,
                                                          int ntiles, const float* __restrict__ pts,
                                                          TailList tail, int base, int nround) {
    const int hl = blockIdx.y * kTailBatch + threadIdx.x;
    if (hl >= nround) return;  // no barriers in this kernel
    const int ti = blockIdx.x;
    const int begin = static_cast<int>(static_cast<long long>(n) * ti / ntiles);
    const int end = static_cast<int>(static_cast<long long>(n) * (ti + 1) / ntiles);
    const int q = tail.list[base + hl];
    const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
    KnnTable<K> tab;
    tab.init();
    for (int slot = begin; slot < end; ++slot) {
        int id;
        const float d2 = Ops::dist2(p, leaves, slot, id);
        tab.insert(d2, id, K);
    }
    uint2* dst = tail.partial + static_cast<size_t>(hl) * kTailCands + static_cast<size_t>(ti) * K;
#pragma unroll
    for (int j = 0; j < K; ++j) dst[j] = make_uint2(__float_as_uint(tab.d[j]), static_cast<unsigned>(tab.id[j]));
}

// The tail merge: one warp per heavy query of the round; each lane keeps the K best of its
// share of the query's candidates, then k rounds of a warp-wide (dist2, id) minimum pop the k
// nearest.
template <int K>
__global__ __launch_bounds__(kBlock) void k_tail_merge(TailList tail, int ncand, int k, int stride,
                                                       uint2* __restrict__ out, int base,
                                                       int nround) {
    const int hl = (blockIdx.x * kBlock + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (hl >= nround) return;  // whole warps
    const int q = tail.list[base + hl];
    KnnTable<K> tab;
    tab.init();
    const uint2* cand = tail.partial + static_cast<size_t>(hl) * kTailCands;
    for (int c = lane; c < ncand; c += 32) {
        const uint2 v = cand[c];
        if (v.y != 0x7fffffffu) tab.insert(__uint_as_float(v.x), static_cast<int>(v.y), K);
    }
    for (int r = 0; r < k; ++r) {
        float bd = tab.d[0];
        int bid = tab.id[0];
        warp_min_lex(bd, bid);
        if (lane == 0)
            out[static_cast<size_t>(q) * stride + r] =
                bid != 0x7fffffff ? make_uint2(__float_as_uint(bd), static_cast<unsigned>(bid))
                                  : make_uint2(0u, 0xffffffffu);
        if (bid != 0x7fffffff && tab.id[0] == bid) {  // ids are unique: the owner pops its head
#pragma unroll
            for (int j = 0; j + 1 < K; ++j) {
                tab.d[j] = tab.d[j + 1];
                tab.id[j] = tab.id[j + 1];
            }
            tab.d[K - 1] = kInf;
            tab.id[K - 1] = 0x7fffffff;
        }
    }
}

__global__ void k_add_u64(unsigned long long* dst, unsigned long long v) { atomicAdd(dst, v); }

// Answers the listed heavy queries (k = 0: closest; else kNN with K >= k table entries).
// Reads the heavy count back (syncs the stream) and scans in rounds of kTailCap queries.
template <int K>
int tail_resolve(const qk_tree* t, const float* pts, int k, int stride, uint2* out,
                 const TailList& tail, unsigned long long* stats, cudaStream_t s) {
    int heavy = 0;
    cudaError_t e = cudaMemcpyAsync(&heavy, tail.count, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "heavy-query count");
    if (stats && heavy > 0) k_add_u64<<<1, 1, 0, s>>>(stats + 3, static_cast<unsigned long long>(heavy));
    const int n = t->n;
    const int ntiles = max(1, min(kTailCands / K, n));
    const float4* leaves = static_cast<const float4*>(t->leaves);
    for (int base = 0; base < heavy; base += kTailCap) {
        const int nround = min(kTailCap, heavy - base);
        dim3 grid(ntiles, (nround + kTailBatch - 1) / kTailBatch);
        k_tail_scan<PointOps, K><<<grid, kTailBatch, 0, s>>>(leaves, n, ntiles, pts, tail, base,
                                                             nround);
        k_tail_merge<K><<<blocks_for(static_cast<long long>(nround) * 32), kBlock, 0, s>>>(
            tail, ntiles * K, k == 0 ? 1 : k, k == 0 ? 1 : stride, out, base, nround);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "heavy-query tail");
}

// radius, split: the count pass stores every lane's count (lane_counts[q * 32 + lane]) and
// the query's total; the fill pass writes each lane's keys at the query's offset plus the
// counts of the lower lanes.
template <class Ops, bool kFill, bool kStats, int G>
__global__ __launch_bounds__(kBlock) void k_radius_split(
    const BNode* __restrict__ bn, const float4* __restrict__ leaves, const float* __restrict__ pts,
    const uint32_t* __restrict__ order, int count, float r2, int* __restrict__ counts,
    int* __restrict__ lane_counts, const int* __restrict__ offsets,
    unsigned long long* __restrict__ keys, int max_iter, unsigned long long* __restrict__ stats) {
    if (static_cast<long long>(blockIdx.x * kBlock + (threadIdx.x & ~31u)) / G >= count)
        return;  // whole warps past the last query
    bool valid;
    int lane;
    const int q = split_query<G>(count, order, valid, lane);
    const float3 p = f3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
    Trav tv;
    int write = 0, end = 0;
    if (kFill) {
        // lane counts of the query: G per query at q * G
        const int mine = valid ? lane_counts[static_cast<size_t>(q) * G + lane] : 0;
        const int below = warp_exclusive<G>(mine, lane);  // every lane takes part
        write = valid ? offsets[q] + below : 0;
        end = valid ? min(write + mine, offsets[q + 1]) : 0;
    }
    const int found = radius_split_one<Ops, kFill, G>(bn, leaves, p, r2, lane, write, end, keys,
                                                      max_iter, tv, valid);
    if (!kFill) {
        const int total = group_sum<G>(found);
        if (valid) {
            lane_counts[static_cast<size_t>(q) * G + lane] = found;
            if (lane == 0) counts[q] = total;
        }
    }
    // a group past the last query traced query 0: it counts nothing
    flush_stats<kStats>(valid, valid ? tv.nodes : 0, valid ? tv.leaves : 0, valid && tv.overflow, stats);
}

// ---- segment sort of the radius keys ----
constexpr int kWarpSortMax = 1024;   // largest segment sorted by one warp
constexpr int kWarpSortBlock = 128;  // threads per block of the warp sort
// all-ascending bitonic network: comparator (i, i ^ (2^j - 1)) then (i, i ^ stride) for
// shrinking strides, smaller key to the lower index.  Indices >= m are virtual +inf and never
// move, so a segment of any length sorts in place without padding writes.
__device__ __forceinline__ void cswap(unsigned long long* a, int i, int j, int m) {
    if (j < m) {
        const unsigned long long x = a[i], y = a[j];
        if (y < x) {
            a[i] = y;
            a[j] = x;
        }
    }
}

// one warp per segment of up to 32 keys, in registers
// (cap >= 0: nothing is sorted when the keys overran a buffer of cap entries)
__global__ __launch_bounds__(kBlock) void k_seg_sort_warp(const int* __restrict__ offsets, int count,
                                                         unsigned long long* __restrict__ keys,
                                                         int* __restrict__ medium,
                                                         int* __restrict__ large,
                                                         Header* __restrict__ h, long long cap) {
    const int lane = threadIdx.x & 31;
    const int q = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    if (q >= count) return;
    if (cap >= 0 && offsets[count] > cap) return;
    const int b = offsets[q];
    const int m = offsets[q + 1] - b;
    if (m <= 1) return;
    if (m > 32) {
        if (lane == 0) {
            if (m <= kWarpSortMax) medium[atomicAdd(&h->list_count[0], 1)] = q;
            else large[atomicAdd(&h->list_count[1], 1)] = q;
        }
        return;
    }
    unsigned long long v = lane < m ? keys[b + lane] : ~0ull;
    for (int size = 2; size <= 32; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const int partner = (stride == (size >> 1)) ? (lane ^ (size - 1)) : (lane ^ stride);
            const unsigned long long o = __shfl_sync(0xffffffffu, v, partner);
            const bool lower = lane < partner;
            v = lower ? (o < v ? o : v) : (o > v ? o : v);
        }
    }
    if (lane < m) keys[b + lane] = v;
}

// t-th comparator (i, j) of the bitonic stage (size, stride)
__device__ __forceinline__ void bitonic_pair(int t, int size, int stride, int& i, int& j) {
    const int blk = t / stride, off = t % stride;
    if (stride == (size >> 1)) {
        i = blk * size + off;
        j = blk * size + size - 1 - off;
    } else {
        i = blk * 2 * stride + off;
        j = i + stride;
    }
}

// Bitonic sort of 32 E keys held by one warp in registers, striped: key i sits in lane i % 32,
// register i / 32.  The same all-ascending network as cswap's: for each size, the flip
// comparator (i, i ^ (size - 1)), then (i, i ^ stride) for shrinking strides, smaller key to
// the lower index.  Partners 32 or more apart share a lane (register pairs); nearer ones share
// a register (lane shuffles).  The stage loops stay rolled (the unrolled network of 1024 keys
// is far larger than the instruction cache); register indices are constants inside each
// stage body, which a compile-time chain picks by the stage's register distance.

// flip stage of size 64 B: key (r, lane) against (r ^ (2 B - 1), lane ^ 31), the lower key
// having bit B of r clear
template <int E, int B>
__device__ __forceinline__ void bitonic_flip_regs(unsigned long long (&v)[E]) {
#pragma unroll
    for (int r = 0; r < E; ++r) {
        if (r & B) continue;
        const int rp = r ^ (2 * B - 1);
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, v[rp], 31);
        const unsigned long long b = __shfl_xor_sync(0xffffffffu, v[r], 31);
        v[r] = a < v[r] ? a : v[r];
        v[rp] = b > v[rp] ? b : v[rp];
    }
}

// stride 32 S: key (r, lane) against (r ^ S, lane), inside each lane
template <int E, int S>
__device__ __forceinline__ void bitonic_pair_regs(unsigned long long (&v)[E]) {
#pragma unroll
    for (int r = 0; r < E; ++r) {
        if (r & S) continue;
        const unsigned long long x = v[r], y = v[r ^ S];
        v[r] = y < x ? y : x;
        v[r ^ S] = y < x ? x : y;
    }
}

template <int E, int B = 1>
__device__ __forceinline__ void bitonic_flip_at(unsigned long long (&v)[E], int b) {
    if constexpr (B < E) {
        if (b == B) bitonic_flip_regs<E, B>(v);
        else bitonic_flip_at<E, 2 * B>(v, b);
    }
}

template <int E, int S = 1>
__device__ __forceinline__ void bitonic_pair_at(unsigned long long (&v)[E], int s) {
    if constexpr (S < E) {
        if (s == S) bitonic_pair_regs<E, S>(v);
        else bitonic_pair_at<E, 2 * S>(v, s);
    }
}

template <int E>
__device__ __forceinline__ void warp_bitonic(unsigned long long (&v)[E], int lane) {
#pragma unroll 1
    for (int size = 2; size <= 32 * E; size <<= 1) {
        int stride = size >> 1;
        if (size > 32) {
            bitonic_flip_at<E>(v, size / 64);
#pragma unroll 1
            for (stride = size >> 2; stride >= 32; stride >>= 1) bitonic_pair_at<E>(v, stride / 32);
        }
        // strides below 32: lane ^ (size - 1) for the flip of a size up to 32, else lane ^ stride
#pragma unroll 1
        for (; stride > 0; stride >>= 1) {
            const int lx = stride == (size >> 1) ? size - 1 : stride;
            const bool lower = (lane & stride) == 0;
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const unsigned long long o = __shfl_xor_sync(0xffffffffu, v[r], lx);
                v[r] = lower ? (o < v[r] ? o : v[r]) : (o > v[r] ? o : v[r]);
            }
        }
    }
}

// one segment of m (<= 32 E) keys at keys[b..b+m): coalesced striped loads, padded with the
// largest 64-bit value (which sorts after, or ties with, every real key), sorted in registers
template <int E>
__device__ __forceinline__ void warp_sort_segment(unsigned long long* __restrict__ keys, int b,
                                                  int m, int lane) {
    unsigned long long v[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const int i = r * 32 + lane;
        v[r] = i < m ? keys[b + i] : ~0ull;
    }
    warp_bitonic<E>(v, lane);
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const int i = r * 32 + lane;
        if (i < m) keys[b + i] = v[r];
    }
}

// one warp per listed segment of 33..kWarpSortMax keys, sorted in registers (the smallest
// power-of-two network that holds the segment)
__global__ __launch_bounds__(kWarpSortBlock) void k_seg_sort_warp_reg(
    const int* __restrict__ offsets, unsigned long long* __restrict__ keys,
    const int* __restrict__ list, const Header* __restrict__ h) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int n_list = h->list_count[0];
    const int warps = gridDim.x * (kWarpSortBlock / 32);
    for (int e = blockIdx.x * (kWarpSortBlock / 32) + w; e < n_list; e += warps) {
        const int q = list[e];
        const int b = offsets[q];
        const int m = min(offsets[q + 1] - b, kWarpSortMax);
        if (m <= 64) warp_sort_segment<2>(keys, b, m, lane);
        else if (m <= 128) warp_sort_segment<4>(keys, b, m, lane);
        else if (m <= 256) warp_sort_segment<8>(keys, b, m, lane);
        else if (m <= 512) warp_sort_segment<16>(keys, b, m, lane);
        else warp_sort_segment<32>(keys, b, m, lane);
    }
}

// one block per listed segment of more than kWarpSortMax keys: in shared memory up to 4096,
// in place in global memory beyond
__global__ __launch_bounds__(kBlock) void k_seg_sort_block(const int* __restrict__ offsets,
                                                          unsigned long long* __restrict__ keys,
                                                          const int* __restrict__ list,
                                                          const Header* __restrict__ h) {
    __shared__ unsigned long long sm[4096];
    const int n_list = h->list_count[1];
    for (int e = blockIdx.x; e < n_list; e += gridDim.x) {
        const int q = list[e];
        const int b = offsets[q];
        const int m = offsets[q + 1] - b;
        const bool shared = m <= 4096;
        unsigned long long* a = shared ? sm : keys + b;
        if (shared) {
            for (int t = threadIdx.x; t < m; t += kBlock) sm[t] = keys[b + t];
        }
        __syncthreads();
        int pow2 = 1;
        while (pow2 < m) pow2 <<= 1;
        for (int size = 2; size <= pow2; size <<= 1) {
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int t = threadIdx.x; t < pow2 / 2; t += kBlock) {
                    int i, j;
                    bitonic_pair(t, size, stride, i, j);
                    if (i < m) cswap(a, i, j, m);
                }
                __syncthreads();
            }
        }
        if (shared) {
            for (int t = threadIdx.x; t < m; t += kBlock) keys[b + t] = sm[t];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
struct OrderBufs {
    Header* h = nullptr;
    uint32_t* keys = nullptr;
    uint32_t* idx = nullptr;
    uint32_t* keys_s = nullptr;
    uint32_t* idx_s = nullptr;
    void* sort_ws = nullptr;
};

OrderBufs carve_order(Carve& c, int count) {
    OrderBufs o;
    o.h = c.take<Header>(1);
    o.keys = c.take<uint32_t>(count);
    o.idx = c.take<uint32_t>(count);
    o.keys_s = c.take<uint32_t>(count);
    o.idx_s = c.take<uint32_t>(count);
    o.sort_ws = c.take<char>(sort_ws_bytes(count));
    return o;
}

// Morton order of positions (stride floats apart, `offset` floats into each record);
// returns the permutation or nullptr for input order.
// Coherent order of the records (rays: 6 floats of origin and direction; points: 3) by the
// counting sort above.  The buffers of the Morton sort hold it: keys in o.keys, ranks in
// o.idx, the bucket counts and the key parameters in o.keys_s (at most count / 4 buckets,
// so they and the 14 parameter words fit in its count words), the order in o.idx_s.
const uint32_t* make_coherent_order(const float* pos, int stride, int count, OrderBufs& o,
                                    cudaStream_t s, int* status) {
    if (count < kCohMinCount || (stride != 8 && stride != 3)) return nullptr;
    int key_bits = 4;
    while ((2 << key_bits) <= kCohMaxBuckets && (2 << key_bits) <= count / 4) ++key_bits;
    const int buckets = 1 << key_bits;
    uint32_t* hist = o.keys_s;
    CohGrid* grid = reinterpret_cast<CohGrid*>(o.keys_s + buckets);
    cudaMemsetAsync(hist, 0, sizeof(uint32_t) * static_cast<size_t>(buckets), s);
    const int g = blocks_for(count, kBlock * kCohItems);
    if (stride == 8) {
        k_coh_grid<6><<<1, kCohThreads, 0, s>>>(pos, count, key_bits, grid);
        launch_pdl(k_coh_keys<6>, dim3(g), dim3(kBlock), s, pos, count, grid, o.keys, o.idx, hist);
    } else {
        k_coh_grid<3><<<1, kCohThreads, 0, s>>>(pos, count, key_bits, grid);
        launch_pdl(k_coh_keys<3>, dim3(g), dim3(kBlock), s, pos, count, grid, o.keys, o.idx, hist);
    }
    launch_pdl(k_coh_scan, dim3(1), dim3(kCohThreads), s, hist, buckets);
    launch_pdl(k_coh_scatter, dim3(g), dim3(kBlock), s, o.keys, o.idx, count, hist, o.idx_s);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) *status = cuda_status(e, "coherent order");
    return o.idx_s;
}

const uint32_t* make_order(const float* pos, int stride, int offset, int count, unsigned flags,
                           OrderBufs& o, cudaStream_t s, int* status) {
    *status = QK_OK;
    if (flags & QK_ORDER_COHERENT) return make_coherent_order(pos, stride, count, o, s, status);
    if (!(flags & (QK_ORDER_MORTON | QK_ORDER_DIRECTION))) return nullptr;
    const bool dir = (flags & QK_ORDER_DIRECTION) != 0;
    k_bounds_reset<<<1, 32, 0, s>>>(o.h, dir ? 1 : 0);
    if (!dir) {
        const int grid = min(blocks_for(count), 148 * 4);
        k_pos_bounds<<<grid, kBlock, 0, s>>>(pos + offset, stride, count, o.h);
    }
    k_pos_keys<<<blocks_for(count), kBlock, 0, s>>>(pos, stride, offset, count, o.h, o.keys, o.idx);
    const cudaError_t e = sort_pairs(o.keys, o.idx, o.keys_s, o.idx_s, count, 30, o.sort_ws, s);
    if (e != cudaSuccess) *status = cuda_status(e, "order sort");
    return o.idx_s;
}

// lanes per query of the split schedules: QK_TUNE_SPLIT a warp, QK_TUNE_SPLIT8 / 4 groups of
// 8 / 4 lanes; 0 for one thread per query
constexpr unsigned kSplitFlags = QK_TUNE_SPLIT | QK_TUNE_SPLIT8 | QK_TUNE_SPLIT4;
inline int split_lanes(unsigned flags) {
    return (flags & QK_TUNE_SPLIT) ? 32 : (flags & QK_TUNE_SPLIT8) ? 8 : (flags & QK_TUNE_SPLIT4) ? 4 : 0;
}

template <class Ops, bool kStats>
void launch_closest_split(int lanes, const BNode* bn, const float4* leaves, const float* pts,
                          const uint32_t* order, int count, uint2* out, int max_iter,
                          unsigned long long* stats, const TailList& tail, cudaStream_t s) {
    const int g = blocks_for(static_cast<long long>(count) * lanes);
    if (lanes == 4)
        k_closest_split<Ops, kStats, 4><<<g, kBlock, 0, s>>>(bn, leaves, pts, order, count, out, max_iter, stats, tail);
    else if (lanes == 8)
        k_closest_split<Ops, kStats, 8><<<g, kBlock, 0, s>>>(bn, leaves, pts, order, count, out, max_iter, stats, tail);
    else
        k_closest_split<Ops, kStats, 32><<<g, kBlock, 0, s>>>(bn, leaves, pts, order, count, out, max_iter, stats, tail);
}

// kNN keeps its table one entry per lane: at least k lanes (the next group size up)
inline int knn_lanes(int requested, int k) {
    const int need = k <= 4 ? 4 : (k <= 8 ? 8 : 32);
    return requested > need ? requested : need;
}

template <class Ops, bool kStats>
void launch_knn_split(int lanes, const BNode* bn, const float4* leaves, const float* pts,
                      const uint32_t* order, int count, int k, int stride, uint2* out,
                      int max_iter, unsigned long long* stats, const TailList& tail,
                      cudaStream_t s) {
    const int g = blocks_for(static_cast<long long>(count) * lanes);
    if (lanes == 4)
        k_knn_split<Ops, kStats, 4><<<g, kBlock, 0, s>>>(bn, leaves, pts, order, count, k, stride, out, max_iter, stats, tail);
    else if (lanes == 8)
        k_knn_split<Ops, kStats, 8><<<g, kBlock, 0, s>>>(bn, leaves, pts, order, count, k, stride, out, max_iter, stats, tail);
    else
        k_knn_split<Ops, kStats, 32><<<g, kBlock, 0, s>>>(bn, leaves, pts, order, count, k, stride, out, max_iter, stats, tail);
}

template <class Ops>
int closest_impl(const qk_tree* t, const float* pts, int count, uint2* out, unsigned flags,
                 unsigned long long* stats, const uint32_t* order, cudaStream_t s,
                 const TailList& tail = TailList{}) {
    const float4* leaves = static_cast<const float4*>(t->leaves);
    const int qb = query_block(count);
    const int g = blocks_for(count, qb);
    const bool wide = (flags & QK_WIDE) != 0;
    const bool st = stats != nullptr;
    if (tail.count) {
        // budgeted traversal (binary nodes, thread or warp per query), then the shared scan
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        cudaMemsetAsync(tail.count, 0, sizeof(int), s);
        if (flags & kSplitFlags)
            launch_closest_split<Ops, false>(split_lanes(flags), bn, leaves, pts, order, count, out,
                                             kTailBudgetLane, nullptr, tail, s);
        else
            k_closest_bin<Ops, false><<<g, qb, 0, s>>>(bn, leaves, pts, order, count, out,
                                                           kTailBudgetThread, nullptr, nullptr, tail);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_status(e, "closest (tail)");
        return tail_resolve<1>(t, pts, 0, 1, out, tail, stats, s);
    }
    if (wide) {
        const WideNode* wn = static_cast<const WideNode*>(t->wide);
        if (t->wide_leaf == 4) {
            if (st) k_closest_wide<Ops, true, true><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, out, t->n * 2 + 64, stats);
            else k_closest_wide<Ops, false, true><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, out, t->n * 2 + 64, stats);
        } else {
            if (st) k_closest_wide<Ops, true><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, out, t->n * 2 + 64, stats);
            else k_closest_wide<Ops, false><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, out, t->n * 2 + 64, stats);
        }
    } else if (flags & kSplitFlags) {
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        if (st) launch_closest_split<Ops, true>(split_lanes(flags), bn, leaves, pts, order, count, out, t->n * 2 + 64, stats, TailList{}, s);
        else launch_closest_split<Ops, false>(split_lanes(flags), bn, leaves, pts, order, count, out, t->n * 2 + 64, stats, TailList{}, s);
    } else if (flags & QK_TUNE_LEAF4) {
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        if (st) k_closest_bin<Ops, true, true><<<g, qb, 0, s>>>(bn, leaves, pts, order, count, out, t->n * 2 + 64, stats, leaf_nodes(t));
        else k_closest_bin<Ops, false, true><<<g, qb, 0, s>>>(bn, leaves, pts, order, count, out, t->n * 2 + 64, stats, leaf_nodes(t));
    } else {
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        if (st) k_closest_bin<Ops, true><<<g, qb, 0, s>>>(bn, leaves, pts, order, count, out, t->n * 2 + 64, stats);
        else k_closest_bin<Ops, false><<<g, qb, 0, s>>>(bn, leaves, pts, order, count, out, t->n * 2 + 64, stats);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "closest");
}

template <class Ops, int K>
void launch_knn(const qk_tree* t, const float* pts, int count, int k, int stride, uint2* out,
                bool wide, int split, bool leaf4, unsigned long long* stats,
                const uint32_t* order, cudaStream_t s) {
    const float4* leaves = static_cast<const float4*>(t->leaves);
    const int qb = query_block(count);
    const int g = blocks_for(count, qb);
    if (split && !wide) {
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        const int lanes = knn_lanes(split, k);
        if (stats) launch_knn_split<Ops, true>(lanes, bn, leaves, pts, order, count, k, stride, out, t->n * 2 + 64, stats, TailList{}, s);
        else launch_knn_split<Ops, false>(lanes, bn, leaves, pts, order, count, k, stride, out, t->n * 2 + 64, stats, TailList{}, s);
    } else if (wide) {
        const WideNode* wn = static_cast<const WideNode*>(t->wide);
        if (t->wide_leaf == 4) {
            if (stats) k_knn_wide<Ops, K, true, true><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, k, stride, out, t->n * 2 + 64, stats);
            else k_knn_wide<Ops, K, false, true><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, k, stride, out, t->n * 2 + 64, stats);
        } else {
            if (stats) k_knn_wide<Ops, K, true><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, k, stride, out, t->n * 2 + 64, stats);
            else k_knn_wide<Ops, K, false><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, k, stride, out, t->n * 2 + 64, stats);
        }
    } else if (leaf4) {
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        if (stats) k_knn_bin<Ops, K, true, true><<<g, qb, 0, s>>>(bn, leaves, pts, order, count, k, stride, out, t->n * 2 + 64, stats, leaf_nodes(t));
        else k_knn_bin<Ops, K, false, true><<<g, qb, 0, s>>>(bn, leaves, pts, order, count, k, stride, out, t->n * 2 + 64, stats, leaf_nodes(t));
    } else {
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        if (stats) k_knn_bin<Ops, K, true><<<g, qb, 0, s>>>(bn, leaves, pts, order, count, k, stride, out, t->n * 2 + 64, stats);
        else k_knn_bin<Ops, K, false><<<g, qb, 0, s>>>(bn, leaves, pts, order, count, k, stride, out, t->n * 2 + 64, stats);
    }
}

template <class Ops, int K>
int knn_tail(const qk_tree* t, const float* pts, int count, int k, int stride, uint2* out,
             int split, const uint32_t* order, const TailList& tail,
             unsigned long long* stats, cudaStream_t s) {
    const BNode* bn = static_cast<const BNode*>(t->bnodes);
    const float4* leaves = static_cast<const float4*>(t->leaves);
    cudaMemsetAsync(tail.count, 0, sizeof(int), s);
    if (split)
        launch_knn_split<Ops, false>(knn_lanes(split, k), bn, leaves, pts, order, count, k,
                                     stride, out, kTailBudgetLane, nullptr, tail, s);
    else
        k_knn_bin<Ops, K, false><<<blocks_for(count, query_block(count)), query_block(count), 0, s>>>(
            bn, leaves, pts, order, count, k, stride, out, kTailBudgetThread, nullptr, nullptr, tail);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "knn (tail)");
    return tail_resolve<K>(t, pts, k, stride, out, tail, stats, s);
}

template <class Ops>
int knn_impl(const qk_tree* t, const float* pts, int count, int k, int stride, uint2* out,
             unsigned flags, unsigned long long* stats, const uint32_t* order, cudaStream_t s,
             const TailList& tail = TailList{}) {
    const bool wide = (flags & QK_WIDE) != 0;
    const int split = split_lanes(flags);  // 0: one thread per query
    const bool leaf4 = (flags & QK_TUNE_LEAF4) != 0;
    if (tail.count) {
        if (k <= 4) return knn_tail<Ops, 4>(t, pts, count, k, stride, out, split, order, tail, stats, s);
        if (k <= 8) return knn_tail<Ops, 8>(t, pts, count, k, stride, out, split, order, tail, stats, s);
        if (k <= 16) return knn_tail<Ops, 16>(t, pts, count, k, stride, out, split, order, tail, stats, s);
        return knn_tail<Ops, 32>(t, pts, count, k, stride, out, split, order, tail, stats, s);
    }
    if (k <= 4) launch_knn<Ops, 4>(t, pts, count, k, stride, out, wide, split, leaf4, stats, order, s);
    else if (k <= 8) launch_knn<Ops, 8>(t, pts, count, k, stride, out, wide, split, leaf4, stats, order, s);
    else if (k <= 16) launch_knn<Ops, 16>(t, pts, count, k, stride, out, wide, split, leaf4, stats, order, s);
    else launch_knn<Ops, 32>(t, pts, count, k, stride, out, wide, split, leaf4, stats, order, s);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "knn");
}

template <class Ops, bool kFill>
int radius_launch(const qk_tree* t, const float* pts, int count, float r2, int* counts,
                  int* lane_counts, const int* offsets, unsigned long long* keys, unsigned flags,
                  unsigned long long* stats, const uint32_t* order, cudaStream_t s) {
    const float4* leaves = static_cast<const float4*>(t->leaves);
    const int qb = query_block(count);
    const int g = blocks_for(count, qb);
    if ((flags & kSplitFlags) && !(flags & QK_WIDE)) {
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        const int lanes = split_lanes(flags);
        const int gs = blocks_for(static_cast<long long>(count) * lanes);
        if (lanes == 4) {
            if (stats) k_radius_split<Ops, kFill, true, 4><<<gs, kBlock, 0, s>>>(bn, leaves, pts, order, count, r2, counts, lane_counts, offsets, keys, t->n * 2 + 64, stats);
            else k_radius_split<Ops, kFill, false, 4><<<gs, kBlock, 0, s>>>(bn, leaves, pts, order, count, r2, counts, lane_counts, offsets, keys, t->n * 2 + 64, stats);
        } else if (lanes == 8) {
            if (stats) k_radius_split<Ops, kFill, true, 8><<<gs, kBlock, 0, s>>>(bn, leaves, pts, order, count, r2, counts, lane_counts, offsets, keys, t->n * 2 + 64, stats);
            else k_radius_split<Ops, kFill, false, 8><<<gs, kBlock, 0, s>>>(bn, leaves, pts, order, count, r2, counts, lane_counts, offsets, keys, t->n * 2 + 64, stats);
        } else {
            if (stats) k_radius_split<Ops, kFill, true, 32><<<gs, kBlock, 0, s>>>(bn, leaves, pts, order, count, r2, counts, lane_counts, offsets, keys, t->n * 2 + 64, stats);
            else k_radius_split<Ops, kFill, false, 32><<<gs, kBlock, 0, s>>>(bn, leaves, pts, order, count, r2, counts, lane_counts, offsets, keys, t->n * 2 + 64, stats);
        }
    } else if (flags & QK_WIDE) {
        const WideNode* wn = static_cast<const WideNode*>(t->wide);
        if (t->wide_leaf == 4) {
            if (stats) k_radius_wide<Ops, kFill, true, true><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, r2, counts, offsets, keys, t->n * 2 + 64, stats);
            else k_radius_wide<Ops, kFill, false, true><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, r2, counts, offsets, keys, t->n * 2 + 64, stats);
        } else {
            if (stats) k_radius_wide<Ops, kFill, true><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, r2, counts, offsets, keys, t->n * 2 + 64, stats);
            else k_radius_wide<Ops, kFill, false><<<g, qb, 0, s>>>(wn, leaves, pts, order, count, r2, counts, offsets, keys, t->n * 2 + 64, stats);
        }
    } else if (flags & QK_TUNE_LEAF4) {
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        const Node* nodes = static_cast<const Node*>(t->nodes);
        if (stats) k_radius_bin<Ops, kFill, true, true><<<g, qb, 0, s>>>(bn, leaves, nodes, pts, order, count, r2, counts, offsets, keys, t->n * 2 + 64, stats, leaf_nodes(t));
        else k_radius_bin<Ops, kFill, false, true><<<g, qb, 0, s>>>(bn, leaves, nodes, pts, order, count, r2, counts, offsets, keys, t->n * 2 + 64, stats, leaf_nodes(t));
    } else {
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        const Node* nodes = static_cast<const Node*>(t->nodes);
        if (stats) k_radius_bin<Ops, kFill, true><<<g, qb, 0, s>>>(bn, leaves, nodes, pts, order, count, r2, counts, offsets, keys, t->n * 2 + 64, stats);
        else k_radius_bin<Ops, kFill, false><<<g, qb, 0, s>>>(bn, leaves, nodes, pts, order, count, r2, counts, offsets, keys, t->n * 2 + 64, stats);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "radius traversal");
}

template <bool kFill>
int radius_dispatch(const qk_tree* t, const float* pts, int count, float r2, int* counts,
                    int* lane_counts, const int* offsets, unsigned long long* keys, unsigned flags,
                    unsigned long long* stats, const uint32_t* order, cudaStream_t s) {
    switch (t->kind) {
        case kTri: return radius_launch<TriOps, kFill>(t, pts, count, r2, counts, lane_counts, offsets, keys, flags, stats, order, s);
        case kPoint: return radius_launch<PointOps, kFill>(t, pts, count, r2, counts, lane_counts, offsets, keys, flags, stats, order, s);
        case kGauss: return radius_launch<GaussOps, kFill>(t, pts, count, r2, counts, lane_counts, offsets, keys, flags, stats, order, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", t->kind);
    }
}

}  // namespace

// the tail's buffers: the heavy count, the heavy list (every query) and the candidates
TailList carve_tail(Carve& c, int count) {
    TailList t;
    t.count = c.take<int>(1);
    t.list = c.take<int>(count);
    t.partial = c.take<uint2>(static_cast<size_t>(kTailCap) * kTailCands);
    return t;
}

bool use_tail(const qk_tree* t, unsigned flags) {
    return (flags & QK_TUNE_TAIL) && t->kind == kPoint && !(flags & (QK_WIDE | QK_TUNE_LEAF4));
}

size_t point_query_ws_bytes(int count, unsigned flags) {
    Carve c;
    carve_order(c, count);
    if (flags & QK_TUNE_TAIL) carve_tail(c, count);
    return c.used;
}

size_t order_ws_bytes(int count) {
    Carve c;
    carve_order(c, count);
    return c.used;
}

int ray_query(const qk_tree* t, const void* rays, int count, uint64_t* out, int* ids,
              unsigned flags, uint64_t* stats, void* ws, cudaStream_t s) {
    if (count <= 0) return QK_OK;
    Carve c{static_cast<char*>(ws)};
    OrderBufs o = carve_order(c, count);
    int st = QK_OK;
    const bool dir = (flags & QK_ORDER_DIRECTION) != 0;
    const uint32_t* order = make_order(static_cast<const float*>(rays), 8, dir ? 3 : 0, count,
                                       flags, o, s, &st);
    if (st != QK_OK) return st;
    const float4* r4 = static_cast<const float4*>(rays);
    auto* res = reinterpret_cast<unsigned long long*>(out);
    auto* stt = reinterpret_cast<unsigned long long*>(stats);
    const float4* leaves = static_cast<const float4*>(t->leaves);
    const int g = blocks_for(count);
    if (flags & QK_WIDE) {
        const WideNode* wn = static_cast<const WideNode*>(t->wide);
        if (t->wide_leaf == 4) {
            if (stt) k_ray_wide<true, true><<<g, kBlock, 0, s>>>(wn, leaves, r4, order, count, res, ids, t->n * 2 + 64, stt);
            else k_ray_wide<false, true><<<g, kBlock, 0, s>>>(wn, leaves, r4, order, count, res, ids, t->n * 2 + 64, stt);
        } else {
            if (stt) k_ray_wide<true><<<g, kBlock, 0, s>>>(wn, leaves, r4, order, count, res, ids, t->n * 2 + 64, stt);
            else k_ray_wide<false><<<g, kBlock, 0, s>>>(wn, leaves, r4, order, count, res, ids, t->n * 2 + 64, stt);
        }
    } else if (flags & QK_TUNE_DYNAMIC) {
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        const Node* nodes = static_cast<const Node*>(t->nodes);
        cudaMemsetAsync(&o.h->counter, 0, sizeof(int), s);
        int sms = 148;
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const bool occ = (flags & QK_TUNE_HIGH_OCC) != 0;
        const int grid = min(blocks_for(count), sms * (occ ? 5 : 4));
        if (occ) {
            if (stt) k_ray_bin_dyn<true, 5><<<grid, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, &o.h->counter, t->n * 2 + 64, stt);
            else k_ray_bin_dyn<false, 5><<<grid, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, &o.h->counter, t->n * 2 + 64, stt);
        } else {
            if (stt) k_ray_bin_dyn<true, 4><<<grid, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, &o.h->counter, t->n * 2 + 64, stt);
            else k_ray_bin_dyn<false, 4><<<grid, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, &o.h->counter, t->n * 2 + 64, stt);
        }
    } else {
        const BNode* bn = static_cast<const BNode*>(t->bnodes);
        const Node* nodes = static_cast<const Node*>(t->nodes);
        if ((flags & QK_TUNE_HIGH_OCC) && (flags & QK_TUNE_SHORT_STACK)) {
            if (stt) k_ray_bin<true, 5, 8><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt);
            else k_ray_bin<false, 5, 8><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt);
        } else if (flags & QK_TUNE_SHORT_STACK) {
            if (stt) k_ray_bin<true, 1, 8><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt);
            else k_ray_bin<false, 1, 8><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt);
        } else if ((flags & QK_TUNE_HIGH_OCC) && (flags & QK_TUNE_LEAF4)) {
            if (stt) k_ray_bin<true, 5, 0, true><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt, leaf_nodes(t));
            else k_ray_bin<false, 5, 0, true><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt, leaf_nodes(t));
        } else if (flags & QK_TUNE_LEAF4) {
            if (stt) k_ray_bin<true, 1, 0, true><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt, leaf_nodes(t));
            else k_ray_bin<false, 1, 0, true><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt, leaf_nodes(t));
        } else if (order) {
            // the previous kernel in the stream wrote the order: start while it drains
            const Node* no_leaf4 = nullptr;
            if (flags & QK_TUNE_HIGH_OCC) {
                if (stt) launch_pdl(k_ray_bin<true, 5>, dim3(g), dim3(kBlock), s, bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt, no_leaf4);
                else launch_pdl(k_ray_bin<false, 5>, dim3(g), dim3(kBlock), s, bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt, no_leaf4);
            } else {
                if (stt) launch_pdl(k_ray_bin<true, 1>, dim3(g), dim3(kBlock), s, bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt, no_leaf4);
                else launch_pdl(k_ray_bin<false, 1>, dim3(g), dim3(kBlock), s, bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt, no_leaf4);
            }
        } else if (flags & QK_TUNE_HIGH_OCC) {
            if (stt) k_ray_bin<true, 5><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt);
            else k_ray_bin<false, 5><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt);
        } else {
            if (stt) k_ray_bin<true, 1><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt);
            else k_ray_bin<false, 1><<<g, kBlock, 0, s>>>(bn, leaves, nodes, r4, order, count, res, ids, t->n * 2 + 64, stt);
        }
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "raycast");
}

int closest_query(const qk_tree* t, const float* pts, int count, void* out, unsigned flags,
                  uint64_t* stats, void* ws, cudaStream_t s) {
    if (count <= 0) return QK_OK;
    Carve c{static_cast<char*>(ws)};
    OrderBufs o = carve_order(c, count);
    TailList tail;
    if (flags & QK_TUNE_TAIL) {
        const TailList carved = carve_tail(c, count);
        if (use_tail(t, flags)) tail = carved;
    }
    int st = QK_OK;
    const uint32_t* order = make_order(pts, 3, 0, count, flags, o, s, &st);
    if (st != QK_OK) return st;
    auto* res = static_cast<uint2*>(out);
    auto* stt = reinterpret_cast<unsigned long long*>(stats);
    switch (t->kind) {
        case kTri: return closest_impl<TriOps>(t, pts, count, res, flags, stt, order, s);
        case kPoint: return closest_impl<PointOps>(t, pts, count, res, flags, stt, order, s, tail);
        case kGauss: return closest_impl<GaussOps>(t, pts, count, res, flags, stt, order, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", t->kind);
    }
}

int knn_query(const qk_tree* t, const float* pts, int count, int k, int stride, void* out,
              unsigned flags, uint64_t* stats, void* ws, cudaStream_t s) {
    if (count <= 0) return QK_OK;
    Carve c{static_cast<char*>(ws)};
    OrderBufs o = carve_order(c, count);
    TailList tail;
    if (flags & QK_TUNE_TAIL) {
        const TailList carved = carve_tail(c, count);
        if (use_tail(t, flags)) tail = carved;
    }
    int st = QK_OK;
    const uint32_t* order = make_order(pts, 3, 0, count, flags, o, s, &st);
    if (st != QK_OK) return st;
    auto* res = static_cast<uint2*>(out);
    auto* stt = reinterpret_cast<unsigned long long*>(stats);
    switch (t->kind) {
        case kTri: return knn_impl<TriOps>(t, pts, count, k, stride, res, flags, stt, order, s);
        case kPoint: return knn_impl<PointOps>(t, pts, count, k, stride, res, flags, stt, order, s, tail);
        case kGauss: return knn_impl<GaussOps>(t, pts, count, k, stride, res, flags, stt, order, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", t->kind);
    }
}

// the single-pass pool applies to the binary thread-per-query traversal only
bool use_stash(unsigned flags) {
    return (flags & QK_TUNE_STASH) && !(flags & (kSplitFlags | QK_WIDE));
}

size_t radius_ws_bytes(int count, unsigned flags) {
    Carve c;
    carve_order(c, count);
    c.take<int>(count);            // counts
    c.take<char>(scan_ws_bytes(count));
    c.take<int>(count);            // medium segment list
    c.take<int>(count);            // large segment list
    if (flags & kSplitFlags) c.take<int>(static_cast<size_t>(count) * 32);  // lane counts
    if (use_stash(flags)) carve_pool(c, count);
    return c.used;
}

template <class Ops>
int radius_pool_launch(const qk_tree* t, const float* pts, int count, float r2, int* counts,
                       const int* offsets, const RadiusPool& pool, unsigned long long* keys,
                       unsigned flags, unsigned long long* stats, const uint32_t* order,
                       bool fill, cudaStream_t s) {
    const BNode* bn = static_cast<const BNode*>(t->bnodes);
    const Node* nodes = static_cast<const Node*>(t->nodes);
    const float4* leaves = static_cast<const float4*>(t->leaves);
    const int qb = query_block(count);
    const int g = blocks_for(count, qb);
    const int it = t->n * 2 + 64;
    const bool leaf4 = (flags & QK_TUNE_LEAF4) != 0;
    if (fill) {
        k_radius_gather<<<blocks_for(static_cast<long long>(count) * 32), kBlock, 0, s>>>(
            pool, offsets, count, keys, -1);
        if (leaf4) k_radius_fill_lost<Ops, true><<<g, qb, 0, s>>>(bn, leaves, nodes, pts, count, r2, offsets, pool, keys, it, leaf_nodes(t));
        else k_radius_fill_lost<Ops><<<g, qb, 0, s>>>(bn, leaves, nodes, pts, count, r2, offsets, pool, keys, it);
    } else {
        cudaMemsetAsync(pool.taken, 0, sizeof(int), s);
        if (leaf4) {
            if (stats) k_radius_count_pool<Ops, true, true><<<g, qb, 0, s>>>(bn, leaves, nodes, pts, order, count, r2, counts, pool, it, stats, leaf_nodes(t));
            else k_radius_count_pool<Ops, false, true><<<g, qb, 0, s>>>(bn, leaves, nodes, pts, order, count, r2, counts, pool, it, stats, leaf_nodes(t));
        } else {
            if (stats) k_radius_count_pool<Ops, true><<<g, qb, 0, s>>>(bn, leaves, nodes, pts, order, count, r2, counts, pool, it, stats);
            else k_radius_count_pool<Ops, false><<<g, qb, 0, s>>>(bn, leaves, nodes, pts, order, count, r2, counts, pool, it, stats);
        }
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "radius traversal (single pass)");
}

int radius_pool_dispatch(const qk_tree* t, const float* pts, int count, float r2, int* counts,
                         const int* offsets, const RadiusPool& pool, unsigned long long* keys,
                         unsigned flags, unsigned long long* stats, const uint32_t* order,
                         bool fill, cudaStream_t s) {
    switch (t->kind) {
        case kTri: return radius_pool_launch<TriOps>(t, pts, count, r2, counts, offsets, pool, keys, flags, stats, order, fill, s);
        case kPoint: return radius_pool_launch<PointOps>(t, pts, count, r2, counts, offsets, pool, keys, flags, stats, order, fill, s);
        case kGauss: return radius_pool_launch<GaussOps>(t, pts, count, r2, counts, offsets, pool, keys, flags, stats, order, fill, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", t->kind);
    }
}

int radius_count(const qk_tree* t, const float* pts, int count, float r, int* offsets,
                 long long* total, unsigned flags, uint64_t* stats, void* ws, cudaStream_t s) {
    *total = 0;
    if (count <= 0) {
        cudaMemsetAsync(offsets, 0, sizeof(int), s);
        return QK_OK;
    }
    Carve c{static_cast<char*>(ws)};
    OrderBufs o = carve_order(c, count);
    int* counts = c.take<int>(count);
    void* scan_ws = c.take<char>(scan_ws_bytes(count));
    c.take<int>(count);
    c.take<int>(count);
    int* lane_counts = (flags & kSplitFlags) ? c.take<int>(static_cast<size_t>(count) * 32) : nullptr;
    const bool pooled = use_stash(flags);
    const RadiusPool pool = pooled ? carve_pool(c, count) : RadiusPool{};
    int st = QK_OK;
    const uint32_t* order = make_order(pts, 3, 0, count, flags, o, s, &st);
    if (st != QK_OK) return st;
    if (pooled)
        st = radius_pool_dispatch(t, pts, count, r * r, counts, nullptr, pool, nullptr, flags,
                                  reinterpret_cast<unsigned long long*>(stats), order, false, s);
    else
        st = radius_dispatch<false>(t, pts, count, r * r, counts, lane_counts, nullptr, nullptr, flags,
                                    reinterpret_cast<unsigned long long*>(stats), order, s);
    if (st != QK_OK) return st;
    cudaError_t e = scan_exclusive(counts, offsets, count, true, scan_ws, s);
    if (e != cudaSuccess) return cuda_status(e, "radius scan");
    int tot = 0;
    e = cudaMemcpyAsync(&tot, offsets + count, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "radius total readback");
    *total = tot;
    return QK_OK;
}

int radius_fill(const qk_tree* t, const float* pts, int count, float r, const int* offsets,
                uint64_t* keys, unsigned flags, void* ws, cudaStream_t s) {
    if (count <= 0) return QK_OK;
    Carve c{static_cast<char*>(ws)};
    OrderBufs o = carve_order(c, count);
    c.take<int>(count);
    c.take<char>(scan_ws_bytes(count));
    int* medium = c.take<int>(count);
    int* large = c.take<int>(count);
    int* lane_counts = (flags & kSplitFlags) ? c.take<int>(static_cast<size_t>(count) * 32) : nullptr;
    const bool pooled = use_stash(flags);
    const RadiusPool pool = pooled ? carve_pool(c, count) : RadiusPool{};
    auto* k64 = reinterpret_cast<unsigned long long*>(keys);
    int st = QK_OK;
    if (pooled) {
        // the fill pass only copies (and traverses again the queries the pool could not hold,
        // in query order): no ray order is needed
        st = radius_pool_dispatch(t, pts, count, r * r, nullptr, offsets, pool, k64, flags, nullptr,
                                  nullptr, true, s);
        if (st != QK_OK) return st;
        return radius_sort_segments(offsets, count, keys, medium, large, o.h, -1, s);
    }
    const uint32_t* order = make_order(pts, 3, 0, count, flags, o, s, &st);
    if (st != QK_OK) return st;
    st = radius_dispatch<true>(t, pts, count, r * r, nullptr, lane_counts, offsets, k64, flags,
                               nullptr, order, s);
    if (st != QK_OK) return st;
    // reset the segment lists (make_order only resets them on its Morton path)
    return radius_sort_segments(offsets, count, keys, medium, large, o.h, -1, s);
}

int radius_sort_segments(const int* offsets, int count, uint64_t* keys, int* medium, int* large,
                         Header* h, long long cap, cudaStream_t s) {
    auto* k64 = reinterpret_cast<unsigned long long*>(keys);
    k_bounds_reset<<<1, 32, 0, s>>>(h, 0);
    k_seg_sort_warp<<<blocks_for(count, kBlock / 32), kBlock, 0, s>>>(offsets, count, k64, medium,
                                                                      large, h, cap);
    k_seg_sort_warp_reg<<<148 * 8, kWarpSortBlock, 0, s>>>(offsets, k64, medium, h);
    k_seg_sort_block<<<148 * 2, kBlock, 0, s>>>(offsets, k64, large, h);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "radius sort");
}

}  // namespace qk
