// qk_sah.cu -- top-down binned SAH builder (the reference's buildBVHSahGPU,
// src/gpu/lbvh.cu:827-1291 and 1777-2135), organised for B200.
//
// The output keeps the LBVH numbering (internal nodes 0..n-2, leaf of slot s at n-1+s), so
// boxes, traversal nodes, 4-wide collapse, refit and validation are shared with the LBVH.
// Three tiers, all deterministic (commutative atomics for bins, stable partitions, node ids
// from prefix sums or from sequential per-subtree counters):
//   global   ranges of more than kTaskRange primitives, level by level: chunks of 4096
//            primitives bin their centroids in shared memory (count + primitive box per bin,
//            3 axes) and merge into per-range bins with ordered-uint atomics; one thread per
//            range sweeps the bins for the cheapest area(L)*nL + area(R)*nR split; a stable
//            partition by chunk-local block scans writes the new order.  One host sync per
//            level (the next level's range count); chunk grids are sized by a bound.
//   warp     every range of at most kTaskRange (256) primitives is handed to one warp
//            (k_warp_tasks): binned SAH with warp-private bins down to 32 primitives
//            (warp_piece_tree), then the exact sweep below; no block barriers, no global
//            synchronisation.  The block tier (k_block_build: one thread block per range of up
//            to 1024 in shared memory) now only builds forest tasks above 256 (topology edits).
//   warp     pieces of at most 32 primitives are finished by one warp each with an exact
//            sweep: for every axis the lanes sort by centroid (bitonic, ties by position), scan
//            prefix and suffix boxes, and evaluate every split position.
// Depth stays below the 64-entry traversal stacks: a split is only taken while
// depth + ceil(log2(larger child)) <= kMaxDepth, otherwise the range is halved by count.
#include "qk_build.cuh"

namespace qk {

namespace {

constexpr int kChunk = 2048;       // primitives binned per block at the global tier
constexpr int kBlockRange = 1024;  // largest range built by one block (forest tasks)
constexpr int kTaskRange = 256;    // largest range the global tier hands to one warp
constexpr int kWarpRange = 32;     // largest range finished by one warp
constexpr int kMaxBins = 64;
constexpr int kMaxDepth = 62;
constexpr int kLevelsPerSync = 4;  // global-tier levels between host read-backs
constexpr int kBinWords = 7;       // count, lo xyz, hi xyz

struct Task {
    int begin, end, node, depth;
};

__device__ __forceinline__ int ceil_log2(int c) { return c <= 1 ? 0 : 32 - __clz(c - 1); }

__device__ __forceinline__ float half_area(float3 lo, float3 hi) {
    const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
    return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ int bin_of(float c, float lo, float hi, int bins) {
    const float ext = hi - lo;
    if (!(ext > 0.0f)) return 0;
    int b = __float2int_rd((c - lo) * (static_cast<float>(bins) / ext));
    return b < 0 ? 0 : (b >= bins ? bins - 1 : b);
}

// child reference as the traversal nodes store it
__device__ __forceinline__ int child_ref(int id, int n) { return id >= n - 1 ? ~(id - (n - 1)) : id; }

__device__ __forceinline__ void link(Node* nodes, BNode* bn, int* parent, int node, int l, int r,
                                     int n) {
    nodes[node].left = l;
    nodes[node].right = r;
    parent[l] = node;
    parent[r] = node;
    bn[node].v3 = make_float4(__int_as_float(child_ref(l, n)), __int_as_float(child_ref(r, n)),
                              0.0f, 0.0f);
}

// centroid and box of every primitive, in scene order
template <class Ops>
__global__ __launch_bounds__(kBlock) void k_prim_geom(const float* __restrict__ items, int n,
                                                     float4* __restrict__ cen,
                                                     float4* __restrict__ lo,
                                                     float4* __restrict__ hi,
                                                     int* __restrict__ order) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= n) return;
    const float* it = items + static_cast<size_t>(i) * Ops::kFloats;
    const float3 c = Ops::centroid(it);
    const Box b = Ops::bounds(it);
    cen[i] = make_float4(c.x, c.y, c.z, 0.0f);
    lo[i] = make_float4(b.lo.x, b.lo.y, b.lo.z, 0.0f);
    hi[i] = make_float4(b.hi.x, b.hi.y, b.hi.z, 0.0f);
    order[i] = i;
}

// ---------------------------------------------------------------------------------------
// global tier
// ---------------------------------------------------------------------------------------
struct Level {
    Task* tasks;        // current big tasks
    int* chunk_task;    // chunk -> task
    int* chunk_begin;
    int* chunk_first;   // first chunk of each task
    unsigned* cb;       // per task: centroid bounds lo xyz, hi xyz (ordered)
    unsigned* bins;     // per task: 3 * bins * kBinWords
    int* split;         // per task: axis * 256 + bin (-1 = count split)
    int* left_count;    // per task
    int* chunk_left;    // per chunk: left primitives
    int* counters;      // [0] chunks, [1] next big tasks, [2] block tasks, [3] internal base,
                        // [4] this level's big tasks (the previous level's [1]), [5] the warp
                        // tier's next task
};

// One block of 1024 threads: the chunk list of `ntask` tasks (kChunk primitives per chunk):
// each task's first chunk, every chunk's task and first position, the chunk count.
__device__ __forceinline__ void level_chunks(const Level& L, const Task* __restrict__ tasks,
                                             int ntask) {
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ntask; base += 1024) {
        const int t = base + threadIdx.x;
        int nch = 0;
        if (t < ntask) nch = (tasks[t].end - tasks[t].begin + kChunk - 1) / kChunk;
        // block exclusive scan of nch (warp shuffles + shared totals)
        __shared__ int wsum[32];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        int v = nch;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        if (lane == 31) wsum[warp] = v;
        __syncthreads();
        if (warp == 0) {
            int s = wsum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            wsum[lane] = s;
        }
        __syncthreads();
        const int excl = carry + (warp ? wsum[warp - 1] : 0) + v - nch;
        if (t < ntask) {
            L.chunk_first[t] = excl;
            for (int c = 0; c < nch; ++c) {
                L.chunk_task[excl + c] = t;
                L.chunk_begin[excl + c] = tasks[t].begin + c * kChunk;
            }
        }
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + nch;
        __syncthreads();
    }
    if (threadIdx.x == 0) L.counters[0] = carry;
}

// single block: chunk list of the first level's tasks (later levels' come from k_level_assign)
__global__ __launch_bounds__(1024) void k_level_prep(Level L) {
    level_chunks(L, L.tasks, L.counters[4]);
}

// one block per range: reset its centroid bounds and bins
__global__ __launch_bounds__(kBlock) void k_level_reset(Level L, int bins) {
    const int t = blockIdx.x;
    if (t >= L.counters[4]) return;  // grid sized by a bound
    if (threadIdx.x < 6) L.cb[6 * t + threadIdx.x] = threadIdx.x < 3 ? ord_f(kInf) : ord_f(-kInf);
    unsigned* B = L.bins + static_cast<size_t>(t) * 3 * kMaxBins * kBinWords;
    for (int j = threadIdx.x; j < 3 * bins * kBinWords; j += kBlock) {
        const int w = j % kBinWords;
        B[j] = w == 0 ? 0u : (w <= 3 ? ord_f(kInf) : ord_f(-kInf));
    }
}

__global__ __launch_bounds__(kBlock) void k_level_cbounds(Level L, const int* __restrict__ order,
                                                         const float4* __restrict__ cen) {
    if (static_cast<int>(blockIdx.x) >= L.counters[0]) return;  // grid sized by a bound
    const int c = blockIdx.x;
    const int t = L.chunk_task[c];
    const int b = L.chunk_begin[c];
    const int e = min(b + kChunk, L.tasks[t].end);
    float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
    for (int i = b + threadIdx.x; i < e; i += kBlock) {
        const float4 p = cen[order[i]];
        lo[0] = fminf(lo[0], p.x);
        lo[1] = fminf(lo[1], p.y);
        lo[2] = fminf(lo[2], p.z);
        hi[0] = fmaxf(hi[0], p.x);
        hi[1] = fmaxf(hi[1], p.y);
        hi[2] = fmaxf(hi[2], p.z);
    }
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    // the block's bounds, then six atomics per block (every block of a large range updates
    // the same six words)
    __shared__ unsigned wb[kBlock / 32][6];
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; ++a) {
            wb[threadIdx.x >> 5][a] = ord_f(lo[a]);
            wb[threadIdx.x >> 5][3 + a] = ord_f(hi[a]);
        }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int j = threadIdx.x;
        unsigned v = wb[0][j];
        for (int w = 1; w < kBlock / 32; ++w) v = j < 3 ? min(v, wb[w][j]) : max(v, wb[w][j]);
        if (j < 3) atomicMin(&L.cb[6 * t + j], v);
        else atomicMax(&L.cb[6 * t + j], v);
    }
}

__global__ __launch_bounds__(kBlock) void k_level_bins(Level L, const int* __restrict__ order,
                                                      const float4* __restrict__ cen,
                                                      const float4* __restrict__ plo,
                                                      const float4* __restrict__ phi, int bins) {
    __shared__ unsigned sb[3 * kMaxBins * kBinWords];
    if (static_cast<int>(blockIdx.x) >= L.counters[0]) return;  // grid sized by a bound
    for (int j = threadIdx.x; j < 3 * bins * kBinWords; j += kBlock) {
        const int w = j % kBinWords;
        sb[j] = w == 0 ? 0u : (w <= 3 ? ord_f(kInf) : ord_f(-kInf));
    }
    __syncthreads();
    const int c = blockIdx.x;
    const int t = L.chunk_task[c];
    const int b = L.chunk_begin[c];
    const int e = min(b + kChunk, L.tasks[t].end);
    float clo[3], chi[3];
    for (int a = 0; a < 3; ++a) {
        clo[a] = unord_f(L.cb[6 * t + a]);
        chi[a] = unord_f(L.cb[6 * t + 3 + a]);
    }
    // Each thread bins a contiguous run of positions.  Partitioned ranges keep nearby
    // primitives together, so consecutive positions mostly fall in the same bin: the thread
    // accumulates a bin's count and box in registers and issues the shared-memory atomics only
    // when the bin changes (count, min and max are exact in any grouping).
    const int per = (e - b + kBlock - 1) / kBlock;
    const int i0 = b + threadIdx.x * per, i1 = min(i0 + per, e);
    int cur[3] = {-1, -1, -1};
    unsigned acc[3][kBinWords];
    auto flush = [&](int a) {
        unsigned* w = sb + (a * bins + cur[a]) * kBinWords;
        atomicAdd(&w[0], acc[a][0]);
        atomicMin(&w[1], acc[a][1]);
        atomicMin(&w[2], acc[a][2]);
        atomicMin(&w[3], acc[a][3]);
        atomicMax(&w[4], acc[a][4]);
        atomicMax(&w[5], acc[a][5]);
        atomicMax(&w[6], acc[a][6]);
    };
    // the run in pairs: both primitives' gathers are issued together (groups of four held 108
    // registers and ran slower at the lower occupancy)
    constexpr int kGroup = 2;
    for (int g = i0; g < i1; g += kGroup) {
        int pg[kGroup];
#pragma unroll
        for (int u = 0; u < kGroup; ++u) pg[u] = g + u < i1 ? order[g + u] : -1;
        float4 cg[kGroup], lg[kGroup], hg[kGroup];
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
            if (pg[u] >= 0) {
                cg[u] = cen[pg[u]];
                lg[u] = plo[pg[u]];
                hg[u] = phi[pg[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
            if (pg[u] < 0) break;
            const float4 lo = lg[u], hi = hg[u];
            const float cv[3] = {cg[u].x, cg[u].y, cg[u].z};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int bin = bin_of(cv[a], clo[a], chi[a], bins);
                if (bin != cur[a]) {
                    if (cur[a] >= 0) flush(a);
                    cur[a] = bin;
                    acc[a][0] = 1u;
                    acc[a][1] = ord_f(lo.x);
                    acc[a][2] = ord_f(lo.y);
                    acc[a][3] = ord_f(lo.z);
                    acc[a][4] = ord_f(hi.x);
                    acc[a][5] = ord_f(hi.y);
                    acc[a][6] = ord_f(hi.z);
                } else {
                    acc[a][0] += 1u;
                    acc[a][1] = min(acc[a][1], ord_f(lo.x));
                    acc[a][2] = min(acc[a][2], ord_f(lo.y));
                    acc[a][3] = min(acc[a][3], ord_f(lo.z));
                    acc[a][4] = max(acc[a][4], ord_f(hi.x));
                    acc[a][5] = max(acc[a][5], ord_f(hi.y));
                    acc[a][6] = max(acc[a][6], ord_f(hi.z));
                }
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
        if (cur[a] >= 0) flush(a);
    __syncthreads();
    unsigned* B = L.bins + static_cast<size_t>(t) * 3 * kMaxBins * kBinWords;
    for (int j = threadIdx.x; j < 3 * bins * kBinWords; j += kBlock) {
        const int w = j % kBinWords;
        if (w == 0) {
            if (sb[j]) atomicAdd(&B[j], sb[j]);
        } else if (w <= 3) {
            atomicMin(&B[j], sb[j]);
        } else {
            atomicMax(&B[j], sb[j]);
        }
    }
}

// Sweep of 3 x (bins - 1) candidate planes of one range given its bins (ordered-uint words),
// by one warp: plane b (between bins b-1 and b) costs area(left) * nL + area(right) * nR over
// the bins' primitive boxes; planes with an empty side are skipped; the cheapest wins, ties
// to the lowest axis and then the lowest plane.  Returns axis * 256 + plane and the left
// count, or -1 when no plane separates the centroids.
// Lane l owns bins 2l and 2l+1; prefix and suffix boxes and counts come from warp scans (min /
// max and integer sums are exact, so every cost equals a sequential sweep's).  All 32 lanes
// call it; all get the result.
__device__ int warp_sweep_bins(const unsigned* B, int bins, int count, int* left_out) {
    const int lane = threadIdx.x & 31;
    float best = kInf;
    int best_split = -1, best_left = 0;
    const float3 elo = f3(kInf, kInf, kInf), ehi = f3(-kInf, -kInf, -kInf);
    auto uni = [](float3& lo, float3& hi, float3 l2, float3 h2) {
        lo = f3(fminf(lo.x, l2.x), fminf(lo.y, l2.y), fminf(lo.z, l2.z));
        hi = f3(fmaxf(hi.x, h2.x), fmaxf(hi.y, h2.y), fmaxf(hi.z, h2.z));
    };
    auto shfl3 = [](float3 v, int src) {
        return f3(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                  __shfl_sync(0xffffffffu, v.z, src));
    };
    for (int a = 0; a < 3; ++a) {
        float3 lo[2], hi[2];
        int c[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int b = 2 * lane + k;
            lo[k] = elo;
            hi[k] = ehi;
            c[k] = 0;
            if (b < bins) {
                const unsigned* w = B + (a * bins + b) * kBinWords;
                c[k] = static_cast<int>(w[0]);
                if (c[k]) {
                    lo[k] = f3(unord_f(w[1]), unord_f(w[2]), unord_f(w[3]));
                    hi[k] = f3(unord_f(w[4]), unord_f(w[5]), unord_f(w[6]));
                }
            }
        }
        // lane totals, exclusive prefix from the lower lanes, exclusive suffix from the upper
        float3 tlo = lo[0], thi = hi[0];
        uni(tlo, thi, lo[1], hi[1]);
        const int tc = c[0] + c[1];
        float3 plo = tlo, phi = thi;
        int pc = tc;
        float3 qlo = tlo, qhi = thi;
        int qc = tc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float3 ul = shfl3(plo, max(lane - o, 0)), uh = shfl3(phi, max(lane - o, 0));
            const int ucnt = __shfl_sync(0xffffffffu, pc, max(lane - o, 0));
            const float3 dl = shfl3(qlo, min(lane + o, 31)), dh = shfl3(qhi, min(lane + o, 31));
            const int dcnt = __shfl_sync(0xffffffffu, qc, min(lane + o, 31));
            if (lane >= o) {
                uni(plo, phi, ul, uh);
                pc += ucnt;
            }
            if (lane + o < 32) {
                uni(qlo, qhi, dl, dh);
                qc += dcnt;
            }
        }
        // exclusive = inclusive of the neighbour
        float3 xlo = shfl3(plo, max(lane - 1, 0)), xhi = shfl3(phi, max(lane - 1, 0));
        int xc = __shfl_sync(0xffffffffu, pc, max(lane - 1, 0));
        float3 ylo = shfl3(qlo, min(lane + 1, 31)), yhi = shfl3(qhi, min(lane + 1, 31));
        int yc = __shfl_sync(0xffffffffu, qc, min(lane + 1, 31));
        if (lane == 0) {
            xlo = elo;
            xhi = ehi;
            xc = 0;
        }
        if (lane == 31) {
            ylo = elo;
            yhi = ehi;
            yc = 0;
        }
        // left prefix through bin 2l and 2l+1; right suffix from bin 2l+1 and 2l+2
        float3 l0lo = xlo, l0hi = xhi;
        uni(l0lo, l0hi, lo[0], hi[0]);
        const int l0c = xc + c[0];
        float3 l1lo = l0lo, l1hi = l0hi;
        uni(l1lo, l1hi, lo[1], hi[1]);
        const int l1c = l0c + c[1];
        float3 r1lo = ylo, r1hi = yhi;  // suffix from bin 2l+1
        uni(r1lo, r1hi, lo[1], hi[1]);
        const float3 r2lo = ylo, r2hi = yhi;  // suffix from bin 2l+2
        float lcost = kInf;
        int lsplit = 0x7fffffff, lleft = 0;
        // plane after bin 2l (valid when 2l <= bins - 2)
        if (2 * lane <= bins - 2 && l0c != 0 && l0c != count) {
            lcost = half_area(l0lo, l0hi) * static_cast<float>(l0c) +
                    half_area(r1lo, r1hi) * static_cast<float>(count - l0c);
            lsplit = 2 * lane + 1;
            lleft = l0c;
        }
        if (2 * lane + 1 <= bins - 2 && l1c != 0 && l1c != count) {
            const float cost = half_area(l1lo, l1hi) * static_cast<float>(l1c) +
                               half_area(r2lo, r2hi) * static_cast<float>(count - l1c);
            if (cost < lcost) {
                lcost = cost;
                lsplit = 2 * lane + 2;
                lleft = l1c;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float oc = __shfl_xor_sync(0xffffffffu, lcost, o);
            const int os = __shfl_xor_sync(0xffffffffu, lsplit, o);
            const int ol = __shfl_xor_sync(0xffffffffu, lleft, o);
            if (oc < lcost || (oc == lcost && os < lsplit)) {
                lcost = oc;
                lsplit = os;
                lleft = ol;
            }
        }
        if (lcost < best) {
            best = lcost;
            best_split = a * 256 + lsplit;
            best_left = lleft;
        }
    }
    *left_out = best_left;
    return best_split;
}

// one warp per range
__global__ __launch_bounds__(kBlock) void k_level_split(Level L, int bins) {
    const int t = (blockIdx.x * kBlock + threadIdx.x) >> 5;
    if (t >= L.counters[4]) return;  // grid sized by a bound
    const Task tk = L.tasks[t];
    const int count = tk.end - tk.begin;
    int lc = 0;
    int s = warp_sweep_bins(L.bins + static_cast<size_t>(t) * 3 * kMaxBins * kBinWords, bins,
                            count, &lc);
    if (s >= 0 && tk.depth + 1 + ceil_log2(max(lc, count - lc)) > kMaxDepth) s = -1;
    if (s < 0) lc = count / 2;
    if ((threadIdx.x & 31) == 0) {
        L.split[t] = s;
        L.left_count[t] = lc;
    }
}

__device__ __forceinline__ bool goes_left(int split, int pos, int begin, int lc, float4 c,
                                          const unsigned* cb, int bins) {
    if (split < 0) return pos - begin < lc;
    const int a = split >> 8;
    const float v = a == 0 ? c.x : (a == 1 ? c.y : c.z);
    return bin_of(v, unord_f(cb[a]), unord_f(cb[3 + a]), bins) < (split & 255);
}

// per chunk: count the primitives that go left
__global__ __launch_bounds__(kBlock) void k_level_count_left(Level L, const int* __restrict__ order,
                                                            const float4* __restrict__ cen,
                                                            int bins) {
    if (static_cast<int>(blockIdx.x) >= L.counters[0]) return;  // grid sized by a bound
    const int c = blockIdx.x;
    const int t = L.chunk_task[c];
    const Task tk = L.tasks[t];
    const int b = L.chunk_begin[c];
    const int e = min(b + kChunk, tk.end);
    const int split = L.split[t], lc = L.left_count[t];
    int cnt = 0;
    for (int i = b + threadIdx.x; i < e; i += kBlock) {
        cnt += goes_left(split, i, tk.begin, lc, cen[order[i]], L.cb + 6 * t, bins) ? 1 : 0;
    }
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    __shared__ int ws[kBlock / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < kBlock / 32; ++w) s += ws[w];
        L.chunk_left[c] = s;
    }
}

// stable partition of each chunk (left block first, then right block) into `out` where the
// child stays in the global tier (more than kTaskRange primitives) and into `fin`, the final
// order the warp tier and the leaves read, where the child's range is final; the lefts of the
// task's earlier chunks are summed from their counts by the whole block
__global__ __launch_bounds__(kBlock) void k_level_partition(Level L, const int* __restrict__ order,
                                                           int* __restrict__ out,
                                                           int* __restrict__ fin,
                                                           const float4* __restrict__ cen,
                                                           int bins) {
    if (static_cast<int>(blockIdx.x) >= L.counters[0]) return;  // grid sized by a bound
    const int c = blockIdx.x;
    const int t = L.chunk_task[c];
    const Task tk = L.tasks[t];
    const int b = L.chunk_begin[c];
    const int e = min(b + kChunk, tk.end);
    const int split = L.split[t], lc = L.left_count[t];
    __shared__ int wsum[kBlock / 32];
    __shared__ int carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int before = 0;
    for (int j = L.chunk_first[t] + threadIdx.x; j < c; j += kBlock) before += L.chunk_left[j];
    before = __reduce_add_sync(0xffffffffu, before);
    if (lane == 0) wsum[warp] = before;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    int left_before = 0;                            // lefts in earlier chunks of this task
    for (int w = 0; w < kBlock / 32; ++w) left_before += wsum[w];
    __syncthreads();
    const int right_before = (b - tk.begin) - left_before;
    for (int base = b; base < e; base += kBlock) {
        const int i = base + threadIdx.x;
        int p = 0;
        int f = 0;
        if (i < e) {
            p = order[i];
            f = goes_left(split, i, tk.begin, lc, cen[p], L.cb + 6 * t, bins) ? 1 : 0;
        }
        int v = f;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        if (lane == 31) wsum[warp] = v;
        __syncthreads();
        int wpre = 0, tot = 0;
        for (int w = 0; w < kBlock / 32; ++w) {
            if (w < warp) wpre += wsum[w];
            tot += wsum[w];
        }
        const int lrank = carry + wpre + v - f;  // lefts before i inside this chunk
        if (i < e) {
            const int dst = f ? tk.begin + left_before + lrank
                              : tk.begin + lc + right_before + (i - b - lrank);
            const int child = f ? lc : tk.end - tk.begin - lc;
            (child > kTaskRange ? out : fin)[dst] = p;
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
}

// single block: node ids for the children (prefix sums over tasks), next big tasks and the
// block-tier list; the next level's task count to counters[4]
__global__ __launch_bounds__(1024) void k_level_assign(Level L, Task* __restrict__ next,
                                                      Task* __restrict__ blocks, Node* nodes,
                                                      BNode* bn, int* parent, int n) {
    __shared__ int carry[3];
    __shared__ int wsum[3][32];
    const int ntask = L.counters[4];  // read by every thread before the first barrier
    if (threadIdx.x < 3) carry[threadIdx.x] = 0;
    __syncthreads();
    const int base_id = L.counters[3];
    const int base_big = L.counters[1];
    const int base_blk = L.counters[2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < ntask; base += 1024) {
        const int t = base + threadIdx.x;
        int lc = 0, rc = 0;
        Task tk{0, 0, 0, 0};
        if (t < ntask) {
            tk = L.tasks[t];
            lc = L.left_count[t];
            rc = tk.end - tk.begin - lc;
        }
        int cnt[3];
        cnt[0] = t < ntask ? (lc >= 2) + (rc >= 2) : 0;                           // internal ids
        cnt[1] = t < ntask ? (lc > kTaskRange) + (rc > kTaskRange) : 0;           // big tasks
        cnt[2] = t < ntask ? (lc >= 2 && lc <= kTaskRange) + (rc >= 2 && rc <= kTaskRange) : 0;
        int ex[3];
        for (int k = 0; k < 3; ++k) {
            int v = cnt[k];
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += y;
            }
            if (lane == 31) wsum[k][warp] = v;
            ex[k] = v - cnt[k];
        }
        __syncthreads();
        if (warp == 0) {
            for (int k = 0; k < 3; ++k) {
                int s = wsum[k][lane];
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, s, o);
                    if (lane >= o) s += y;
                }
                wsum[k][lane] = s;
            }
        }
        __syncthreads();
        for (int k = 0; k < 3; ++k) ex[k] += carry[k] + (warp ? wsum[k][warp - 1] : 0);
        if (t < ntask) {
            const int lid = lc >= 2 ? base_id + ex[0] : n - 1 + tk.begin;
            const int rid = rc >= 2 ? base_id + ex[0] + (lc >= 2) : n - 1 + tk.begin + lc;
            link(nodes, bn, parent, tk.node, lid, rid, n);
            int bi = base_big + ex[1], ki = base_blk + ex[2];
            if (lc > kTaskRange) next[bi++] = Task{tk.begin, tk.begin + lc, lid, tk.depth + 1};
            else if (lc >= 2) blocks[ki++] = Task{tk.begin, tk.begin + lc, lid, tk.depth + 1};
            if (rc > kTaskRange) next[bi] = Task{tk.begin + lc, tk.end, rid, tk.depth + 1};
            else if (rc >= 2) blocks[ki] = Task{tk.begin + lc, tk.end, rid, tk.depth + 1};
        }
        __syncthreads();
        if (threadIdx.x == 1023) {
            for (int k = 0; k < 3; ++k) carry[k] = ex[k] + cnt[k];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        L.counters[3] = base_id + carry[0];
        L.counters[1] = base_big + carry[1];
        L.counters[2] = base_blk + carry[2];
        L.counters[4] = base_big + carry[1];
    }
    // the next level's chunk list, from the tasks this block wrote above
    __syncthreads();
    level_chunks(L, next, base_big + carry[1]);
}

// ---------------------------------------------------------------------------------------
// block tier: one block builds the subtree of one range of <= kBlockRange primitives.
// Centroids and boxes stay at their load index in shared memory; splits permute `perm`
// (position -> load index) only.
// ---------------------------------------------------------------------------------------
struct Piece {
    int begin, count, node, depth, ids;  // ids: first reserved node id (warp pieces)
};

constexpr int kPieceCap = 128;  // block pieces pending (DFS: at most depth + 1)
constexpr int kMediumRange = 256;  // pieces of 33..256 primitives go to one warp each
constexpr int kWarpStack = 16;     // pending pieces > 32 inside one medium piece
constexpr int kMediumCap = kBlockRange / (kWarpRange + 1) + 1;

// Warp-level exact SAH over <= 32 primitives at positions [b, b + c) of the block's range.
// Each primitive stays in the lane that loaded it ("item" = that lane's index).  The items are
// ranked once per axis by centroid (ties by position); ord[a] in lane p is the item at
// position p of the axis-a order.  Every node owns the same position segment [s, s + m) in
// all three orders: its split sweeps each axis order with warp scans (left box of the first
// r + 1 items, right box of the rest) and takes the cheapest plane (lowest axis, then lowest
// plane, on ties; a count split when no plane is allowed by the depth limit), and the three
// orders are then stably partitioned by side, so the children own [s, s + k) and
// [s + k, s + m) again.  Two-item nodes split 1 | 1 without a sweep.  At the end position p
// of the axis-0 order is leaf slot b + p.  `scratch` holds 32 ints of this warp.
// Nodes of at most `small` items (2, or 4 for leaf-size-4 trees) are SAH leaves: no sweep,
// they are split by count (left m / 2 items, in position order) down to single items, so the
// range keeps the one-primitive-per-leaf node format that every other pass reads.
__device__ void warp_build(int* perm, const float4* sc, const float4* slo, const float4* shi,
                           int b, int c, int node, int depth, int next_id, Node* nodes, BNode* bn,
                           int* parent, int n, int gbase, int* scratch, int small) {
    const int lane = threadIdx.x & 31;
    const bool mine = lane < c;
    const int li = perm[b + (mine ? lane : 0)];
    const float4 cc = sc[li], blo = slo[li], bhi = shi[li];
    int ord[3];
    for (int a = 0; a < 3; ++a) {
        const float key = mine ? (a == 0 ? cc.x : (a == 1 ? cc.y : cc.z)) : kInf;
        int rank = 0;
        for (int j = 0; j < c; ++j) {  // c is warp-uniform: only the piece's lanes are ranked
            const float kj = __shfl_sync(0xffffffffu, key, j);
            if (kj < key || (kj == key && j < lane)) ++rank;
        }
        if (mine) scratch[rank] = lane;
        __syncwarp();
        ord[a] = mine ? scratch[lane] : lane;
        __syncwarp();
    }
    int stk_s[kWarpRange], stk_m[kWarpRange], stk_n[kWarpRange], stk_d[kWarpRange];
    stk_s[0] = 0;
    stk_m[0] = c;
    stk_n[0] = node;
    stk_d[0] = depth;
    int top = 1;
    int guard = 0;
    const float3 elo = f3(kInf, kInf, kInf), ehi = f3(-kInf, -kInf, -kInf);
    while (top > 0 && guard++ < 4 * kWarpRange) {
        --top;
        const int s = stk_s[top], m = stk_m[top], rn = stk_n[top], rd = stk_d[top];
        if (m <= small) {
            const int leaf0 = n - 1 + gbase + b + s;
            if (m == 2) {
                if (lane == 0) link(nodes, bn, parent, rn, leaf0, leaf0 + 1, n);
            } else if (m == 3) {
                const int rid = next_id++;
                if (lane == 0) {
                    link(nodes, bn, parent, rn, leaf0, rid, n);
                    link(nodes, bn, parent, rid, leaf0 + 1, leaf0 + 2, n);
                }
            } else {
                const int lid = next_id++;
                const int rid = next_id++;
                if (lane == 0) {
                    link(nodes, bn, parent, rn, lid, rid, n);
                    link(nodes, bn, parent, lid, leaf0, leaf0 + 1, n);
                    link(nodes, bn, parent, rid, leaf0 + 2, leaf0 + 3, n);
                }
            }
            continue;
        }
        float best = kInf;
        int best_axis = -1, best_k = m / 2;
        const int r = lane;
        for (int a = 0; a < 3; ++a) {
            const int it = __shfl_sync(0xffffffffu, ord[a], min(s + r, 31));
            float3 lo = f3(__shfl_sync(0xffffffffu, blo.x, it), __shfl_sync(0xffffffffu, blo.y, it),
                           __shfl_sync(0xffffffffu, blo.z, it));
            float3 hi = f3(__shfl_sync(0xffffffffu, bhi.x, it), __shfl_sync(0xffffffffu, bhi.y, it),
                           __shfl_sync(0xffffffffu, bhi.z, it));
            if (r >= m) {
                lo = elo;
                hi = ehi;
            }
            float3 plo = lo, phi = hi, qlo = lo, qhi = hi;
            // scans over the node's m positions only (lanes >= m hold empty boxes): log2(m) steps
            for (int o = 1; o < m; o <<= 1) {
                const float3 ulo = f3(__shfl_up_sync(0xffffffffu, plo.x, o), __shfl_up_sync(0xffffffffu, plo.y, o), __shfl_up_sync(0xffffffffu, plo.z, o));
                const float3 uhi = f3(__shfl_up_sync(0xffffffffu, phi.x, o), __shfl_up_sync(0xffffffffu, phi.y, o), __shfl_up_sync(0xffffffffu, phi.z, o));
                const float3 dlo = f3(__shfl_down_sync(0xffffffffu, qlo.x, o), __shfl_down_sync(0xffffffffu, qlo.y, o), __shfl_down_sync(0xffffffffu, qlo.z, o));
                const float3 dhi = f3(__shfl_down_sync(0xffffffffu, qhi.x, o), __shfl_down_sync(0xffffffffu, qhi.y, o), __shfl_down_sync(0xffffffffu, qhi.z, o));
                if (lane >= o) {
                    plo = f3(fminf(plo.x, ulo.x), fminf(plo.y, ulo.y), fminf(plo.z, ulo.z));
                    phi = f3(fmaxf(phi.x, uhi.x), fmaxf(phi.y, uhi.y), fmaxf(phi.z, uhi.z));
                }
                if (lane + o < 32) {
                    qlo = f3(fminf(qlo.x, dlo.x), fminf(qlo.y, dlo.y), fminf(qlo.z, dlo.z));
                    qhi = f3(fmaxf(qhi.x, dhi.x), fmaxf(qhi.y, dhi.y), fmaxf(qhi.z, dhi.z));
                }
            }
            // plane after position r: left r + 1 items, right the rest
            const float3 rlo = f3(__shfl_down_sync(0xffffffffu, qlo.x, 1), __shfl_down_sync(0xffffffffu, qlo.y, 1), __shfl_down_sync(0xffffffffu, qlo.z, 1));
            const float3 rhi = f3(__shfl_down_sync(0xffffffffu, qhi.x, 1), __shfl_down_sync(0xffffffffu, qhi.y, 1), __shfl_down_sync(0xffffffffu, qhi.z, 1));
            const int kl = r + 1;
            float cost = kInf;
            if (kl < m && rd + 1 + ceil_log2(max(kl, m - kl)) <= kMaxDepth) {
                cost = half_area(plo, phi) * static_cast<float>(kl) +
                       half_area(rlo, rhi) * static_cast<float>(m - kl);
            }
            float bc = cost;
            int bk = kl;
            int span = 1;  // lanes holding candidates: below m, rounded up to a power of two
            while (span < m) span <<= 1;
            for (int o = span >> 1; o > 0; o >>= 1) {
                const float oc = __shfl_xor_sync(0xffffffffu, bc, o);
                const int ok = __shfl_xor_sync(0xffffffffu, bk, o);
                if (oc < bc || (oc == bc && ok < bk)) {
                    bc = oc;
                    bk = ok;
                }
            }
            // lanes [0, span) hold the winner; every lane takes it from lane 0
            bc = __shfl_sync(0xffffffffu, bc, 0);
            bk = __shfl_sync(0xffffffffu, bk, 0);
            if (bc < best) {
                best = bc;
                best_axis = a;
                best_k = bk;
            }
        }
        const int axis = best_axis < 0 ? 0 : best_axis;
        const int k = best_k;
        // items of the left side (bit per item), then a stable partition of every order
        const int ax_ord = axis == 0 ? ord[0] : (axis == 1 ? ord[1] : ord[2]);
        const int it = __shfl_sync(0xffffffffu, ax_ord, min(s + r, 31));
        const unsigned leftmask = __reduce_or_sync(0xffffffffu, (r < k) ? (1u << it) : 0u);
        const bool inseg = lane >= s && lane < s + m;
        const unsigned segmask = __ballot_sync(0xffffffffu, inseg);
        for (int a = 0; a < 3; ++a) {
            const int item = ord[a];
            const bool left = inseg && ((leftmask >> item) & 1u);
            const unsigned lm = __ballot_sync(0xffffffffu, left);
            const int below = __popc(lm & ((1u << lane) - 1u));
            const int segbelow = __popc(segmask & ((1u << lane) - 1u));  // = lane - s in the segment
            const int pos = left ? s + below : s + k + (segbelow - below);
            if (inseg) scratch[pos] = item;
            __syncwarp();
            if (inseg) ord[a] = scratch[lane];
            __syncwarp();
        }
        const int kr = m - k;
        const int lid = k >= 2 ? next_id++ : n - 1 + gbase + b + s;
        const int rid = kr >= 2 ? next_id++ : n - 1 + gbase + b + s + k;
        if (lane == 0) link(nodes, bn, parent, rn, lid, rid, n);
        if (kr >= 2 && top < kWarpRange) {
            stk_s[top] = s + k;
            stk_m[top] = kr;
            stk_n[top] = rid;
            stk_d[top] = rd + 1;
            ++top;
        }
        if (k >= 2 && top < kWarpRange) {
            stk_s[top] = s;
            stk_m[top] = k;
            stk_n[top] = lid;
            stk_d[top] = rd + 1;
            ++top;
        }
    }
    // leaf order: position p of the axis-0 order
    const int src = __shfl_sync(0xffffffffu, li, ord[0]);
    __syncwarp();
    if (mine) perm[b + lane] = src;
    __syncwarp();
}

// One warp builds the subtree of a medium piece (33..kMediumRange primitives) with the block
// tier's algorithm -- centroid bounds, binned SAH (warp-private bins), stable partition --
// recursing until pieces reach 32, which it finishes with warp_build.  Node ids come from
// the piece's reserved range (root.ids: count - 2 ids) in a fixed order, so the tree does
// not depend on how warps are scheduled.
__device__ void warp_piece_tree(Piece root, int* perm, int* tmp, const float4* sc,
                                const float4* slo, const float4* shi, unsigned* wb, Piece* wstk,
                                int* scratch, int bins, Node* nodes, BNode* bn, int* parent, int n,
                                int gbase, int* err, int small) {
    const int lane = threadIdx.x & 31;
    int next = root.ids;
    if (lane == 0) wstk[0] = root;
    int top = 1;
    __syncwarp();
    int guard = 0;
    while (top > 0 && guard++ < 4 * kMediumRange) {
        const Piece pc = wstk[top - 1];
        --top;
        __syncwarp();
        float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
        for (int i = lane; i < pc.count; i += 32) {
            const float4 c = sc[perm[pc.begin + i]];
            lo[0] = fminf(lo[0], c.x);
            lo[1] = fminf(lo[1], c.y);
            lo[2] = fminf(lo[2], c.z);
            hi[0] = fmaxf(hi[0], c.x);
            hi[1] = fmaxf(hi[1], c.y);
            hi[2] = fmaxf(hi[2], c.z);
        }
        for (int a = 0; a < 3; ++a) {
            for (int o = 16; o > 0; o >>= 1) {
                lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
                hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
            }
        }
        for (int j = lane; j < 3 * bins * kBinWords; j += 32) {
            const int w = j % kBinWords;
            wb[j] = w == 0 ? 0u : (w <= 3 ? ord_f(kInf) : ord_f(-kInf));
        }
        __syncwarp();
        for (int i = lane; i < pc.count; i += 32) {
            const int li = perm[pc.begin + i];
            const float4 c = sc[li], l = slo[li], h = shi[li];
            const float cv[3] = {c.x, c.y, c.z};
            for (int a = 0; a < 3; ++a) {
                unsigned* w = wb + (a * bins + bin_of(cv[a], lo[a], hi[a], bins)) * kBinWords;
                atomicAdd(&w[0], 1u);
                atomicMin(&w[1], ord_f(l.x));
                atomicMin(&w[2], ord_f(l.y));
                atomicMin(&w[3], ord_f(l.z));
                atomicMax(&w[4], ord_f(h.x));
                atomicMax(&w[5], ord_f(h.y));
                atomicMax(&w[6], ord_f(h.z));
            }
        }
        __syncwarp();
        int lc = 0;
        int sp = warp_sweep_bins(wb, bins, pc.count, &lc);
        if (sp >= 0 && pc.depth + 1 + ceil_log2(max(lc, pc.count - lc)) > kMaxDepth) sp = -1;
        if (sp < 0) lc = pc.count / 2;
        // stable partition: left side in position order, then the right side
        int carry = 0;
        for (int base = 0; base < pc.count; base += 32) {
            const int i = base + lane;
            bool f = false;
            if (i < pc.count) {
                if (sp < 0) {
                    f = i < lc;
                } else {
                    const int a = sp >> 8;
                    const float4 c = sc[perm[pc.begin + i]];
                    const float v = a == 0 ? c.x : (a == 1 ? c.y : c.z);
                    f = bin_of(v, lo[a], hi[a], bins) < (sp & 255);
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, f);
            const int lrank = carry + __popc(m & ((1u << lane) - 1u));
            if (i < pc.count) tmp[pc.begin + (f ? lrank : lc + (i - lrank))] = perm[pc.begin + i];
            carry += __popc(m);
        }
        __syncwarp();
        for (int i = lane; i < pc.count; i += 32) perm[pc.begin + i] = tmp[pc.begin + i];
        __syncwarp();
        const int rc = pc.count - lc;
        const int lid = lc >= 2 ? next++ : n - 1 + gbase + pc.begin;
        const int rid = rc >= 2 ? next++ : n - 1 + gbase + pc.begin + lc;
        if (lane == 0) link(nodes, bn, parent, pc.node, lid, rid, n);
        const Piece L = Piece{pc.begin, lc, lid, pc.depth + 1, 0};
        const Piece R = Piece{pc.begin + lc, rc, rid, pc.depth + 1, 0};
        for (int k = 0; k < 2; ++k) {
            const Piece q = k == 0 ? L : R;
            if (q.count >= 2 && q.count <= kWarpRange) {
                warp_build(perm, sc, slo, shi, q.begin, q.count, q.node, q.depth, next, nodes, bn,
                           parent, n, gbase, scratch, small);
                next += q.count - 2;
            }
        }
        for (int k = 0; k < 2; ++k) {
            const Piece q = k == 0 ? R : L;
            if (q.count > kWarpRange) {
                if (top < kWarpStack) {
                    if (lane == 0) wstk[top] = q;
                    ++top;
                } else if (lane == 0) {
                    atomicAdd(err, 1);
                }
            }
        }
        __syncwarp();
    }
    if (top > 0 && lane == 0) atomicAdd(err, 1);
}

__global__ __launch_bounds__(kBlock) void k_block_build(const Task* __restrict__ tasks, int ntask,
                                                       const int* __restrict__ id_base,
                                                       int* __restrict__ order,
                                                       const float4* __restrict__ cen,
                                                       const float4* __restrict__ plo,
                                                       const float4* __restrict__ phi, Node* nodes,
                                                       BNode* bn, int* parent, int n, int bins,
                                                       int* __restrict__ err, int skip_small = 0) {
    extern __shared__ float4 smem[];
    float4* sc = smem;                                      // centroids   [kBlockRange]
    float4* slo = sc + kBlockRange;                         // box lo      [kBlockRange]
    float4* shi = slo + kBlockRange;                        // box hi      [kBlockRange]
    int* perm = reinterpret_cast<int*>(shi + kBlockRange);  // position -> load index
    int* tmp = perm + kBlockRange;                          // partition scratch
    int* sid = tmp + kBlockRange;                           // load index -> scene index
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned* wbins = reinterpret_cast<unsigned*>(sid + kBlockRange) +
                      static_cast<size_t>(warp) * 3 * bins * kBinWords;  // this warp's bins
    Piece* wstk_all = reinterpret_cast<Piece*>(reinterpret_cast<unsigned*>(sid + kBlockRange) +
                                               static_cast<size_t>(kBlock / 32) * 3 * bins * kBinWords);
    Piece* wstk = wstk_all + warp * kWarpStack;
    int* wscratch = reinterpret_cast<int*>(wstk_all + (kBlock / 32) * kWarpStack) + warp * 32;
    __shared__ unsigned sb[3 * kMaxBins * kBinWords];
    __shared__ Piece pieces[kPieceCap];
    __shared__ Piece wpieces[kBlockRange / 2];
    __shared__ Piece mpieces[kMediumCap];
    __shared__ int npieces, nw, nm, next_id, wsum[kBlock / 32];
    __shared__ unsigned sbu[6];
    __shared__ float sbf[6];
    __shared__ int s_split, s_left;

    for (int ti = blockIdx.x; ti < ntask; ti += gridDim.x) {
        const Task tk = tasks[ti];
        const int count = tk.end - tk.begin;
        if (tk.node < 0) continue;  // a forest slot with nothing to build (0 or 1 primitive)
        if (skip_small && count <= kTaskRange) continue;  // built by k_warp_tasks
        if (count < 2 || count > kBlockRange) {
            if (threadIdx.x == 0) atomicAdd(err, 1);
            continue;
        }
        for (int i = threadIdx.x; i < count; i += kBlock) {
            const int p = order[tk.begin + i];
            sid[i] = p;
            perm[i] = i;
            sc[i] = cen[p];
            slo[i] = plo[p];
            shi[i] = phi[p];
        }
        if (threadIdx.x == 0) {
            npieces = 0;
            nw = 0;
            nm = 0;
            next_id = id_base[ti];
            if (count > kMediumRange) {
                pieces[0] = Piece{0, count, tk.node, tk.depth, 0};
                npieces = 1;
            } else if (count > kWarpRange) {
                mpieces[0] = Piece{0, count, tk.node, tk.depth, id_base[ti]};
                nm = 1;
            } else {
                wpieces[0] = Piece{0, count, tk.node, tk.depth, id_base[ti]};
                nw = 1;
            }
        }
        __syncthreads();
        int guard = 0;
        while (npieces > 0 && guard++ < 2 * kBlockRange) {
            const Piece pc = pieces[npieces - 1];
            // centroid bounds of the piece
            float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
            for (int i = threadIdx.x; i < pc.count; i += kBlock) {
                const float4 c = sc[perm[pc.begin + i]];
                lo[0] = fminf(lo[0], c.x);
                lo[1] = fminf(lo[1], c.y);
                lo[2] = fminf(lo[2], c.z);
                hi[0] = fmaxf(hi[0], c.x);
                hi[1] = fmaxf(hi[1], c.y);
                hi[2] = fmaxf(hi[2], c.z);
            }
            for (int a = 0; a < 3; ++a) {
                for (int o = 16; o > 0; o >>= 1) {
                    lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
                    hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
                }
            }
            for (int j = threadIdx.x; j < 3 * bins * kBinWords; j += kBlock) {
                const int w = j % kBinWords;
                sb[j] = w == 0 ? 0u : (w <= 3 ? ord_f(kInf) : ord_f(-kInf));
            }
            if (threadIdx.x < 6) sbu[threadIdx.x] = threadIdx.x < 3 ? ord_f(kInf) : ord_f(-kInf);
            __syncthreads();
            if (threadIdx.x == 0) --npieces;
            if (lane == 0) {
                for (int a = 0; a < 3; ++a) {
                    atomicMin(&sbu[a], ord_f(lo[a]));
                    atomicMax(&sbu[3 + a], ord_f(hi[a]));
                }
            }
            __syncthreads();
            float cbl[3], cbh[3];
            for (int a = 0; a < 3; ++a) {
                cbl[a] = unord_f(sbu[a]);
                cbh[a] = unord_f(sbu[3 + a]);
            }
            for (int i = threadIdx.x; i < pc.count; i += kBlock) {
                const int li = perm[pc.begin + i];
                const float4 c = sc[li], l = slo[li], h = shi[li];
                const float cv[3] = {c.x, c.y, c.z};
                for (int a = 0; a < 3; ++a) {
                    unsigned* w = sb + (a * bins + bin_of(cv[a], cbl[a], cbh[a], bins)) * kBinWords;
                    atomicAdd(&w[0], 1u);
                    atomicMin(&w[1], ord_f(l.x));
                    atomicMin(&w[2], ord_f(l.y));
                    atomicMin(&w[3], ord_f(l.z));
                    atomicMax(&w[4], ord_f(h.x));
                    atomicMax(&w[5], ord_f(h.y));
                    atomicMax(&w[6], ord_f(h.z));
                }
            }
            __syncthreads();
            if (warp == 0) {
                int lc = 0;
                int sp = warp_sweep_bins(sb, bins, pc.count, &lc);
                if (sp >= 0 && pc.depth + 1 + ceil_log2(max(lc, pc.count - lc)) > kMaxDepth) sp = -1;
                if (sp < 0) lc = pc.count / 2;
                if (lane == 0) {
                    s_split = sp;
                    s_left = lc;
                    for (int a = 0; a < 3; ++a) {
                        sbf[a] = cbl[a];
                        sbf[3 + a] = cbh[a];
                    }
                }
            }
            __syncthreads();
            const int split = s_split, lc = s_left;
            // stable partition: destination of every position into tmp
            int carry = 0;
            for (int base = 0; base < pc.count; base += kBlock) {
                const int i = base + threadIdx.x;
                int f = 0;
                if (i < pc.count) {
                    if (split < 0) {
                        f = i < lc;
                    } else {
                        const int a = split >> 8;
                        const float4 c = sc[perm[pc.begin + i]];
                        const float v = a == 0 ? c.x : (a == 1 ? c.y : c.z);
                        f = bin_of(v, sbf[a], sbf[3 + a], bins) < (split & 255);
                    }
                }
                int v = f;
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, v, o);
                    if (lane >= o) v += y;
                }
                if (lane == 31) wsum[warp] = v;
                __syncthreads();
                int wpre = 0, tot = 0;
                for (int w = 0; w < kBlock / 32; ++w) {
                    if (w < warp) wpre += wsum[w];
                    tot += wsum[w];
                }
                const int lrank = carry + wpre + v - f;
                if (i < pc.count) tmp[pc.begin + (f ? lrank : lc + (i - lrank))] = perm[pc.begin + i];
                __syncthreads();
                carry += tot;
            }
            for (int i = threadIdx.x; i < pc.count; i += kBlock) perm[pc.begin + i] = tmp[pc.begin + i];
            if (threadIdx.x == 0) {
                const int rc = pc.count - lc;
                const int lid = lc >= 2 ? next_id++ : n - 1 + tk.begin + pc.begin;
                const int rid = rc >= 2 ? next_id++ : n - 1 + tk.begin + pc.begin + lc;
                link(nodes, bn, parent, pc.node, lid, rid, n);
                const Piece L = Piece{pc.begin, lc, lid, pc.depth + 1, 0};
                const Piece R = Piece{pc.begin + lc, rc, rid, pc.depth + 1, 0};
                for (int k = 0; k < 2; ++k) {
                    Piece q = k == 0 ? R : L;
                    if (q.count > kMediumRange) {
                        if (npieces < kPieceCap) pieces[npieces++] = q;
                        else atomicAdd(err, 1);
                    } else if (q.count > kWarpRange) {
                        q.ids = next_id;
                        next_id += q.count - 2;
                        if (nm < kMediumCap) mpieces[nm++] = q;
                        else atomicAdd(err, 1);
                    } else if (q.count >= 2) {
                        q.ids = next_id;
                        next_id += q.count - 2;
                        if (nw < kBlockRange / 2) wpieces[nw++] = q;
                        else atomicAdd(err, 1);
                    }
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0 && npieces > 0) atomicAdd(err, 1);
        __syncthreads();
        const int total_m = nm;
        for (int m = warp; m < total_m; m += kBlock / 32)
            warp_piece_tree(mpieces[m], perm, tmp, sc, slo, shi, wbins, wstk, wscratch, bins,
                            nodes, bn, parent, n, tk.begin, err, 2);
        __syncthreads();
        const int total_w = nw;
        for (int w = warp; w < total_w; w += kBlock / 32) {
            const Piece q = wpieces[w];
            warp_build(perm, sc, slo, shi, q.begin, q.count, q.node, q.depth, q.ids, nodes, bn,
                       parent, n, tk.begin, wscratch, 2);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < count; i += kBlock) order[tk.begin + i] = sid[perm[i]];
        __syncthreads();
    }
}

// Tasks of 2..kTaskRange primitives, one warp each, over global arrays: `order` maps positions
// to primitive indices (cen / plo / phi), `tmp` is partition scratch of the same size.  A task
// of up to 32 goes straight to warp_build, a larger one through warp_piece_tree; node ids come
// from the task's reserved range, so the tree does not depend on scheduling.  No block-wide
// barriers: each warp works on its own task.  A task of more than kTaskRange primitives is an
// error unless `large_ok` says that the block builder (k_block_build) takes those tasks after
// this launch (the forest of a topology edit, whose cuts grow by the primitives they receive).
__global__ __launch_bounds__(kBlock, 4) void k_warp_tasks(const Task* __restrict__ tasks, int ntask,
                                                      const int* __restrict__ id_base,
                                                      int* __restrict__ order, int* __restrict__ tmp,
                                                      const float4* __restrict__ cen,
                                                      const float4* __restrict__ plo,
                                                      const float4* __restrict__ phi, Node* nodes,
                                                      BNode* bn, int* parent, int n, int bins,
                                                      int* __restrict__ err, int large_ok,
                                                      int small, int* __restrict__ fetch) {
    extern __shared__ unsigned wsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned* wb = wsm + static_cast<size_t>(warp) * 3 * bins * kBinWords;
    Piece* wstk_all = reinterpret_cast<Piece*>(wsm + static_cast<size_t>(kBlock / 32) * 3 * bins * kBinWords);
    Piece* wstk = wstk_all + warp * kWarpStack;
    int* scratch = reinterpret_cast<int*>(wstk_all + (kBlock / 32) * kWarpStack) + warp * 32;
    const int w = (blockIdx.x * kBlock + threadIdx.x) >> 5;
    const int nw = (gridDim.x * kBlock) >> 5;
    // with `fetch` (a zeroed counter) each warp takes its next task from it, so warps that drew
    // small ranges take more of them; without, warp w takes tasks w, w + nw, ...
    for (int ti = w;; ti += nw) {
        if (fetch) {
            int next = 0;
            if (lane == 0) next = atomicAdd(fetch, 1);
            ti = __shfl_sync(0xffffffffu, next, 0);
        }
        if (ti >= ntask) break;
        const Task tk = tasks[ti];
        const int count = tk.end - tk.begin;
        if (tk.node < 0 || count < 2 || count > kTaskRange) {
            if (tk.node >= 0 && count > kTaskRange && !large_ok && lane == 0) atomicAdd(err, 1);
            continue;
        }
        if (count <= kWarpRange) {
            warp_build(order, cen, plo, phi, tk.begin, count, tk.node, tk.depth, id_base[ti], nodes,
                       bn, parent, n, 0, scratch, small);
        } else {
            warp_piece_tree(Piece{tk.begin, count, tk.node, tk.depth, id_base[ti]}, order, tmp, cen,
                            plo, phi, wb, wstk, scratch, bins, nodes, bn, parent, n, 0, err, small);
        }
    }
}

// dynamic shared memory of k_warp_tasks: every warp's bins, piece stack and scratch
size_t warp_tasks_smem(int bins) {
    return static_cast<size_t>(kBlock / 32) *
           (3 * static_cast<size_t>(bins) * kBinWords * sizeof(unsigned) + kWarpStack * sizeof(Piece) +
            32 * sizeof(int));
}

constexpr size_t kBlockSmemBase = 3 * kBlockRange * sizeof(float4) + 3 * kBlockRange * sizeof(int);

// dynamic shared memory of k_block_build: the range arrays plus every warp's bins and stack
size_t block_smem(int bins) {
    return kBlockSmemBase + static_cast<size_t>(kBlock / 32) *
                                (3 * static_cast<size_t>(bins) * kBinWords * sizeof(unsigned) +
                                 kWarpStack * sizeof(Piece) + 32 * sizeof(int));
}

// leaves of the final order: sorted items, ids, inverse map, canonical leaf nodes, payload
template <class Ops>
__global__ __launch_bounds__(kBlock) void k_sah_leaves(const float* __restrict__ items, int n,
                                                      const int* __restrict__ order,
                                                      Node* __restrict__ nodes,
                                                      float* __restrict__ sorted,
                                                      int* __restrict__ prim_ids,
                                                      int* __restrict__ slot_of,
                                                      float4* __restrict__ leaves) {
    // the LBVH emit's leaf writer (per-warp staging for triangles and Gaussians)
    __shared__ __align__(16) float stage[kBlock / 32][emit_stage_floats<Ops>()];
    const int k0 = blockIdx.x * kBlock + (threadIdx.x & ~31);
    if (k0 >= n) return;  // whole warps
    emit_leaves_warp<Ops>(items, n, reinterpret_cast<const uint32_t*>(order), nodes, sorted,
                          prim_ids, slot_of, leaves, k0, min(32, n - k0), stage[threadIdx.x >> 5]);
}

__global__ void k_task_sizes(const Task* __restrict__ t, int m, int* __restrict__ out) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < m) out[i] = t[i].end - t[i].begin - 2;
}

__global__ void k_add_base(int* __restrict__ v, int m, const int* __restrict__ base) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < m) v[i] += base[3];
}

struct SahWs {
    Header* h;
    int* orderA;
    int* orderB;
    int* orderF;  // final order: each primitive's position once its range leaves the global tier
    float4* cen;
    float4* plo;
    float4* phi;
    Task* tasksA;
    Task* tasksB;
    Task* blocks;
    int* id_base;
    void* scan_ws;
    Level L;
};

SahWs carve_sah(Carve& c, int n) {
    const int max_big = n / (kTaskRange + 1) + 2;
    const int max_chunks = n / kChunk + max_big + 2;
    const int max_blocks = n / 2 + 2;
    SahWs w;
    w.h = c.take<Header>(1);
    w.orderA = c.take<int>(n);
    w.orderB = c.take<int>(n);
    w.orderF = c.take<int>(n);
    w.cen = c.take<float4>(n);
    w.plo = c.take<float4>(n);
    w.phi = c.take<float4>(n);
    w.tasksA = c.take<Task>(max_big);
    w.tasksB = c.take<Task>(max_big);
    w.blocks = c.take<Task>(max_blocks);
    w.id_base = c.take<int>(max_blocks + 1);
    w.scan_ws = c.take<char>(scan_ws_bytes(max_blocks));
    w.L.tasks = w.tasksA;
    w.L.chunk_task = c.take<int>(max_chunks);
    w.L.chunk_begin = c.take<int>(max_chunks);
    w.L.chunk_first = c.take<int>(max_big);
    w.L.cb = c.take<unsigned>(6 * static_cast<size_t>(max_big));
    w.L.bins = c.take<unsigned>(static_cast<size_t>(max_big) * 3 * kMaxBins * kBinWords);
    w.L.split = c.take<int>(max_big);
    w.L.left_count = c.take<int>(max_big);
    w.L.chunk_left = c.take<int>(max_chunks);
    w.L.counters = c.take<int>(8);
    return w;
}

template <class Ops>
int build_sah_impl(qk_tree* t, int bins, int small, const void* items_v, void* ws,
                   cudaStream_t s) {
    const int n = t->n;
    const float* items = static_cast<const float*>(items_v);
    Carve c{static_cast<char*>(ws)};
    SahWs w = carve_sah(c, n);
    Node* nodes = static_cast<Node*>(t->nodes);
    BNode* bn = static_cast<BNode*>(t->bnodes);
    int* err = &w.h->error;
    cudaMemsetAsync(w.h, 0, sizeof(Header), s);
    cudaMemsetAsync(t->parent, 0xff, sizeof(int) * (2 * static_cast<size_t>(n) - 1), s);
    k_prim_geom<Ops><<<blocks_for(n), kBlock, 0, s>>>(items, n, w.cen, w.plo, w.phi, w.orderA);

    // counters: [1] next big tasks, [2] block tasks, [3] next internal id, [4] this level's
    // big tasks
    int init[8] = {0, 0, 0, 1, 0, 0, 0, 0};
    Task root{0, n, 0, 0};
    int nbig = 0, nblk = 0;
    if (n > kTaskRange) {
        cudaMemcpyAsync(w.tasksA, &root, sizeof(Task), cudaMemcpyHostToDevice, s);
        nbig = 1;
    } else {
        cudaMemcpyAsync(w.blocks, &root, sizeof(Task), cudaMemcpyHostToDevice, s);
        init[2] = 1;
        nblk = 1;
    }
    init[4] = nbig;
    cudaMemcpyAsync(w.L.counters, init, sizeof(init), cudaMemcpyHostToDevice, s);
    Task* cur = w.tasksA;
    Task* nxt = w.tasksB;
    int* ord = w.orderA;
    int* alt = w.orderB;
    int level = 0;
    // Levels run in batches between host read-backs of the counters: every level kernel reads
    // its task count from counters[4] and the grids are sized by a bound (a level has at most
    // twice the previous level's tasks, and at most n / (kTaskRange + 1)); a level after the
    // last one has no tasks and every kernel of it returns at once.  With a StageClock
    // installed every level is read back, so that its stage times are its own.
    StageClock* clk = stage_clock();
    const int per_sync = clk ? 1 : kLevelsPerSync;
    const int max_big = n / (kTaskRange + 1) + 1;
    // the first level's chunk list; each level's k_level_assign writes the next one's
    if (nbig > 0) k_level_prep<<<1, 1024, 0, s>>>(w.L);
    while (nbig > 0) {
        if (level >= kMaxDepth) return fail(QK_ERR_DEPTH, "SAH: too many levels");
        int bound = nbig;
        const int batch = std::min(per_sync, kMaxDepth - level);
        cudaError_t e;
        for (int j = 0; j < batch; ++j, ++level) {
            w.L.tasks = cur;
            k_level_reset<<<bound, kBlock, 0, s>>>(w.L, bins);
            // chunk kernels: grid sized by a bound on the chunk count (every task spans at most
            // size / kChunk + 1 chunks); blocks beyond the count k_level_prep wrote return at once
            const int nch = n / kChunk + bound + 1;
            // per-level stage times when a StageClock is installed: binning (centroid bounds +
            // bins), split selection, partition (+ child assignment)
            if (clk) cudaEventRecord(clk->lv[0], s);
            k_level_cbounds<<<nch, kBlock, 0, s>>>(w.L, ord, w.cen);
            k_level_bins<<<nch, kBlock, 0, s>>>(w.L, ord, w.cen, w.plo, w.phi, bins);
            if (clk) cudaEventRecord(clk->lv[1], s);
            k_level_split<<<blocks_for(static_cast<long long>(bound) * 32), kBlock, 0, s>>>(w.L, bins);
            if (clk) cudaEventRecord(clk->lv[2], s);
            k_level_count_left<<<nch, kBlock, 0, s>>>(w.L, ord, w.cen, bins);
            k_level_partition<<<nch, kBlock, 0, s>>>(w.L, ord, alt, w.orderF, w.cen, bins);
            // next big tasks start from zero each level; block tasks accumulate
            cudaMemsetAsync(w.L.counters + 1, 0, sizeof(int), s);
            k_level_assign<<<1, 1024, 0, s>>>(w.L, nxt, w.blocks, nodes, bn, t->parent, n);
            if (clk) cudaEventRecord(clk->lv[3], s);
            Task* tmpt = cur;
            cur = nxt;
            nxt = tmpt;
            int* tmpo = ord;  // the next level reads what this one partitioned
            ord = alt;
            alt = tmpo;
            bound = std::min(2 * bound, max_big);
        }
        int cnt[4] = {0, 0, 0, 0};
        e = cudaMemcpyAsync(cnt, w.L.counters, sizeof(cnt), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "SAH level");
        if (clk) {
            float a = 0.f, b = 0.f, c3 = 0.f;
            if (cudaEventElapsedTime(&a, clk->lv[0], clk->lv[1]) == cudaSuccess &&
                cudaEventElapsedTime(&b, clk->lv[1], clk->lv[2]) == cudaSuccess &&
                cudaEventElapsedTime(&c3, clk->lv[2], clk->lv[3]) == cudaSuccess) {
                clk->sah_bin += a;
                clk->sah_split += b;
                clk->sah_part += c3;
            }
        }
        nbig = cnt[1];
        nblk = cnt[2];
    }
    // the final order: written by the partitions, or the initial order when the root went
    // straight to the warp tier; either order buffer is then free scratch
    int* fin = n > kTaskRange ? w.orderF : w.orderA;
    int* scratch = n > kTaskRange ? w.orderA : w.orderB;
    if (nblk > 0) {
        // reserved ids for the block subtrees: base + exclusive sum of (count - 2)
        k_task_sizes<<<blocks_for(nblk), kBlock, 0, s>>>(w.blocks, nblk, w.id_base);
        cudaError_t e = scan_exclusive(w.id_base, w.id_base, nblk, true, w.scan_ws, s);
        if (e != cudaSuccess) return cuda_status(e, "SAH id scan");
        int tail[2] = {0, 0};
        e = cudaMemcpyAsync(&tail[0], w.id_base + nblk, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&tail[1], w.L.counters + 3, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "SAH id readback");
        if (tail[1] + tail[0] != n - 1) {
            return fail(QK_ERR_INVALID, "SAH node accounting: %d + %d != %d", tail[1], tail[0], n - 1);
        }
        k_add_base<<<blocks_for(nblk), kBlock, 0, s>>>(w.id_base, nblk, w.L.counters);
        // every range of at most kTaskRange primitives: one warp each
        // a resident grid (4 blocks per SM) whose warps fetch tasks from counters[5]
        k_warp_tasks<<<min(blocks_for(static_cast<long long>(nblk) * 32), 148 * 4), kBlock,
                       warp_tasks_smem(bins), s>>>(w.blocks, nblk, w.id_base, fin, scratch, w.cen,
                                                   w.plo, w.phi, nodes, bn, t->parent, n, bins, err,
                                                   0, small, w.L.counters + 5);
    } else {
        int base = 0;
        cudaMemcpyAsync(&base, w.L.counters + 3, sizeof(int), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        if (base != n - 1) return fail(QK_ERR_INVALID, "SAH node accounting: %d != %d", base, n - 1);
    }
    stage_mark(kMarkTopo, s);
    // the scatter: items, leaf payloads and prim ids in leaf order
    k_sah_leaves<Ops><<<blocks_for(n), kBlock, 0, s>>>(items, n, fin, nodes,
                                                       static_cast<float*>(t->items), t->prim_ids,
                                                       t->slot_of, static_cast<float4*>(t->leaves));
    stage_mark(kMarkScatter, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "SAH kernels");
    int errors = 0;
    e = cudaMemcpyAsync(&errors, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "SAH readback");
    if (errors) return fail(QK_ERR_OVERFLOW, "SAH block builder reported %d errors", errors);
    return QK_OK;
}

}  // namespace

size_t sah_ws_bytes(int n) {
    Carve c;
    carve_sah(c, n);
    return c.used;
}

int sah_forest(const int4* tasks, int ntask, int max_count, const int* id_base, int* order,
               int* tmp, const float4* cen, const float4* plo, const float4* phi, qk_tree* t,
               int bins, int* err, cudaStream_t s) {
    static_assert(sizeof(Task) == sizeof(int4), "forest tasks are {begin, end, node, depth}");
    if (bins < 4 || bins > kMaxBins) return fail(QK_ERR_INVALID, "sah_bins must be in [4, 64]");
    if (ntask <= 0) return QK_OK;
    const Task* tk = reinterpret_cast<const Task*>(tasks);
    Node* nodes = static_cast<Node*>(t->nodes);
    BNode* bn = static_cast<BNode*>(t->bnodes);
    k_warp_tasks<<<min(blocks_for(static_cast<long long>(ntask) * 32), 148 * 8), kBlock,
                   warp_tasks_smem(bins), s>>>(tk, ntask, id_base, order, tmp, cen, plo, phi, nodes,
                                               bn, t->parent, t->n, bins, err,
                                               max_count > kTaskRange ? 1 : 0, 2, nullptr);
    if (max_count > kTaskRange) {
        cudaFuncSetAttribute(k_block_build, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(block_smem(kMaxBins)));
        k_block_build<<<min(ntask, 148 * 4), kBlock, block_smem(bins), s>>>(
            tk, ntask, id_base, order, cen, plo, phi, nodes, bn, t->parent, t->n, bins, err, 1);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "SAH forest");
}

int build_sah(qk_tree* t, int bins, int leaf_size, const void* items, void* ws, cudaStream_t s) {
    if (bins < 4 || bins > kMaxBins) return fail(QK_ERR_INVALID, "sah_bins must be in [4, 64]");
    if (leaf_size != 1 && leaf_size != 4) return fail(QK_ERR_INVALID, "SAH leaf size must be 1 or 4");
    const int small = leaf_size == 4 ? 4 : 2;  // nodes of at most `small` primitives are not swept
    switch (t->kind) {
        case kTri: return build_sah_impl<TriOps>(t, bins, small, items, ws, s);
        case kPoint: return build_sah_impl<PointOps>(t, bins, small, items, ws, s);
        case kGauss: return build_sah_impl<GaussOps>(t, bins, small, items, ws, s);
        default: return fail(QK_ERR_INVALID, "unknown primitive kind %d", t->kind);
    }
}

}  // namespace qk
