// qk_sort.cu -- stable LSD radix sort of (uint32 key, uint32 value) pairs and an exclusive
// int scan, written for the engine's build (Morton codes) and query reordering.
//
// Radix sort: 8-bit digits, one pass per digit, three kernels per pass:
//   upsweep    one block per 4096-key tile counts its digits (warp-private histograms in
//              shared memory) and writes hist[digit * tiles + tile]
//   scan       exclusive scan of hist (digit-major), so every (digit, tile) pair knows where
//              its run starts in the output
//   downsweep  each warp ranks its 512 keys in input order: __match_any_sync groups lanes
//              holding the same digit, the rank inside a round is the popcount of lower
//              peers, and a per-warp running count carries ranks across rounds; warps are
//              then offset by an exclusive prefix over the per-warp counts.  The tile is
//              laid out in digit order in shared memory, and consecutive threads write
//              consecutive slots of each digit's run (coalesced stores).  Equal digits keep
//              their input order, so the sort is stable.
// Stability makes sorting (morton, index) pairs on the 30 Morton bits alone equal to the
// reference's full 64-bit sort of (morton << 32 | index) keys (src/gpu/lbvh.cu:1995-2003).
#include "qk_internal.cuh"

namespace qk {

namespace {

constexpr int kRadix = 256;
constexpr int kWarps = kBlock / 32;
constexpr int kItems = kSortTile / kBlock;  // 16 keys per thread
static_assert(kItems * kBlock == kSortTile, "tile size");

// ---- warp and block scans (the sort's digit runs and the exclusive scan below) ----
__device__ __forceinline__ int warp_incl_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

// Exclusive block scan of one value per thread; returns the block total in *total.
__device__ __forceinline__ int block_excl_scan(int v, int* total) {
    __shared__ int ws[kBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int inc = warp_incl_scan(v);
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int s = lane < kBlock / 32 ? ws[lane] : 0;
        s = warp_incl_scan(s);
        if (lane < kBlock / 32) ws[lane] = s;
    }
    __syncthreads();
    const int wprefix = warp > 0 ? ws[warp - 1] : 0;
    *total = ws[kBlock / 32 - 1];
    __syncthreads();
    return wprefix + inc - v;
}

__global__ __launch_bounds__(kBlock) void k_rs_upsweep(const uint32_t* __restrict__ keys, int n,
                                                       int shift, uint32_t* __restrict__ hist,
                                                       int tiles) {
    __shared__ uint32_t wh[kWarps][kRadix];
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kBlock) (&wh[0][0])[i] = 0;
    __syncthreads();
    const int tile = blockIdx.x;
    const int base = tile * kSortTile;
#pragma unroll 4
    for (int j = 0; j < kItems; ++j) {
        const int idx = base + j * kBlock + threadIdx.x;
        if (idx < n) atomicAdd(&wh[warp][(keys[idx] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kBlock) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s += wh[w][d];
        hist[static_cast<size_t>(d) * tiles + tile] = s;
    }
}

__global__ __launch_bounds__(kBlock) void k_rs_downsweep(
    const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    uint32_t* __restrict__ vout, int n, int shift, const uint32_t* __restrict__ hist, int tiles) {
    __shared__ uint32_t wcount[kWarps][kRadix];
    __shared__ uint32_t gbase[kRadix];
    __shared__ uint32_t lstart[kRadix];
    __shared__ uint32_t skey[kSortTile];
    __shared__ uint32_t sval[kSortTile];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kBlock) (&wcount[0][0])[i] = 0;
    const int tile = blockIdx.x;
    for (int d = threadIdx.x; d < kRadix; d += kBlock) {
        gbase[d] = hist[static_cast<size_t>(d) * tiles + tile];
    }
    __syncthreads();

    const int wbase = tile * kSortTile + warp * (kSortTile / kWarps);
    const unsigned lower = (1u << lane) - 1u;
    uint32_t key[kItems], val[kItems];
    uint16_t rank[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int idx = wbase + j * 32 + lane;
        const bool ok = idx < n;
        key[j] = ok ? kin[idx] : 0u;
        val[j] = ok ? vin[idx] : 0u;
        const uint32_t d = ok ? ((key[j] >> shift) & 0xffu) : 0x100u;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = ok ? wcount[warp][d] : 0u;
        __syncwarp();
        if (ok && lane == __ffs(peers) - 1) wcount[warp][d] = before + __popc(peers);
        __syncwarp();
        rank[j] = static_cast<uint16_t>(before + __popc(peers & lower));
    }
    __syncthreads();
    // per digit: the tile's count, its run's start inside the tile (a block scan over the
    // digits) and every warp's offset inside that run
    static_assert(kRadix == kBlock, "one thread per digit");
    {
        const int d = threadIdx.x;
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = wcount[w][d];
            wcount[w][d] = run;
            run += c;
        }
        int total;
        lstart[d] = static_cast<uint32_t>(block_excl_scan(static_cast<int>(run), &total));
    }
    __syncthreads();
    // the tile in digit order in shared memory (stable: warps, then items, then lanes)
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int idx = wbase + j * 32 + lane;
        if (idx < n) {
            const uint32_t d = (key[j] >> shift) & 0xffu;
            const uint32_t at = lstart[d] + wcount[warp][d] + rank[j];
            skey[at] = key[j];
            sval[at] = val[j];
        }
    }
    __syncthreads();
    // consecutive threads write consecutive slots of one digit's run
    const int m = min(kSortTile, n - tile * kSortTile);
#pragma unroll 4
    for (int i = threadIdx.x; i < m; i += kBlock) {
        const uint32_t k = skey[i];
        const uint32_t d = (k >> shift) & 0xffu;
        const uint32_t dst = gbase[d] + (static_cast<uint32_t>(i) - lstart[d]);
        kout[dst] = k;
        vout[dst] = sval[i];
    }
}

// ---- exclusive scan: block-local scans, a scan of the block sums, then a fix-up ----
// in and out may alias: each thread reads its own four elements before any write
__global__ __launch_bounds__(kBlock) void k_scan_blocks(const int* in, int* out, int n,
                                                        int* __restrict__ sums) {
    const int base = blockIdx.x * kScanBlock + threadIdx.x * 4;
    int v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = base + j < n ? in[base + j] : 0;
    const int tsum = v[0] + v[1] + v[2] + v[3];
    int total;
    int run = block_excl_scan(tsum, &total);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (base + j < n) out[base + j] = run;
        run += v[j];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// single block: exclusive scan of the block sums in place, total to *total_out
__global__ __launch_bounds__(kBlock) void k_scan_sums(int* __restrict__ sums, int nb,
                                                      int* __restrict__ total_out) {
    int carry = 0;
    for (int base = 0; base < nb; base += kBlock) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? sums[i] : 0;
        int total;
        const int ex = block_excl_scan(v, &total);
        if (i < nb) sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0 && total_out) *total_out = carry;
}

__global__ __launch_bounds__(kBlock) void k_scan_add(int* __restrict__ out, int n,
                                                     const int* __restrict__ sums) {
    const int b = blockIdx.x;
    if (b == 0) return;
    const int add = sums[b];
    const int base = b * kScanBlock + threadIdx.x * 4;
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (base + j < n) out[base + j] += add;
}

}  // namespace

size_t scan_ws_bytes(int n) {
    return (static_cast<size_t>(blocks_for(n, kScanBlock)) + 1) * sizeof(int) + 256;
}

cudaError_t scan_exclusive(const int* in, int* out, int n, bool write_total, void* ws,
                           cudaStream_t s) {
    if (n <= 0) {
        if (write_total) return cudaMemsetAsync(out, 0, sizeof(int), s);
        return cudaSuccess;
    }
    const int nb = blocks_for(n, kScanBlock);
    int* sums = static_cast<int*>(ws);
    k_scan_blocks<<<nb, kBlock, 0, s>>>(in, out, n, sums);
    k_scan_sums<<<1, kBlock, 0, s>>>(sums, nb, write_total ? out + n : nullptr);
    if (nb > 1) k_scan_add<<<nb, kBlock, 0, s>>>(out, n, sums);
    return cudaGetLastError();
}

size_t sort_ws_bytes(int n) {
    const int tiles = blocks_for(n, kSortTile);
    const size_t hist = static_cast<size_t>(kRadix) * tiles;
    Carve c;
    c.take<uint32_t>(hist);
    c.take<char>(scan_ws_bytes(static_cast<int>(hist)));
    return c.used;
}

// Sorts (kin, vin) by the low `bits` bits into (kout, vout).  Passes ping-pong between the
// output pair and the input pair (pass p writes the output pair when p is even), so kin /
// vin are clobbered when more than one pass runs; an even pass count ends with one copy.
cudaError_t sort_pairs(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout,
                       int n, int bits, void* ws, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int tiles = blocks_for(n, kSortTile);
    const size_t hlen = static_cast<size_t>(kRadix) * tiles;
    Carve c{static_cast<char*>(ws)};
    uint32_t* hist = c.take<uint32_t>(hlen);
    void* scan_ws = c.take<char>(scan_ws_bytes(static_cast<int>(hlen)));
    const int passes = bits <= 0 ? 1 : (bits + 7) / 8;
    const uint32_t* sk = kin;
    const uint32_t* sv = vin;
    for (int p = 0; p < passes; ++p) {
        uint32_t* dk = (p % 2 == 0) ? kout : const_cast<uint32_t*>(kin);
        uint32_t* dv = (p % 2 == 0) ? vout : const_cast<uint32_t*>(vin);
        k_rs_upsweep<<<tiles, kBlock, 0, s>>>(sk, n, 8 * p, hist, tiles);
        const cudaError_t e = scan_exclusive(reinterpret_cast<const int*>(hist),
                                             reinterpret_cast<int*>(hist), static_cast<int>(hlen),
                                             false, scan_ws, s);
        if (e != cudaSuccess) return e;
        k_rs_downsweep<<<tiles, kBlock, 0, s>>>(sk, sv, dk, dv, n, 8 * p, hist, tiles);
        sk = dk;
        sv = dv;
    }
    if (sk != kout) {
        cudaMemcpyAsync(kout, sk, sizeof(uint32_t) * static_cast<size_t>(n),
                        cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(vout, sv, sizeof(uint32_t) * static_cast<size_t>(n),
                        cudaMemcpyDeviceToDevice, s);
    }
    return cudaGetLastError();
}

}  // namespace qk
