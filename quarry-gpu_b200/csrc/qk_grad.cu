// qk_grad.cu -- adjoints of the spatial queries (the differentiable-query layer; quarry has
// no backward pass, so nothing here mirrors a reference function).
//
// The forward pass picks a primitive discretely (closest / first hit); the backward
// differentiates only that primitive's leaf test, recomputing it in FP64 from the inputs
// instead of storing any traversal state:
//   triangle distance   d = |p - q|, q the Ericson closest point with barycentrics
//                       (w_a, w_b, w_c); by the envelope theorem dd/dp = n, dd/da = -w_a n,
//                       dd/db = -w_b n, dd/dc = -w_c n with n = (p - q) / d
//   ellipsoid distance  d = |y - x| in the ellipsoid frame (y = R^T (p - m), x the closest
//                       surface point from Eberly's secular equation solved to FP64
//                       precision); dd/dp = R n_l, dd/dm = -R n_l, dd/ds_i = -n_l,i x_i / s_i,
//                       dd/d(axis j) = n_l,j (p - m), then through the quaternion
//                       normalisation to dd/dq
//   ray hit t           t = n.(a - o) / n.d for the hit triangle; dt/da = w_a n / (n.d),
//                       dt/db = u n / (n.d), dt/dc = v n / (n.d), dt/do = -n / (n.d),
//                       dt/dd = -t n / (n.d)
// Inside a solid ellipsoid or on a triangle (d = 0) the gradient is taken as 0.
// Per-primitive sums are deterministic: contributions are written per query, stably sorted
// by primitive index, and each primitive sums its run in query order (no float atomics).
#include "qk_internal.cuh"

namespace qk {

namespace {

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 d3(double x, double y, double z) { return D3{x, y, z}; }
__device__ __forceinline__ D3 dsub(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ D3 dadd(D3 a, D3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ D3 dmul(D3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 dcross(D3 a, D3 b) {
    return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ D3 ld3(const float* p) { return d3(p[0], p[1], p[2]); }

// Ericson closest point in FP64; returns q and the barycentrics of b and c.
__device__ D3 closest_tri_fp64(D3 p, D3 a, D3 b, D3 c, double& wb, double& wc) {
    const D3 ab = dsub(b, a), ac = dsub(c, a), ap = dsub(p, a);
    const double d1 = ddot(ab, ap), d2 = ddot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { wb = 0; wc = 0; return a; }
    const D3 bp = dsub(p, b);
    const double d3_ = ddot(ab, bp), d4 = ddot(ac, bp);
    if (d3_ >= 0.0 && d4 <= d3_) { wb = 1; wc = 0; return b; }
    const double vc = d1 * d4 - d3_ * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3_ <= 0.0) {
        const double t = d1 / (d1 - d3_);
        wb = t; wc = 0;
        return dadd(a, dmul(ab, t));
    }
    const D3 cp = dsub(p, c);
    const double d5 = ddot(ab, cp), d6 = ddot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) { wb = 0; wc = 1; return c; }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double t = d2 / (d2 - d6);
        wb = 0; wc = t;
        return dadd(a, dmul(ac, t));
    }
    const double va = d3_ * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3_) >= 0.0 && (d5 - d6) >= 0.0) {
        const double t = (d4 - d3_) / ((d4 - d3_) + (d5 - d6));
        wb = 1.0 - t; wc = t;
        return dadd(b, dmul(dsub(c, b), t));
    }
    const double denom = va + vb + vc;
    if (!(denom > 1e-300)) {  // degenerate: nearest vertex
        const double da = ddot(dsub(p, a), dsub(p, a)), db = ddot(bp, bp), dc = ddot(cp, cp);
        if (db < da && db <= dc) { wb = 1; wc = 0; return b; }
        if (dc < da && dc < db) { wb = 0; wc = 1; return c; }
        wb = 0; wc = 0;
        return a;
    }
    wb = vb / denom;
    wc = vc / denom;
    return dadd(dadd(a, dmul(ab, wb)), dmul(ac, wc));
}

// quaternion -> rotation columns u, v, w (the engine's gaussianAxes convention) in FP64
__device__ void axes_fp64(const float* q4, D3& u, D3& v, D3& w, double qn[4], double& len) {
    const double x = q4[0], y = q4[1], z = q4[2], ww = q4[3];
    len = sqrt(x * x + y * y + z * z + ww * ww);
    const double inv = len > 0.0 ? 1.0 / len : 1.0;
    const double qx = x * inv, qy = y * inv, qz = z * inv, qw = ww * inv;
    qn[0] = qx; qn[1] = qy; qn[2] = qz; qn[3] = qw;
    u = d3(1.0 - 2.0 * (qy * qy + qz * qz), 2.0 * (qx * qy + qz * qw), 2.0 * (qx * qz - qy * qw));
    v = d3(2.0 * (qx * qy - qz * qw), 1.0 - 2.0 * (qx * qx + qz * qz), 2.0 * (qy * qz + qx * qw));
    w = d3(2.0 * (qx * qz + qy * qw), 2.0 * (qy * qz - qx * qw), 1.0 - 2.0 * (qx * qx + qy * qy));
}

// distance from local point y to the solid ellipsoid with semi-axes s; x the closest point
__device__ double ellipsoid_fp64(D3 y, D3 s, D3& x) {
    const double r = (y.x / s.x) * (y.x / s.x) + (y.y / s.y) * (y.y / s.y) + (y.z / s.z) * (y.z / s.z);
    if (r <= 1.0) {
        x = y;
        return 0.0;
    }
    const double aa = s.x * s.x, bb = s.y * s.y, cc = s.z * s.z;
    const double gy0 = s.x * y.x, gy1 = s.y * y.y, gy2 = s.z * y.z;
    const double amax = fmax(s.x, fmax(s.y, s.z));
    double lo = 0.0, hi = 2.0 * amax * sqrt(ddot(y, y));
    double t = 0.5 * hi;
    // F(t) = sum (s_i y_i / (t + s_i^2))^2 - 1 is decreasing and convex on t >= 0:
    // bracketed Newton, falling back to bisection, until the bracket is tight
    for (int it = 0; it < 200; ++it) {
        const double i0 = 1.0 / (t + aa), i1 = 1.0 / (t + bb), i2 = 1.0 / (t + cc);
        const double s0 = gy0 * i0, s1 = gy1 * i1, s2 = gy2 * i2;
        const double f = s0 * s0 + s1 * s1 + s2 * s2 - 1.0;
        if (f > 0.0) lo = t; else hi = t;
        const double fp = -2.0 * (s0 * s0 * i0 + s1 * s1 * i1 + s2 * s2 * i2);
        double next = 0.5 * (lo + hi);
        if (fp < 0.0) {
            const double nt = t - f / fp;
            if (nt > lo && nt < hi) next = nt;
        }
        if (next == t || hi - lo <= 1e-15 * hi) break;
        t = next;
    }
    x = d3(aa * y.x / (t + aa), bb * y.y / (t + bb), cc * y.z / (t + cc));
    return sqrt(ddot(dsub(y, x), dsub(y, x)));
}

// per query: gradient of w * d for the selected primitive (written in query order)
template <int kKind>
__global__ __launch_bounds__(kBlock) void k_dist_grad(const float* __restrict__ items, int stride,
                                                     const float* __restrict__ pts,
                                                     const uint2* __restrict__ res,
                                                     const float* __restrict__ gw, int count,
                                                     float* __restrict__ gpts,
                                                     double* __restrict__ contrib,
                                                     int* __restrict__ keys) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= count) return;
    const int id = static_cast<int>(res[i].y);
    double* c = contrib + static_cast<size_t>(i) * stride;
    for (int j = 0; j < stride; ++j) c[j] = 0.0;
    gpts[3 * i] = gpts[3 * i + 1] = gpts[3 * i + 2] = 0.0f;
    keys[i] = id;  // -1: no primitive, sorts first and is dropped
    if (id < 0) return;
    const double g = gw ? static_cast<double>(gw[i]) : 1.0;
    const D3 p = ld3(pts + 3 * i);
    const float* it = items + static_cast<size_t>(id) * stride;
    if (kKind == kTri) {
        double wb, wc;
        const D3 a = ld3(it), b = ld3(it + 3), cc = ld3(it + 6);
        const D3 q = closest_tri_fp64(p, a, b, cc, wb, wc);
        const D3 e = dsub(p, q);
        const double d = sqrt(ddot(e, e));
        if (!(d > 0.0)) return;
        const D3 n = dmul(e, g / d);
        const double wa = 1.0 - wb - wc;
        gpts[3 * i] = static_cast<float>(n.x);
        gpts[3 * i + 1] = static_cast<float>(n.y);
        gpts[3 * i + 2] = static_cast<float>(n.z);
        const double w3[3] = {wa, wb, wc};
        for (int k = 0; k < 3; ++k) {
            c[3 * k] = -w3[k] * n.x;
            c[3 * k + 1] = -w3[k] * n.y;
            c[3 * k + 2] = -w3[k] * n.z;
        }
    } else if (kKind == kPoint) {
        const D3 e = dsub(p, ld3(it));
        const double d = sqrt(ddot(e, e));
        if (!(d > 0.0)) return;
        const D3 n = dmul(e, g / d);
        gpts[3 * i] = static_cast<float>(n.x);
        gpts[3 * i + 1] = static_cast<float>(n.y);
        gpts[3 * i + 2] = static_cast<float>(n.z);
        c[0] = -n.x;
        c[1] = -n.y;
        c[2] = -n.z;
    } else {
        D3 u, v, w;
        double qn[4], qlen;
        axes_fp64(it + 3, u, v, w, qn, qlen);
        const D3 m = ld3(it), s = ld3(it + 7);
        const D3 dp = dsub(p, m);
        const D3 y = d3(ddot(dp, u), ddot(dp, v), ddot(dp, w));
        D3 x;
        const double d = ellipsoid_fp64(y, s, x);
        if (!(d > 0.0)) return;
        const D3 nl = dmul(dsub(y, x), 1.0 / d);
        const D3 nw = dadd(dadd(dmul(u, nl.x), dmul(v, nl.y)), dmul(w, nl.z));
        gpts[3 * i] = static_cast<float>(g * nw.x);
        gpts[3 * i + 1] = static_cast<float>(g * nw.y);
        gpts[3 * i + 2] = static_cast<float>(g * nw.z);
        c[0] = -g * nw.x;
        c[1] = -g * nw.y;
        c[2] = -g * nw.z;
        // scales: -n_l,i * x_i / s_i
        c[7] = -g * nl.x * x.x / s.x;
        c[8] = -g * nl.y * x.y / s.y;
        c[9] = -g * nl.z * x.z / s.z;
        // axes: dd/du = n_l.x dp, dd/dv = n_l.y dp, dd/dw = n_l.z dp
        const D3 gu = dmul(dp, nl.x), gv = dmul(dp, nl.y), gwv = dmul(dp, nl.z);
        const double X = qn[0], Y = qn[1], Z = qn[2], W = qn[3];
        // d(u, v, w) / d(qx, qy, qz, qw) of the normalised quaternion
        double gq[4];
        gq[0] = gu.y * 2 * Y + gu.z * 2 * Z + gv.x * 2 * Y + gv.y * -4 * X + gv.z * 2 * W +
                gwv.x * 2 * Z + gwv.y * -2 * W + gwv.z * -4 * X;
        gq[1] = gu.x * -4 * Y + gu.y * 2 * X + gu.z * -2 * W + gv.x * 2 * X + gv.z * 2 * Z +
                gwv.x * 2 * W + gwv.y * 2 * Z + gwv.z * -4 * Y;
        gq[2] = gu.x * -4 * Z + gu.y * 2 * W + gu.z * 2 * X + gv.x * -2 * W + gv.y * -4 * Z +
                gv.z * 2 * Y + gwv.x * 2 * X + gwv.y * 2 * Y;
        gq[3] = gu.y * 2 * Z + gu.z * -2 * Y + gv.x * -2 * Z + gv.z * 2 * X + gwv.x * 2 * Y +
                gwv.y * -2 * X;
        // through q_hat = q / |q|: (I - q_hat q_hat^T) / |q|
        const double dotq = gq[0] * X + gq[1] * Y + gq[2] * Z + gq[3] * W;
        const double inv = qlen > 0.0 ? g / qlen : g;
        for (int k = 0; k < 4; ++k) c[3 + k] = (gq[k] - dotq * qn[k]) * inv;
    }
}

// per ray: gradient of w * t for the hit triangle (vertices; origins and directions too)
__global__ __launch_bounds__(kBlock) void k_ray_grad(const float* __restrict__ tris,
                                                    const float* __restrict__ rays,
                                                    const int* __restrict__ ids,
                                                    const float* __restrict__ gw, int count,
                                                    double* __restrict__ contrib,
                                                    int* __restrict__ keys,
                                                    float* __restrict__ grays) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= count) return;
    const int id = ids[i];
    double* c = contrib + static_cast<size_t>(i) * 9;
    for (int j = 0; j < 9; ++j) c[j] = 0.0;
    if (grays) for (int j = 0; j < 6; ++j) grays[6 * i + j] = 0.0f;
    keys[i] = id;
    if (id < 0) return;
    const double g = gw ? static_cast<double>(gw[i]) : 1.0;
    const float* r = rays + 8 * static_cast<size_t>(i);
    const D3 o = ld3(r), d = ld3(r + 3);
    const float* it = tris + 9 * static_cast<size_t>(id);
    const D3 a = ld3(it), b = ld3(it + 3), cc = ld3(it + 6);
    const D3 e1 = dsub(b, a), e2 = dsub(cc, a);
    const D3 n = dcross(e1, e2);
    const double nd = ddot(n, d);
    if (nd == 0.0) return;
    const double t = ddot(n, dsub(a, o)) / nd;
    const D3 h = dadd(o, dmul(d, t));
    // barycentrics of the hit point
    const D3 ah = dsub(h, a);
    const double nn = ddot(n, n);
    const double u = ddot(dcross(ah, e2), n) / nn;
    const double v = ddot(dcross(e1, ah), n) / nn;
    const double w3[3] = {1.0 - u - v, u, v};
    const D3 k = dmul(n, g / nd);
    for (int j = 0; j < 3; ++j) {
        c[3 * j] = w3[j] * k.x;
        c[3 * j + 1] = w3[j] * k.y;
        c[3 * j + 2] = w3[j] * k.z;
    }
    if (grays) {
        grays[6 * i] = static_cast<float>(-k.x);
        grays[6 * i + 1] = static_cast<float>(-k.y);
        grays[6 * i + 2] = static_cast<float>(-k.z);
        grays[6 * i + 3] = static_cast<float>(-t * k.x);
        grays[6 * i + 4] = static_cast<float>(-t * k.y);
        grays[6 * i + 5] = static_cast<float>(-t * k.z);
    }
}

// one thread per segment key: sum its run (sorted order = query order) in FP64; values are
// the FP64 per-query terms of the adjoints, or a caller's FP32 values (qk_segment_sum)
template <class V>
__global__ __launch_bounds__(kBlock) void k_segment_sum(const uint32_t* __restrict__ skeys,
                                                       const uint32_t* __restrict__ sidx,
                                                       const V* __restrict__ vals, int count,
                                                       int channels, int nseg,
                                                       float* __restrict__ out) {
    const int k = blockIdx.x * kBlock + threadIdx.x;
    if (k >= nseg) return;
    // lower_bound of key k in the sorted keys (keys are shifted by one: -1 -> 0)
    const uint32_t want = static_cast<uint32_t>(k) + 1u;
    int lo = 0, hi = count;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (skeys[mid] < want) lo = mid + 1; else hi = mid;
    }
    double acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = lo; j < count && skeys[j] == want; ++j) {
        const V* v = vals + static_cast<size_t>(sidx[j]) * channels;
        for (int ch = 0; ch < channels && ch < 10; ++ch) acc[ch] += static_cast<double>(v[ch]);
    }
    for (int ch = 0; ch < channels && ch < 10; ++ch) out[static_cast<size_t>(k) * channels + ch] = static_cast<float>(acc[ch]);
}

__global__ void k_shift_keys(const int* __restrict__ keys, int count, uint32_t* __restrict__ k32,
                             uint32_t* __restrict__ idx) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= count) return;
    k32[i] = static_cast<uint32_t>(keys[i] + 1);
    idx[i] = static_cast<uint32_t>(i);
}

struct GradWs {
    double* contrib;
    int* keys;
    uint32_t* k32;
    uint32_t* idx;
    uint32_t* k32s;
    uint32_t* idxs;
    void* sort_ws;
};

GradWs carve_grad(Carve& c, int count, int channels) {
    GradWs g;
    g.contrib = c.take<double>(static_cast<size_t>(count) * channels);
    g.keys = c.take<int>(count);
    g.k32 = c.take<uint32_t>(count);
    g.idx = c.take<uint32_t>(count);
    g.k32s = c.take<uint32_t>(count);
    g.idxs = c.take<uint32_t>(count);
    g.sort_ws = c.take<char>(sort_ws_bytes(count));
    return g;
}

template <class V>
int segment_sum_impl(const int* keys, const V* vals, int count, int channels, int nseg,
                     float* out, GradWs& g, cudaStream_t s) {
    if (nseg <= 0) return QK_OK;
    if (count <= 0) {
        cudaMemsetAsync(out, 0, sizeof(float) * static_cast<size_t>(nseg) * channels, s);
        return QK_OK;
    }
    k_shift_keys<<<blocks_for(count), kBlock, 0, s>>>(keys, count, g.k32, g.idx);
    int bits = 1;
    while (bits < 32 && (1ull << bits) <= static_cast<unsigned long long>(nseg)) ++bits;
    cudaError_t e = sort_pairs(g.k32, g.idx, g.k32s, g.idxs, count, bits, g.sort_ws, s);
    if (e != cudaSuccess) return cuda_status(e, "gradient sort");
    k_segment_sum<V><<<blocks_for(nseg), kBlock, 0, s>>>(g.k32s, g.idxs, vals, count, channels, nseg, out);
    e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_status(e, "segment sum");
}

// Corner e = 3 q + j of query q's selected triangle -> its vertex (indices, n x 3), or -1.
__global__ void k_corner_keys(const int* __restrict__ tri_of, const int* __restrict__ indices,
                              int count, int n, int nverts, int* __restrict__ vkeys) {
    const int e = blockIdx.x * kBlock + threadIdx.x;
    if (e >= 3 * count) return;
    const int t = tri_of[e / 3];
    int v = -1;
    if (t >= 0 && t < n) {
        v = indices[3 * t + e % 3];
        if (v < 0 || v >= nverts) v = -1;
    }
    vkeys[e] = v;
}

// vertex form: per-query terms (count x 9), their triangles, then the corner keys; the sort
// and sum run over 3 count corner entries of 3 channels
GradWs carve_grad_vertices(Carve& c, int count, int** tri_of) {
    GradWs g;
    g.contrib = c.take<double>(static_cast<size_t>(count) * 9);
    *tri_of = c.take<int>(count);
    g.keys = c.take<int>(3 * static_cast<size_t>(count));
    g.k32 = c.take<uint32_t>(3 * static_cast<size_t>(count));
    g.idx = c.take<uint32_t>(3 * static_cast<size_t>(count));
    g.k32s = c.take<uint32_t>(3 * static_cast<size_t>(count));
    g.idxs = c.take<uint32_t>(3 * static_cast<size_t>(count));
    g.sort_ws = c.take<char>(sort_ws_bytes(3 * count));
    return g;
}

}  // namespace

size_t grad_vertices_ws_bytes(int count) {
    Carve c;
    int* t = nullptr;
    carve_grad_vertices(c, count, &t);
    return c.used;
}

int ray_t_grad_vertices(int n, const void* tris, const void* rays, const int* ids, const float* gw,
                        int count, const int* indices, int nverts, float* gverts, float* grays,
                        void* ws, cudaStream_t s) {
    Carve c{static_cast<char*>(ws)};
    int* tri_of = nullptr;
    GradWs g = carve_grad_vertices(c, count, &tri_of);
    if (count > 0) {
        k_ray_grad<<<blocks_for(count), kBlock, 0, s>>>(static_cast<const float*>(tris),
                                                        static_cast<const float*>(rays), ids, gw,
                                                        count, g.contrib, tri_of, grays);
        k_corner_keys<<<blocks_for(3ll * count), kBlock, 0, s>>>(tri_of, indices, count, n, nverts,
                                                                 g.keys);
    }
    return segment_sum_impl<double>(g.keys, g.contrib, 3 * count, 3, nverts, gverts, g, s);
}

int distance_grad_vertices(int n, const void* tris, const float* pts, const void* res,
                           const float* gw, int count, const int* indices, int nverts,
                           float* gpts, float* gverts, void* ws, cudaStream_t s) {
    Carve c{static_cast<char*>(ws)};
    int* tri_of = nullptr;
    GradWs g = carve_grad_vertices(c, count, &tri_of);
    if (count > 0) {
        k_dist_grad<kTri><<<blocks_for(count), kBlock, 0, s>>>(
            static_cast<const float*>(tris), 9, pts, static_cast<const uint2*>(res), gw, count, gpts,
            g.contrib, tri_of);
        k_corner_keys<<<blocks_for(3ll * count), kBlock, 0, s>>>(tri_of, indices, count, n, nverts,
                                                                 g.keys);
    }
    return segment_sum_impl<double>(g.keys, g.contrib, 3 * count, 3, nverts, gverts, g, s);
}

size_t grad_ws_bytes(int count, int channels) {
    Carve c;
    carve_grad(c, count, channels);
    return c.used;
}

int closest_distance_grad(int kind, int n, const void* items, const float* pts, const void* res,
                          const float* gw, int count, float* gpts, float* gitems, void* ws,
                          cudaStream_t s) {
    const int stride = kind == kTri ? 9 : kind == kPoint ? 3 : 10;
    Carve c{static_cast<char*>(ws)};
    GradWs g = carve_grad(c, count, stride);
    const float* it = static_cast<const float*>(items);
    const uint2* r = static_cast<const uint2*>(res);
    if (count > 0) {
        if (kind == kTri) k_dist_grad<kTri><<<blocks_for(count), kBlock, 0, s>>>(it, stride, pts, r, gw, count, gpts, g.contrib, g.keys);
        else if (kind == kPoint) k_dist_grad<kPoint><<<blocks_for(count), kBlock, 0, s>>>(it, stride, pts, r, gw, count, gpts, g.contrib, g.keys);
        else k_dist_grad<kGauss><<<blocks_for(count), kBlock, 0, s>>>(it, stride, pts, r, gw, count, gpts, g.contrib, g.keys);
    }
    return segment_sum_impl(g.keys, g.contrib, count, stride, n, gitems, g, s);
}

int ray_t_grad(int n, const void* tris, const void* rays, const int* ids, const float* gw,
               int count, float* gtris, float* grays, void* ws, cudaStream_t s) {
    Carve c{static_cast<char*>(ws)};
    GradWs g = carve_grad(c, count, 9);
    if (count > 0) {
        k_ray_grad<<<blocks_for(count), kBlock, 0, s>>>(static_cast<const float*>(tris),
                                                        static_cast<const float*>(rays), ids, gw,
                                                        count, g.contrib, g.keys, grays);
    }
    return segment_sum_impl(g.keys, g.contrib, count, 9, n, gtris, g, s);
}

int segment_sum(const int* keys, const float* vals, int count, int channels, int nseg, float* out,
                void* ws, cudaStream_t s) {
    Carve c{static_cast<char*>(ws)};
    GradWs g = carve_grad(c, count, 0);
    return segment_sum_impl(keys, vals, count, channels, nseg, out, g, s);
}

}  // namespace qk
