/*
 * scenes.c -- seeded synthetic workloads for the spatial-query engine.
 *
 * Two families:
 *   qs_demo_*  the demo generators behind the Python module's demo_mesh / demo_gaussians
 *              (terrain / random / mixed / city meshes, sheet / volume Gaussian clouds),
 *              restated from quarry's src/core/scene.cpp:53-189 and src/core/gaussian.cpp.
 *   qs_cfg*    the benchmark workloads (z-up terrain, floorless city, sphere / volume point
 *              clouds, Gaussian clouds, uneven scene batches).
 *
 * Determinism: every transcendental function used by the workload generators is computed
 * here from +, -, *, / and sqrt only (Cody-Waite range reduction followed by a Taylor
 * series; log through the atanh series of (m-1)/(m+1) after an exact frexp), in double,
 * and the file is compiled with -ffp-contract=off.  IEEE-754 rounds those operations the
 * same way on every conforming host, so a given seed produces the same bytes on any
 * machine -- the GPU box and the CPU that checks it included.  The demo generators call
 * the C library's sinf/cosf like the reference did, so their bytes may differ between
 * C libraries; nothing checks them against stored fingerprints.
 */
#include "scenes.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* PCG32 with the seeding sequence of quarry's src/core/rng.h:7-38              */
/* ------------------------------------------------------------------------- */
typedef struct {
    uint64_t state, inc;
} pcg32;

static uint32_t pcg_next(pcg32* r) {
    const uint64_t old = r->state;
    r->state = old * 6364136223846793005ull + r->inc;
    const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
}

static pcg32 pcg_make(uint64_t seed, uint64_t stream) {
    pcg32 r;
    r.state = 0;
    r.inc = (stream << 1u) | 1u;
    pcg_next(&r);
    r.state += 0x853c49e6748fea9bull;
    pcg_next(&r);
    r.state += seed;
    pcg_next(&r);
    return r;
}

static float pcg_u01f(pcg32* r) { return (float)(pcg_next(r) >> 8) * (1.0f / 16777216.0f); }
static float pcg_uf(pcg32* r, float lo, float hi) { return lo + (hi - lo) * pcg_u01f(r); }
/* double in [0,1) from 53 random bits */
static double pcg_u01d(pcg32* r) {
    const uint64_t hi = pcg_next(r) >> 5, lo = pcg_next(r) >> 6;
    return (double)(hi * 67108864ull + lo) * (1.0 / 9007199254740992.0);
}

/* ------------------------------------------------------------------------- */
/* deterministic transcendental functions (double, basic IEEE ops only)        */
/* ------------------------------------------------------------------------- */
static const double kPi = 3.14159265358979323846;
static const double kTwoPi = 6.28318530717958647692;
/* 2*pi split so that k*kTwoPiHi is exact for |k| < 2^20 (Cody-Waite) */
static const double kTwoPiHi = 6.28318405151367187500;
static const double kTwoPiLo = 1.2556659146019252e-06;
static const double kLn2Hi = 6.93147180369123816490e-01;
static const double kLn2Lo = 1.90821492927058770002e-10;

/* sin(r), cos(r) for |r| <= pi/4 by Taylor series to degree 25/24 */
static double sin_core(double r) {
    const double r2 = r * r;
    double term = r, sum = r;
    for (int i = 1; i <= 12; ++i) {
        term = -term * r2 / (double)((2 * i) * (2 * i + 1));
        sum += term;
    }
    return sum;
}
static double cos_core(double r) {
    const double r2 = r * r;
    double term = 1.0, sum = 1.0;
    for (int i = 1; i <= 12; ++i) {
        term = -term * r2 / (double)((2 * i - 1) * (2 * i));
        sum += term;
    }
    return sum;
}

/* reduce x to r in [-pi/4, pi/4] and quadrant q, x = q*pi/2 + r (mod 2 pi) */
static double reduce_quadrant(double x, int* q) {
    const double k = floor(x / kTwoPi + 0.5);
    double r = (x - k * kTwoPiHi) - k * kTwoPiLo; /* r in about [-pi, pi] */
    const double h = floor(r / (0.5 * kPi) + 0.5);  /* -2..2 */
    r = (r - h * (0.5 * kTwoPiHi * 0.5)) - h * (0.5 * kTwoPiLo * 0.5);
    *q = ((int)h % 4 + 4) % 4;
    return r;
}

double qs_det_sin(double x) {
    int q;
    const double r = reduce_quadrant(x, &q);
    switch (q) {
        case 0: return sin_core(r);
        case 1: return cos_core(r);
        case 2: return -sin_core(r);
        default: return -cos_core(r);
    }
}

double qs_det_cos(double x) {
    int q;
    const double r = reduce_quadrant(x, &q);
    switch (q) {
        case 0: return cos_core(r);
        case 1: return -sin_core(r);
        case 2: return -cos_core(r);
        default: return sin_core(r);
    }
}

/* natural log for x > 0: x = m * 2^e with m in [sqrt(1/2), sqrt(2)), then
 * log m = 2 atanh(s), s = (m-1)/(m+1), |s| < 0.172 */
double qs_det_log(double x) {
    int e;
    double m = frexp(x, &e); /* exact: m in [0.5, 1) */
    if (m < 0.70710678118654752440) {
        m *= 2.0;
        e -= 1;
    }
    const double s = (m - 1.0) / (m + 1.0);
    const double s2 = s * s;
    double term = s, sum = s;
    for (int i = 1; i <= 14; ++i) {
        term *= s2;
        sum += term / (double)(2 * i + 1);
    }
    return 2.0 * sum + (double)e * kLn2Hi + (double)e * kLn2Lo;
}

/* exp by k = round(x / ln 2), r = x - k ln 2 (two-part), Taylor to degree 22, ldexp */
double qs_det_exp(double x) {
    const double k = floor(x / (kLn2Hi + kLn2Lo) + 0.5);
    const double r = (x - k * kLn2Hi) - k * kLn2Lo;
    double term = 1.0, sum = 1.0;
    for (int i = 1; i <= 22; ++i) {
        term = term * r / (double)i;
        sum += term;
    }
    return ldexp(sum, (int)k);
}

/* standard normal by Box-Muller on two uniforms (u1 in (0,1]) */
static double normal01(pcg32* r) {
    const double u1 = 1.0 - pcg_u01d(r);
    const double u2 = pcg_u01d(r);
    return sqrt(-2.0 * qs_det_log(u1)) * qs_det_cos(kTwoPi * u2);
}

static void put3(float* dst, double x, double y, double z) {
    dst[0] = (float)x;
    dst[1] = (float)y;
    dst[2] = (float)z;
}

/* ========================================================================= */
/* benchmark workloads                                                       */
/* ========================================================================= */

/* Terrain: z-up heightfield on grid x grid unit cells with (grid+1)^2 vertices at integer
 * (x, y).  h(x,y) = sum_k A_k sin(2 pi f_k x + phi_k) sin(2 pi g_k y + psi_k) with
 * A = (8,4,2,1), f_k, g_k uniform in [1/64, 1/8], phases uniform in [0, 2 pi).
 * Two triangles per cell: (v00, v10, v11), (v00, v11, v01); rows of y outermost. */
int64_t qs_cfg_terrain(int grid, uint64_t seed, float* tris9) {
    if (grid < 1) return 0;
    pcg32 rng = pcg_make(seed, 11);
    double f[4], g[4], ph[4], ps[4];
    const double amp[4] = {8.0, 4.0, 2.0, 1.0};
    for (int k = 0; k < 4; ++k) {
        f[k] = 1.0 / 64.0 + (1.0 / 8.0 - 1.0 / 64.0) * pcg_u01d(&rng);
        g[k] = 1.0 / 64.0 + (1.0 / 8.0 - 1.0 / 64.0) * pcg_u01d(&rng);
        ph[k] = kTwoPi * pcg_u01d(&rng);
        ps[k] = kTwoPi * pcg_u01d(&rng);
    }
    const int nv = grid + 1;
    if (tris9 == NULL) return 2ll * grid * grid;
    float* hz = (float*)malloc(sizeof(float) * (size_t)nv * (size_t)nv);
    /* separable: precompute the per-axis sines */
    double* sx = (double*)malloc(sizeof(double) * 4 * (size_t)nv);
    double* sy = (double*)malloc(sizeof(double) * 4 * (size_t)nv);
    for (int i = 0; i < nv; ++i) {
        for (int k = 0; k < 4; ++k) {
            sx[4 * i + k] = qs_det_sin(kTwoPi * f[k] * (double)i + ph[k]);
            sy[4 * i + k] = qs_det_sin(kTwoPi * g[k] * (double)i + ps[k]);
        }
    }
    for (int j = 0; j < nv; ++j) {
        for (int i = 0; i < nv; ++i) {
            double h = 0.0;
            for (int k = 0; k < 4; ++k) h += amp[k] * sx[4 * i + k] * sy[4 * j + k];
            hz[(size_t)j * nv + i] = (float)h;
        }
    }
    int64_t t = 0;
    for (int j = 0; j < grid; ++j) {
        for (int i = 0; i < grid; ++i) {
            float v00[3] = {(float)i, (float)j, hz[(size_t)j * nv + i]};
            float v10[3] = {(float)(i + 1), (float)j, hz[(size_t)j * nv + i + 1]};
            float v11[3] = {(float)(i + 1), (float)(j + 1), hz[(size_t)(j + 1) * nv + i + 1]};
            float v01[3] = {(float)i, (float)(j + 1), hz[(size_t)(j + 1) * nv + i]};
            float* a = tris9 + 9 * t++;
            memcpy(a, v00, 12);
            memcpy(a + 3, v10, 12);
            memcpy(a + 6, v11, 12);
            float* b = tris9 + 9 * t++;
            memcpy(b, v00, 12);
            memcpy(b + 3, v11, 12);
            memcpy(b + 6, v01, 12);
        }
    }
    free(sx);
    free(sy);
    free(hz);
    return t;
}

/* Downward rays: origin uniform over [x0,x1] x [y0,y1] at height z, direction (0,0,-1). */
void qs_cfg_down_rays(int count, float x0, float x1, float y0, float y1, float z, uint64_t seed,
                      float* rays8) {
    pcg32 rng = pcg_make(seed, 12);
    for (int i = 0; i < count; ++i) {
        float* r = rays8 + 8 * (size_t)i;
        r[0] = (float)(x0 + (x1 - x0) * pcg_u01d(&rng));
        r[1] = (float)(y0 + (y1 - y0) * pcg_u01d(&rng));
        r[2] = z;
        r[3] = 0.0f;
        r[4] = 0.0f;
        r[5] = -1.0f;
        r[6] = 1e-6f;
        r[7] = INFINITY;
    }
}

/* Rays from a plane z with cosine-weighted directions about -z:
 * rho = sqrt(u1), phi = 2 pi u2, d = (rho cos phi, rho sin phi, -sqrt(1 - u1)). */
void qs_cfg_cosine_rays(int count, float x0, float x1, float y0, float y1, float z,
                        uint64_t seed, float* rays8) {
    pcg32 rng = pcg_make(seed, 12);
    for (int i = 0; i < count; ++i) {
        float* r = rays8 + 8 * (size_t)i;
        r[0] = (float)(x0 + (x1 - x0) * pcg_u01d(&rng));
        r[1] = (float)(y0 + (y1 - y0) * pcg_u01d(&rng));
        r[2] = z;
        const double u1 = pcg_u01d(&rng), u2 = pcg_u01d(&rng);
        const double rho = sqrt(u1), phi = kTwoPi * u2;
        r[3] = (float)(rho * qs_det_cos(phi));
        r[4] = (float)(rho * qs_det_sin(phi));
        r[5] = (float)(-sqrt(1.0 - u1));
        r[6] = 1e-6f;
        r[7] = INFINITY;
    }
}

/* Query points uniform in the box [lo, hi] (per axis). */
void qs_cfg_uniform_points(int count, const float* lo3, const float* hi3, uint64_t seed,
                           uint64_t stream, float* pts3) {
    pcg32 rng = pcg_make(seed, stream);
    for (int i = 0; i < count; ++i) {
        for (int a = 0; a < 3; ++a) {
            pts3[3 * (size_t)i + a] =
                (float)((double)lo3[a] + ((double)hi3[a] - (double)lo3[a]) * pcg_u01d(&rng));
        }
    }
}

/* City: `buildings` floorless boxes on a cols x rows lot grid (cols = ceil(sqrt(n)),
 * rows = ceil(n / cols)) with 10-unit lots.  Footprint sides uniform in [1, 8], heights
 * log-normal with median 10 and sigma 0.8, each box jittered inside its lot so boxes never
 * overlap.  10 triangles per box: four walls (two each) and the roof (two).
 * Returns the triangle count; max_height receives the tallest roof. */
int64_t qs_cfg_city(int buildings, uint64_t seed, float* tris9, float* max_height) {
    if (buildings <= 0) return 0;
    if (tris9 == NULL) return 10ll * buildings;
    int cols = (int)sqrt((double)buildings);
    while ((int64_t)cols * cols < buildings) ++cols;
    pcg32 rng = pcg_make(seed, 14);
    const double lot = 10.0;
    float top = 0.0f;
    int64_t t = 0;
    for (int b = 0; b < buildings; ++b) {
        const int cx = b % cols, cy = b / cols;
        const double w = 1.0 + 7.0 * pcg_u01d(&rng);
        const double d = 1.0 + 7.0 * pcg_u01d(&rng);
        const double h = 10.0 * qs_det_exp(0.8 * normal01(&rng));
        const double jx = (pcg_u01d(&rng) - 0.5) * (lot - w);
        const double jy = (pcg_u01d(&rng) - 0.5) * (lot - d);
        const double mx = (cx + 0.5) * lot + jx, my = (cy + 0.5) * lot + jy;
        const float x0 = (float)(mx - 0.5 * w), x1 = (float)(mx + 0.5 * w);
        const float y0 = (float)(my - 0.5 * d), y1 = (float)(my + 0.5 * d);
        const float z0 = 0.0f, z1 = (float)h;
        if (z1 > top) top = z1;
        const float c[8][3] = {{x0, y0, z0}, {x1, y0, z0}, {x1, y1, z0}, {x0, y1, z0},
                               {x0, y0, z1}, {x1, y0, z1}, {x1, y1, z1}, {x0, y1, z1}};
        /* walls: (b0 t0 t1) (b0 t1 b1) around the ring, roof (t0 t2 t1) (t0 t3 t2) */
        static const int idx[10][3] = {{0, 4, 5}, {0, 5, 1}, {1, 5, 6}, {1, 6, 2}, {2, 6, 7},
                                       {2, 7, 3}, {3, 7, 4}, {3, 4, 0}, {4, 6, 5}, {4, 7, 6}};
        for (int k = 0; k < 10; ++k) {
            float* dst = tris9 + 9 * t++;
            for (int v = 0; v < 3; ++v) memcpy(dst + 3 * v, c[idx[k][v]], 12);
        }
    }
    if (max_height) *max_height = top;
    return t;
}

/* Point clouds.  kind 0: sphere of radius 50 about the origin with N(0, 0.5) radial noise,
 * directions uniform (z uniform in [-1,1], phi uniform).  kind 1: uniform in [0,100]^3. */
void qs_cfg_points(int kind, int count, uint64_t seed, float* pts3) {
    pcg32 rng = pcg_make(seed, 15);
    for (int i = 0; i < count; ++i) {
        float* p = pts3 + 3 * (size_t)i;
        if (kind == 1) {
            put3(p, 100.0 * pcg_u01d(&rng), 100.0 * pcg_u01d(&rng), 100.0 * pcg_u01d(&rng));
        } else {
            const double z = 2.0 * pcg_u01d(&rng) - 1.0;
            const double phi = kTwoPi * pcg_u01d(&rng);
            const double rxy = sqrt(1.0 - z * z);
            const double rad = 50.0 + 0.5 * normal01(&rng);
            put3(p, rad * rxy * qs_det_cos(phi), rad * rxy * qs_det_sin(phi), rad * z);
        }
    }
}

/* Coherent refit motion: the `dirty` points nearest to a random anchor point (ties by index)
 * move by N(0, sigma) per axis.  Writes the moved cloud to out3 and the dirty indices
 * (ascending) to ids. */
typedef struct {
    double d;
    int32_t i;
} dist_idx;

static int cmp_dist_idx(const void* a, const void* b) {
    const dist_idx* x = (const dist_idx*)a;
    const dist_idx* y = (const dist_idx*)b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return x->i < y->i ? -1 : x->i > y->i ? 1 : 0;
}
static int cmp_i32(const void* a, const void* b) {
    const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return x < y ? -1 : x > y ? 1 : 0;
}

void qs_cfg_coherent_motion(const float* pts3, int count, int dirty, float sigma, uint64_t seed,
                            float* out3, int32_t* ids) {
    pcg32 rng = pcg_make(seed, 16);
    memcpy(out3, pts3, sizeof(float) * 3 * (size_t)count);
    if (dirty <= 0 || count <= 0) return;
    if (dirty > count) dirty = count;
    const int anchor = (int)(pcg_next(&rng) % (uint32_t)count);
    dist_idx* di = (dist_idx*)malloc(sizeof(dist_idx) * (size_t)count);
    for (int i = 0; i < count; ++i) {
        double s = 0.0;
        for (int a = 0; a < 3; ++a) {
            const double e = (double)pts3[3 * (size_t)i + a] - (double)pts3[3 * (size_t)anchor + a];
            s += e * e;
        }
        di[i].d = s;
        di[i].i = i;
    }
    qsort(di, (size_t)count, sizeof(dist_idx), cmp_dist_idx);
    for (int k = 0; k < dirty; ++k) ids[k] = di[k].i;
    free(di);
    qsort(ids, (size_t)dirty, sizeof(int32_t), cmp_i32);
    for (int k = 0; k < dirty; ++k) {
        float* p = out3 + 3 * (size_t)ids[k];
        for (int a = 0; a < 3; ++a) p[a] = (float)((double)p[a] + sigma * normal01(&rng));
    }
}

/* Gaussians: means uniform in [0,100]^3, per-axis scales log-uniform in [smin, smax],
 * rotations uniform unit quaternions (Shoemake 1992). */
void qs_cfg_gaussians(int count, float smin, float smax, uint64_t seed, float* g10) {
    pcg32 rng = pcg_make(seed, 17);
    const double lmin = qs_det_log((double)smin), lmax = qs_det_log((double)smax);
    for (int i = 0; i < count; ++i) {
        float* g = g10 + 10 * (size_t)i;
        put3(g, 100.0 * pcg_u01d(&rng), 100.0 * pcg_u01d(&rng), 100.0 * pcg_u01d(&rng));
        const double u1 = pcg_u01d(&rng), u2 = pcg_u01d(&rng), u3 = pcg_u01d(&rng);
        const double s1 = sqrt(1.0 - u1), s2 = sqrt(u1);
        g[3] = (float)(s1 * qs_det_sin(kTwoPi * u2));
        g[4] = (float)(s1 * qs_det_cos(kTwoPi * u2));
        g[5] = (float)(s2 * qs_det_sin(kTwoPi * u3));
        g[6] = (float)(s2 * qs_det_cos(kTwoPi * u3));
        for (int a = 0; a < 3; ++a) {
            g[7 + a] = (float)qs_det_exp(lmin + (lmax - lmin) * pcg_u01d(&rng));
        }
    }
}

/* log-uniform integer in [lo, hi] */
int qs_log_uniform_int(uint64_t seed, uint64_t stream, int lo, int hi) {
    pcg32 rng = pcg_make(seed, stream);
    const double a = qs_det_log((double)lo), b = qs_det_log((double)hi);
    double v = qs_det_exp(a + (b - a) * pcg_u01d(&rng));
    int r = (int)(v + 0.5);
    if (r < lo) r = lo;
    if (r > hi) r = hi;
    return r;
}

/* ========================================================================= */
/* demo generators (restating quarry's src/core/scene.cpp, gaussian.cpp)     */
/* ========================================================================= */
static float demo_height(float x, float z) {
    return 3.0f * sinf(0.13f * x) * cosf(0.11f * z) +
           1.2f * sinf(0.37f * x + 0.7f) * sinf(0.31f * z + 1.3f) +
           0.4f * sinf(0.90f * x) * sinf(0.80f * z);
}

static int64_t demo_terrain(int grid, float half, float* out) {
    const float step = (2.0f * half) / (float)grid;
    int64_t t = 0;
    for (int zi = 0; zi < grid; ++zi) {
        for (int xi = 0; xi < grid; ++xi) {
            const float x0 = -half + step * (float)xi, z0 = -half + step * (float)zi;
            const float x1 = x0 + step, z1 = z0 + step;
            const float p00[3] = {x0, demo_height(x0, z0), z0};
            const float p10[3] = {x1, demo_height(x1, z0), z0};
            const float p11[3] = {x1, demo_height(x1, z1), z1};
            const float p01[3] = {x0, demo_height(x0, z1), z1};
            if (out) {
                float* a = out + 9 * t;
                memcpy(a, p00, 12);
                memcpy(a + 3, p10, 12);
                memcpy(a + 6, p11, 12);
                float* b = out + 9 * (t + 1);
                memcpy(b, p00, 12);
                memcpy(b + 3, p11, 12);
                memcpy(b + 6, p01, 12);
            }
            t += 2;
        }
    }
    return t;
}

static float len3(const float* v) { return sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

static int64_t demo_random(int count, uint64_t seed, float* out) {
    pcg32 rng = pcg_make(seed, 1);
    int64_t t = 0;
    while (t < count) {
        float a[3], b[3], c[3];
        for (int k = 0; k < 3; ++k) a[k] = pcg_uf(&rng, -50.0f, 50.0f);
        for (int k = 0; k < 3; ++k) b[k] = a[k] + pcg_uf(&rng, -5.0f, 5.0f);
        for (int k = 0; k < 3; ++k) c[k] = a[k] + pcg_uf(&rng, -5.0f, 5.0f);
        const float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        const float e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        const float cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                             e1[0] * e2[1] - e1[1] * e2[0]};
        if (len3(cr) < 1e-4f) continue;
        if (out) {
            memcpy(out + 9 * t, a, 12);
            memcpy(out + 9 * t + 3, b, 12);
            memcpy(out + 9 * t + 6, c, 12);
        }
        ++t;
    }
    return t;
}

static void demo_box(float* out, float cx, float y0, float cz, float w, float h, float d) {
    const float x0 = cx - 0.5f * w, x1 = cx + 0.5f * w;
    const float z0 = cz - 0.5f * d, z1 = cz + 0.5f * d;
    const float y1 = y0 + h;
    const float v[8][3] = {{x0, y0, z0}, {x1, y0, z0}, {x1, y0, z1}, {x0, y0, z1},
                           {x0, y1, z0}, {x1, y1, z0}, {x1, y1, z1}, {x0, y1, z1}};
    /* b00 b10 b11 b01 t00 t10 t11 t01 = 0..7 */
    static const int idx[10][3] = {{0, 4, 5}, {0, 5, 1}, {1, 5, 6}, {1, 6, 2}, {2, 6, 7},
                                   {2, 7, 3}, {3, 7, 4}, {3, 4, 0}, {4, 7, 6}, {4, 6, 5}};
    for (int k = 0; k < 10; ++k)
        for (int j = 0; j < 3; ++j) memcpy(out + 9 * k + 3 * j, v[idx[k][j]], 12);
}

static int64_t demo_city(int buildings, uint64_t seed, float* out) {
    if (buildings <= 0) return demo_terrain(128, 50.0f, out);
    int side = (int)ceil(sqrt((double)buildings));
    if (side < 1) side = 1;
    const float spacing = 8.0f;
    const float half = 0.5f * spacing * (float)side;
    int64_t t = demo_terrain(128, half, out);
    pcg32 rng = pcg_make(seed, 4);
    for (int i = 0; i < buildings; ++i) {
        const int bx = i % side, bz = i / side;
        const float cx = -half + ((float)bx + 0.5f) * spacing + pcg_uf(&rng, -1.2f, 1.2f);
        const float cz = -half + ((float)bz + 0.5f) * spacing + pcg_uf(&rng, -1.2f, 1.2f);
        const float w = pcg_uf(&rng, 1.5f, 5.0f);
        const float d = pcg_uf(&rng, 1.5f, 5.0f);
        const float u = pcg_u01f(&rng);
        const float h = 4.0f + 56.0f * u * u * u;
        if (out) demo_box(out + 9 * t, cx, demo_height(cx, cz) - 0.6f, cz, w, h, d);
        t += 10;
    }
    return t;
}

/* kind: 0 terrain, 1 random, 2 mixed, 3 city.  out NULL returns the count only. */
int64_t qs_demo_mesh(int kind, int grid, int random_tris, uint64_t seed, int buildings,
                     float* tris9) {
    switch (kind) {
        case 0: return demo_terrain(grid, 50.0f, tris9);
        case 1: return demo_random(random_tris, seed, tris9);
        case 2: {
            const int64_t a = demo_terrain(grid, 50.0f, tris9);
            const int64_t b = demo_random(random_tris, seed, tris9 ? tris9 + 9 * a : NULL);
            return a + b;
        }
        case 3: return demo_city(buildings, seed, tris9);
        default: return -1;
    }
}

/* kind: 0 sheet (means on the demo height field), 1 volume.  Scales: major axis uniform in
 * [0.08, 0.5], minor axes major * uniform[0.4, 1]. */
void qs_demo_gaussians(int kind, int count, uint64_t seed, float* g10) {
    pcg32 rng = pcg_make(seed, 5);
    const float half = 50.0f;
    for (int i = 0; i < count; ++i) {
        float* g = g10 + 10 * (size_t)i;
        if (kind == 1) {
            g[0] = pcg_uf(&rng, -half, half);
            g[1] = pcg_uf(&rng, -half, half);
            g[2] = pcg_uf(&rng, -half, half);
        } else {
            const float x = pcg_uf(&rng, -half, half);
            const float z = pcg_uf(&rng, -half, half);
            g[0] = x;
            g[1] = demo_height(x, z);
            g[2] = z;
        }
        const float u1 = pcg_u01f(&rng), u2 = pcg_u01f(&rng), u3 = pcg_u01f(&rng);
        const float twoPi = 6.28318530717958647692f;
        const float s1 = sqrtf(1.0f - u1), s2 = sqrtf(u1);
        g[3] = s1 * sinf(twoPi * u2);
        g[4] = s1 * cosf(twoPi * u2);
        g[5] = s2 * sinf(twoPi * u3);
        g[6] = s2 * cosf(twoPi * u3);
        const float major = pcg_uf(&rng, 0.08f, 0.50f);
        g[7] = major;
        g[8] = major * pcg_uf(&rng, 0.40f, 1.0f);
        g[9] = major * pcg_uf(&rng, 0.40f, 1.0f);
    }
}
