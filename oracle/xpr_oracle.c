/*
 * xpr_oracle.c -- CPU oracle for the XPRecon iterative cone-beam hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see xpr_oracle.h).  Compiled with
 *   gcc -O2 -std=c11 -fopenmp -ffp-contract=off -fno-fast-math -fPIC -shared
 * so that every single-precision operation is an IEEE-754 operation in the
 * written order; fused multiply-adds appear only where fmaf() is called.
 */
#include "xpr_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ======================================================================== */
/* bit helpers                                                              */
/* ======================================================================== */
static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* ======================================================================== */
/* portable single-precision exp / log                                      */
/* ======================================================================== */
/* 2^k for -126 <= k <= 127 */
static inline float pow2i(int k) { return u2f((uint32_t)(k + 127) << 23); }

/* exp(x): Cody & Waite argument reduction x = k ln2 + r with ln2 split into a
 * 16-significant-bit head (so k*ln2_hi is exact for |k| <= 256) and a tail,
 * then the degree-7 Taylor polynomial of e^r on |r| <= ln2/2 (truncation error
 * < 0.05 ulp), then scaling by 2^k in two factors so both stay normal. */
float orc_expf(float x)
{
    if (x != x) return x;
    if (x > 0x1.62e42ep+6f) return INFINITY;     /* largest x with a finite result */
    if (x < -0x1.9fe368p+6f) return 0.0f;        /* below ln(2^-150) */
    float k = rintf(x * 0x1.715476p+0f);         /* round(x / ln2) */
    float r = fmaf(-k, 0x1.62e4p-1f, x);
    r = fmaf(-k, 0x1.7f7d1cp-20f, r);
    float p = 0x1.a01a02p-13f;                   /* 1/7! */
    p = fmaf(p, r, 0x1.6c16c2p-10f);             /* 1/6! */
    p = fmaf(p, r, 0x1.111112p-7f);              /* 1/5! */
    p = fmaf(p, r, 0x1.555556p-5f);              /* 1/4! */
    p = fmaf(p, r, 0x1.555556p-3f);              /* 1/3! */
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    int ki = (int)k;
    int k1 = ki / 2, k2 = ki - k1;
    return (p * pow2i(k1)) * pow2i(k2);
}

/* log(x): x = 2^e m with m in (sqrt(1/2), sqrt(2)]; log m = 2 atanh(s) with
 * s = (m-1)/(m+1), |s| <= 0.1716, summed as 2s(1 + z/3 + z^2/5 + z^3/7 + z^4/9),
 * z = s^2 (truncation < 1e-9 relative); then e*ln2 added with the split ln2. */
float orc_logf(float x)
{
    if (x != x || x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (x == INFINITY) return x;
    int adj = 0;
    if (x < 0x1p-126f) { x = x * 0x1p23f; adj = -23; }
    uint32_t b = f2u(x);
    int e = (int)((b >> 23) & 0xffu) - 127 + adj;
    float m = u2f((b & 0x7fffffu) | 0x3f800000u);
    if (m > 0x1.6a09e6p+0f) { m = m * 0.5f; e += 1; }
    float s = (m - 1.0f) / (m + 1.0f);
    float z = s * s;
    float q = fmaf(z, 0x1.c71c72p-4f, 0x1.24924ap-3f); /* 1/9, 1/7 */
    q = fmaf(q, z, 0x1.99999ap-3f);                     /* 1/5 */
    q = fmaf(q, z, 0x1.555556p-2f);                     /* 1/3 */
    float t = s + s;
    float lm = fmaf(t, z * q, t);
    float fe = (float)e;
    return fmaf(fe, 0x1.62e4p-1f, fmaf(fe, 0x1.7f7d1cp-20f, lm));
}

/* ======================================================================== */
/* std::mt19937 (Matsumoto & Nishimura 1998) and libstdc++'s                */
/* uniform_real_distribution<float> (generate_canonical<float, 24>)         */
/* reference.hpp:36,268-272 draws one value per axis per sub-iteration.     */
/* ======================================================================== */
void orc_mt_seed(orc_mt19937 *g, uint32_t seed)
{
    g->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->idx = 624;
}

uint32_t orc_mt_next(orc_mt19937 *g)
{
    if (g->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->idx = 0;
    }
    uint32_t y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

float orc_uniform_float(orc_mt19937 *g, float a, float b)
{
    /* one 32-bit draw suffices for 24 bits: canonical = float(u) / 2^32,
     * clamped below 1 (it rounds up to 1 for u close to 2^32). */
    float c = (float)orc_mt_next(g) / 4294967296.0f;
    if (c >= 1.0f) c = 0x1.fffffep-1f;
    return c * (b - a) + a;
}

/* ======================================================================== */
/* fixed point, conversions (constants.cl:17-23)                            */
/* ======================================================================== */
/* float -> u32 truncation, saturating, NaN -> 0 (as the GPU cvt does). */
uint32_t orc_float_to_fixed(float x)
{
    float s = x * 4194304.0f;
    if (!(s > 0.0f)) return 0u;
    if (s >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)s;
}

float orc_fixed_to_float(uint32_t x) { return (float)x / 4194304.0f; }

/* float -> i32 truncation, saturating, NaN -> 0 */
static inline int32_t sat_f2i(float f)
{
    if (f != f) return 0;
    if (f >= 2147483648.0f) return INT32_MAX;
    if (f < -2147483648.0f) return INT32_MIN;
    return (int32_t)f;
}

/* fmax semantics for the OpenCL max() of two floats */
static inline float cl_max(float a, float b) { return fmaxf(a, b); }
/* std::min / std::max semantics (data_loader.hpp:84-86) */
static inline float std_min(float a, float b) { return (b < a) ? b : a; }
static inline float std_max(float a, float b) { return (a < b) ? b : a; }

uint64_t orc_ndrange(uint64_t n) { return n + (32u - n % 32u); }

/* ======================================================================== */
/* one (voxel, projection) pair: detector pixel or "out of bounds"          */
/* ======================================================================== */
/* KernelForward.cl:25-36 / KernelBackward.cl:23-37 under IEEE arithmetic. */
static inline int pair_strict(const orc_projdata *d, float px, float py, float pz,
                              float row_off, int32_t rows, int32_t *iu, int32_t *iv)
{
    const float *m = d->mvp;
    float nu = ((m[0] * px + m[1] * py) + m[2] * pz) + m[3];
    float nv = ((m[4] * px + m[5] * py) + m[6] * pz) + m[7];
    float nw = ((m[12] * px + m[13] * py) + m[14] * pz) + m[15];
    float u = nu / nw;
    float v = nv / nw - row_off;
    int32_t cu = sat_f2i(roundf(u));
    int32_t cv = sat_f2i(roundf(v));
    int in = ((float)cu >= d->vp[0]) && ((float)cv >= d->vp[2]) &&
             ((float)cu < d->vp[1]) && ((float)cv < d->vp[3]) && (cv < rows);
    *iu = cu;
    *iv = cv;
    return in;
}

/* The FAST contract (xpr_oracle.h). */
static inline int pair_fast(const orc_projdata *d, float px, float py, float pz,
                            float hv, float rowsf, int32_t *iu, int32_t *iv)
{
    const float *m = d->mvp;
    float cu = fmaf(m[0], px, m[3]) + m[2] * pz;
    float cv = fmaf(m[4], px, m[7]) + m[6] * pz;
    float cw = fmaf(m[12], px, m[15]) + m[14] * pz;
    float rw = 1.0f / fmaf(m[13], py, cw);
    float yu = fmaf(py, m[1] * rw, fmaf(cu, rw, 0.5f));
    float yv = fmaf(py, m[5] * rw, fmaf(cv, rw, hv));
    int in = (yu >= d->vp[0]) && (yu < d->vp[1]) && (yv >= d->vp[2]) && (yv < d->vp[3]) &&
             (yv < rowsf);
    if (in) {
        *iu = (int32_t)floorf(yu);
        *iv = (int32_t)floorf(yv);
    }
    return in;
}

/* voxel id -> absolute voxel coordinates, to3D() of utils.cl:39-45 plus volumeMin:
 * id = (y * sz + z) * sx + x */
static inline void voxel_coords(uint64_t id, const orc_launch *L, int64_t *x, int64_t *y, int64_t *z)
{
    uint64_t sx = (uint64_t)(L->vmax[0] - L->vmin[0]);
    uint64_t sz = (uint64_t)(L->vmax[2] - L->vmin[2]);
    uint64_t s = sx * sz;
    uint64_t yy = id / s;
    uint64_t r = id - yy * s;
    *y = (int64_t)yy + L->vmin[1];
    *z = (int64_t)(r / sx) + L->vmin[2];
    *x = (int64_t)(r % sx) + L->vmin[0];
}

static inline void voxel_position(const orc_launch *L, int64_t x, int64_t y, int64_t z,
                                  float *px, float *py, float *pz)
{
    if (L->arith == XPR_ARITH_FAST) {
        *px = fmaf((float)x, L->voxel[0], L->origin[0]);
        *py = fmaf((float)y, L->voxel[1], L->origin[1]);
        *pz = fmaf((float)z, L->voxel[2], L->origin[2]);
    } else {
        /* convert_float4(id3d)*voxelSize + origin (KernelForward.cl:26) */
        *px = (float)(uint32_t)x * L->voxel[0] + L->origin[0];
        *py = (float)(uint32_t)y * L->voxel[1] + L->origin[1];
        *pz = (float)(uint32_t)z * L->voxel[2] + L->origin[2];
    }
}

static uint64_t launch_items(const orc_launch *L)
{
    uint64_t n = (uint64_t)(L->vmax[0] - L->vmin[0]) * (uint64_t)(L->vmax[1] - L->vmin[1]) *
                 (uint64_t)(L->vmax[2] - L->vmin[2]);
    return L->compat_pad ? orc_ndrange(n) : n;
}

/* ======================================================================== */
/* Forward (KernelForward.cl:10-55, KernelForwardH.cl:8-37)                 */
/* ======================================================================== */
void orc_forward(const float *vol, uint32_t *sum, const orc_projdata *pd, const orc_launch *L)
{
    const uint64_t items = launch_items(L);
    const uint32_t M = L->modules ? L->modules : 1u;
    const uint32_t n_proj = L->list_mvp ? L->n_list : L->n_angles * M;
    const uint64_t img_stride = (uint64_t)L->det_w * L->rows;
    const float row_off = (float)(uint32_t)L->row_offset;
    const float hv = 0.5f - (float)L->row_offset;
    const float rowsf = (float)L->rows;

#pragma omp parallel for schedule(static, 4096)
    for (int64_t id = 0; id < (int64_t)items; ++id) {
        int64_t x, y, z;
        voxel_coords((uint64_t)id, L, &x, &y, &z);
        float px, py, pz;
        voxel_position(L, x, y, z, &px, &py, &pz);
        const uint32_t value = orc_float_to_fixed(vol[id]);
        for (uint32_t m = 0; m < n_proj; ++m) {
            const orc_projdata *d = L->list_mvp ? &pd[L->list_mvp[m]] : &pd[m];
            const uint64_t img = L->list_mvp ? L->list_img[m] : m / M;
            int32_t cu, cv;
            int in = (L->arith == XPR_ARITH_FAST)
                         ? pair_fast(d, px, py, pz, hv, rowsf, &cu, &cv)
                         : pair_strict(d, px, py, pz, row_off, (int32_t)L->rows, &cu, &cv);
            if (in)
                __atomic_fetch_add(&sum[img * img_stride + (uint64_t)cv * L->det_w + (uint64_t)cu],
                                   value, __ATOMIC_RELAXED);
        }
    }
}

/* ======================================================================== */
/* Backward (KernelBackward.cl:8-40, KernelBackwardH.cl:8-42)               */
/* ======================================================================== */
void orc_backward(float *vol, const float *ratio, const orc_projdata *pd, const orc_launch *L)
{
    const uint64_t items = launch_items(L);
    const uint32_t M = L->modules ? L->modules : 1u;
    const uint32_t n_proj = L->list_mvp ? L->n_list : L->n_angles * M;
    const uint64_t img_stride = (uint64_t)L->det_w * L->rows;
    const float row_off = (float)(uint32_t)L->row_offset;
    const float hv = 0.5f - (float)L->row_offset;
    const float rowsf = (float)L->rows;

#pragma omp parallel for schedule(static, 4096)
    for (int64_t id = 0; id < (int64_t)items; ++id) {
        int64_t x, y, z;
        voxel_coords((uint64_t)id, L, &x, &y, &z);
        float px, py, pz;
        voxel_position(L, x, y, z, &px, &py, &pz);
        float s = 0.0f;
        uint32_t cnt = 0;
        for (uint32_t m = 0; m < n_proj; ++m) {
            const orc_projdata *d = L->list_mvp ? &pd[L->list_mvp[m]] : &pd[m];
            const uint64_t img = L->list_mvp ? L->list_img[m] : m / M;
            int32_t cu, cv;
            int in = (L->arith == XPR_ARITH_FAST)
                         ? pair_fast(d, px, py, pz, hv, rowsf, &cu, &cv)
                         : pair_strict(d, px, py, pz, row_off, (int32_t)L->rows, &cu, &cv);
            if (in) {
                float r = ratio[img * img_stride + (uint64_t)cv * L->det_w + (uint64_t)cu];
                if (L->nan_skip && r != r) continue;
                s += r;
                cnt += 1u;
            }
        }
        vol[id] = vol[id] * orc_expf(s / (float)cnt);
    }
}

/* ======================================================================== */
/* Error (KernelError.cl:8-24) and the method_1c CPU variants               */
/* ======================================================================== */
#define ORC_EPS (1.0f / 4194304.0f)

void orc_error(const float *images, uint32_t *sum_ratio, uint64_t n, float weight)
{
#pragma omp parallel for schedule(static, 65536)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        float ref = images[i];
        float got = orc_fixed_to_float(sum_ratio[i]);
        float r = orc_logf(cl_max(ref / cl_max(got, ORC_EPS), ORC_EPS)) * weight;
        sum_ratio[i] = f2u(r);
    }
}

void orc_error_first_1c(const float *images, float *ratio, uint64_t n)
{
#pragma omp parallel for schedule(static, 65536)
    for (int64_t i = 0; i < (int64_t)n; ++i)
        ratio[i] = orc_logf(std_max(images[i], ORC_EPS));
}

void orc_error_1c(const float *images, uint32_t *sum_ratio, uint64_t n, float weight)
{
#pragma omp parallel for schedule(static, 65536)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        float got = orc_fixed_to_float(sum_ratio[i]);
        float r = orc_logf(std_max(images[i] / std_max(got, ORC_EPS), ORC_EPS)) * weight;
        sum_ratio[i] = f2u(r);
    }
}

/* ======================================================================== */
/* preprocessing (data_loader.hpp:48-101)                                   */
/* ======================================================================== */
void orc_minmax_normal(const float *v, uint64_t n, float *mn, float *mx)
{
    float a = *mn, b = *mx;
    for (uint64_t i = 0; i < n; ++i) {
        if (!isnormal(v[i])) continue;
        if (v[i] < a) a = v[i];
        if (v[i] > b) b = v[i];
    }
    *mn = a;
    *mx = b;
}

void orc_preprocess(float *v, uint64_t n, int normalize, float mn, float mx, int mlog)
{
#pragma omp parallel for schedule(static, 65536)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        float x = v[i];
        if (normalize) x = isnormal(x) ? (x - mn) / (mx - mn) : (mx + mn) / 2.0f;
        if (mlog) x = -orc_logf(std_max(std_min(x, 1.0f - ORC_EPS), ORC_EPS));
        v[i] = x;
    }
}

/* ======================================================================== */
/* geometry, restated from geometry.hpp with glm's column-major semantics  */
/* ======================================================================== */
/* Single precision follows glm's operation order: vec3 dot = (x*x'+y*y')+z*z',
 * normalize(v) = v * (1/sqrt(dot(v,v))), cross as usual, mat4(16 scalars) fills
 * columns, (A*B)[j] = ((A0*B[j][0] + A1*B[j][1]) + A2*B[j][2]) + A3*B[j][3]. */
typedef struct { float x, y, z; } v3f;
typedef struct { double x, y, z; } v3d;
typedef struct { float c[4][4]; } m4f;   /* c[col][row] */
typedef struct { double c[4][4]; } m4d;

static v3f v3f_add(v3f a, v3f b) { v3f r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static v3f v3f_sub(v3f a, v3f b) { v3f r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v3f v3f_mul(v3f a, float s) { v3f r = {a.x * s, a.y * s, a.z * s}; return r; }
static float v3f_dot(v3f a, v3f b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static v3f v3f_cross(v3f a, v3f b)
{
    v3f r = {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
    return r;
}
static v3f v3f_norm(v3f a) { return v3f_mul(a, 1.0f / sqrtf(v3f_dot(a, a))); }
static float glm_radians_f(float d) { return d * 0x1.1df46ap-6f; }
static float glm_degrees_f(float r) { return r * 0x1.ca5dc2p+5f; }
/* rotate(vec, origin, x, y, z) of geometry.hpp:88-95: rotateX, rotateY, rotateZ */
static v3f rotate_xyz_f(v3f vec, v3f o, float ax, float ay, float az)
{
    v3f v = v3f_sub(vec, o), t;
    float c = cosf(glm_radians_f(ax)), s = sinf(glm_radians_f(ax));
    t = v; t.y = v.y * c - v.z * s; t.z = v.y * s + v.z * c; v = t;
    c = cosf(glm_radians_f(ay)); s = sinf(glm_radians_f(ay));
    t = v; t.x = v.x * c + v.z * s; t.z = -v.x * s + v.z * c; v = t;
    c = cosf(glm_radians_f(az)); s = sinf(glm_radians_f(az));
    t = v; t.x = v.x * c - v.y * s; t.y = v.x * s + v.y * c; v = t;
    return v3f_add(v, o);
}
/* rotation of v about a unit axis (Rodrigues), used by the per-module extension */
static v3f rotate_axis_f(v3f v, float angle_rad, v3f k)
{
    float c = cosf(angle_rad), s = sinf(angle_rad);
    v3f kxv = v3f_cross(k, v);
    float kd = v3f_dot(k, v) * (1.0f - c);
    v3f r = v3f_add(v3f_add(v3f_mul(v, c), v3f_mul(kxv, s)), v3f_mul(k, kd));
    return r;
}
static m4f m4f_rows(const float r[16])
{
    /* glm::mat4(a0..a15): a0..a3 is column 0 */
    m4f m;
    for (int i = 0; i < 16; ++i) m.c[i / 4][i % 4] = r[i];
    return m;
}
static m4f m4f_mul(m4f A, m4f B)
{
    m4f R;
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 4; ++i)
            R.c[j][i] = ((A.c[0][i] * B.c[j][0] + A.c[1][i] * B.c[j][1]) + A.c[2][i] * B.c[j][2]) +
                        A.c[3][i] * B.c[j][3];
    return R;
}

static v3d v3d_add(v3d a, v3d b) { v3d r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static v3d v3d_sub(v3d a, v3d b) { v3d r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v3d v3d_mul(v3d a, double s) { v3d r = {a.x * s, a.y * s, a.z * s}; return r; }
static double v3d_dot(v3d a, v3d b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static v3d v3d_cross(v3d a, v3d b)
{
    v3d r = {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
    return r;
}
static v3d v3d_norm(v3d a) { return v3d_mul(a, 1.0 / sqrt(v3d_dot(a, a))); }
#define ORC_DEG2RAD 0.017453292519943295769
static v3d rotate_xyz_d(v3d vec, v3d o, double ax, double ay, double az)
{
    v3d v = v3d_sub(vec, o), t;
    double c = cos(ax * ORC_DEG2RAD), s = sin(ax * ORC_DEG2RAD);
    t = v; t.y = v.y * c - v.z * s; t.z = v.y * s + v.z * c; v = t;
    c = cos(ay * ORC_DEG2RAD); s = sin(ay * ORC_DEG2RAD);
    t = v; t.x = v.x * c + v.z * s; t.z = -v.x * s + v.z * c; v = t;
    c = cos(az * ORC_DEG2RAD); s = sin(az * ORC_DEG2RAD);
    t = v; t.x = v.x * c - v.y * s; t.y = v.x * s + v.y * c; v = t;
    return v3d_add(v, o);
}
static v3d rotate_axis_d(v3d v, double angle_rad, v3d k)
{
    double c = cos(angle_rad), s = sin(angle_rad);
    v3d kxv = v3d_cross(k, v);
    double kd = v3d_dot(k, v) * (1.0 - c);
    return v3d_add(v3d_add(v3d_mul(v, c), v3d_mul(kxv, s)), v3d_mul(k, kd));
}
static m4d m4d_rows(const double r[16])
{
    m4d m;
    for (int i = 0; i < 16; ++i) m.c[i / 4][i % 4] = r[i];
    return m;
}
static m4d m4d_mul(m4d A, m4d B)
{
    m4d R;
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 4; ++i)
            R.c[j][i] = ((A.c[0][i] * B.c[j][0] + A.c[1][i] * B.c[j][1]) + A.c[2][i] * B.c[j][2]) +
                        A.c[3][i] * B.c[j][3];
    return R;
}

/* computeGeneralizedProjection (geometry.hpp:182-234), single precision */
static m4f gen_proj_f(v3f pe, v3f pa, v3f pb, v3f pc, float vpl, float vpr, float vpb, float vpt,
                      float sd)
{
    v3f vr = v3f_norm(v3f_sub(pb, pa));
    v3f vu = v3f_norm(v3f_sub(pc, pa));
    v3f vn = v3f_norm(v3f_cross(vu, vr));
    v3f va = v3f_sub(pa, pe), vb = v3f_sub(pb, pe), vc = v3f_sub(pc, pe);
    float d = -v3f_dot(va, vn);
    float n = 1.0f, f = sd * 2.0f;
    float l = v3f_dot(vr, va) * (n / d);
    float r = v3f_dot(vr, vb) * (n / d);
    float b = v3f_dot(vu, va) * (n / d);
    float t = v3f_dot(vu, vc) * (n / d);
    const float P[16] = {(2.0f * n) / (r - l), 0.0f, (r + l) / (r - l), 0.0f,
                         0.0f, (2.0f * n) / (t - b), (t + b) / (t - b), 0.0f,
                         0.0f, 0.0f, -(f + n) / (f - n), -(2.0f * f * n) / (f - n),
                         0.0f, 0.0f, -1.0f, 0.0f};
    const float Mt[16] = {vr.x, vr.y, vr.z, 0.0f, vu.x, vu.y, vu.z, 0.0f,
                          vn.x, vn.y, vn.z, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f};
    const float T[16] = {1.0f, 0.0f, 0.0f, -pe.x, 0.0f, 1.0f, 0.0f, -pe.y,
                         0.0f, 0.0f, 1.0f, -pe.z, 0.0f, 0.0f, 0.0f, 1.0f};
    const float S[16] = {(vpr - vpl) * 0.5f, 0.0f, 0.0f, (vpr + vpl) * 0.5f,
                         0.0f, (vpt - vpb) * 0.5f, 0.0f, (vpt + vpb) * 0.5f,
                         0.0f, 0.0f, 0.5f, 0.5f, 0.0f, 0.0f, 0.0f, 1.0f};
    return m4f_mul(m4f_mul(m4f_mul(m4f_rows(T), m4f_rows(Mt)), m4f_rows(P)), m4f_rows(S));
}

static m4d gen_proj_d(v3d pe, v3d pa, v3d pb, v3d pc, double vpl, double vpr, double vpb, double vpt,
                      double sd)
{
    v3d vr = v3d_norm(v3d_sub(pb, pa));
    v3d vu = v3d_norm(v3d_sub(pc, pa));
    v3d vn = v3d_norm(v3d_cross(vu, vr));
    v3d va = v3d_sub(pa, pe), vb = v3d_sub(pb, pe), vc = v3d_sub(pc, pe);
    double d = -v3d_dot(va, vn);
    double n = 1.0, f = sd * 2.0;
    double l = v3d_dot(vr, va) * (n / d);
    double r = v3d_dot(vr, vb) * (n / d);
    double b = v3d_dot(vu, va) * (n / d);
    double t = v3d_dot(vu, vc) * (n / d);
    const double P[16] = {(2.0 * n) / (r - l), 0.0, (r + l) / (r - l), 0.0,
                          0.0, (2.0 * n) / (t - b), (t + b) / (t - b), 0.0,
                          0.0, 0.0, -(f + n) / (f - n), -(2.0 * f * n) / (f - n),
                          0.0, 0.0, -1.0, 0.0};
    const double Mt[16] = {vr.x, vr.y, vr.z, 0.0, vu.x, vu.y, vu.z, 0.0,
                           vn.x, vn.y, vn.z, 0.0, 0.0, 0.0, 0.0, 1.0};
    const double T[16] = {1.0, 0.0, 0.0, -pe.x, 0.0, 1.0, 0.0, -pe.y,
                          0.0, 0.0, 1.0, -pe.z, 0.0, 0.0, 0.0, 1.0};
    const double S[16] = {(vpr - vpl) * 0.5, 0.0, 0.0, (vpr + vpl) * 0.5,
                          0.0, (vpt - vpb) * 0.5, 0.0, (vpt + vpb) * 0.5,
                          0.0, 0.0, 0.5, 0.5, 0.0, 0.0, 0.0, 1.0};
    return m4d_mul(m4d_mul(m4d_mul(m4d_rows(T), m4d_rows(Mt)), m4d_rows(P)), m4d_rows(S));
}

/* The geometry of orc_geometry in double precision end to end (matrices kept in double):
 * column-major mvp (16 per entry) and viewport {l, r, b, t} (4 per entry). */
static void geometry_f64(const orc_geom_params *gp, int64_t P, int64_t M, uint64_t width, uint64_t height,
                         double *mvp_out, double *vp_out)
{
    const double so = gp->so, sd = gp->sd, px = gp->px;
    v3d dsource_pos = {0.0, 0.0, 0.0};
    v3d dsource_at = {0.0, 0.0, sd};
    v3d daxis = v3d_add(dsource_at, (v3d){-(double)gp->sx + (double)gp->rx_px * px, -(double)gp->sy, 0.0});
    v3d dcenter = v3d_mul(v3d_norm(daxis), so);
    dsource_pos = v3d_sub(dsource_pos, dcenter);
    dsource_at = v3d_sub(dsource_at, dcenter);
    v3d zero = {0.0, 0.0, 0.0};
    for (int64_t i = 0; i < P; ++i) {
        double heli = ((double)gp->heli_offset / (double)P) * (double)i - (double)gp->heli_offset * 0.5;
        double angle_deg = gp->angle_list ? (double)gp->angle_list[i] : (double)i * ((double)gp->angle / (double)P);
        v3d rsp = v3d_add(rotate_xyz_d(dsource_pos, zero, 0.0, angle_deg, 0.0), (v3d){0.0, heli, 0.0});
        v3d rsa = v3d_add(rotate_xyz_d(dsource_at, zero, 0.0, angle_deg, 0.0), (v3d){0.0, heli, 0.0});
        for (int64_t mod = 0; mod < M; ++mod) {
            v3d vv = {0.0, 1.0, 0.0};
            v3d dir = v3d_sub(rsa, rsp);
            v3d u = v3d_norm(v3d_cross(vv, dir));
            v3d nrm = v3d_norm(dir);
            v3d detector = v3d_sub(v3d_sub(rsa, v3d_mul(u, gp->sx)), v3d_mul(vv, gp->sy));
            if (gp->mod_offset) {
                const float *o = gp->mod_offset + 3 * mod;
                detector = v3d_add(detector, v3d_add(v3d_add(v3d_mul(u, o[0] * px), v3d_mul(vv, o[1] * px)),
                                                     v3d_mul(nrm, o[2] * px)));
            }
            v3d ul = v3d_sub(v3d_sub(detector, v3d_mul(u, 0.5 * (double)width * px)),
                             v3d_mul(vv, 0.5 * (double)height * px));
            v3d ur = v3d_add(ul, v3d_mul(u, (double)width * px));
            v3d bl = v3d_add(ul, v3d_mul(vv, (double)height * px));
            if (gp->mod_rpy) {
                const float *a = gp->mod_rpy + 3 * mod;
                v3d *cs[3] = {&ul, &ur, &bl};
                for (int c = 0; c < 3; ++c) {
                    v3d w = v3d_sub(*cs[c], detector);
                    w = rotate_axis_d(w, a[2] * ORC_DEG2RAD, u);
                    w = rotate_axis_d(w, a[1] * ORC_DEG2RAD, vv);
                    w = rotate_axis_d(w, a[0] * ORC_DEG2RAD, nrm);
                    *cs[c] = v3d_add(w, detector);
                }
            }
            v3d center = detector;
            v3d mc = v3d_add(center, v3d_mul(v3d_norm(v3d_sub(rsp, rsa)), sd - (double)gp->module_center_offset_z));
            double dist = sqrt(v3d_dot(v3d_sub(center, mc), v3d_sub(center, mc)));
            double mang = gp->module_angle_offset_set
                              ? (double)gp->module_angle_offset
                              : (2.0 * atan2((double)width * 0.5 * px, dist)) * 57.295779513082320877;
            double mcur = mang * ((double)mod - floor((double)M / 2.0));
            v3d pa = rotate_xyz_d(ul, mc, 0.0, mcur, 0.0);
            v3d pb = rotate_xyz_d(ur, mc, 0.0, mcur, 0.0);
            v3d pc = rotate_xyz_d(bl, mc, 0.0, mcur, 0.0);
            double vpl = (double)(width * (uint64_t)mod), vpr = (double)(width * (uint64_t)(mod + 1));
            m4d mvp = gen_proj_d(rsp, pa, pb, pc, vpl, vpr, 0.0, (double)gp->dheight, sd);
            double *om = mvp_out + (i * M + mod) * 16, *ov = vp_out + (i * M + mod) * 4;
            for (int c = 0; c < 4; ++c)
                for (int r = 0; r < 4; ++r) om[c * 4 + r] = mvp.c[c][r];
            ov[0] = vpl; ov[1] = vpr; ov[2] = 0.0; ov[3] = (double)gp->dheight;
        }
    }
}

int orc_geometry(const orc_geom_params *gp, int fp64, orc_projdata *out, orc_geom_out *go)
{
    const int64_t P = gp->projections, M = gp->module_number;
    /* geometry.hpp:49-68 */
    const float rx = gp->rx_px * gp->px;                       /* parameters.hpp:39 */
    go->vx = gp->px * (gp->so / gp->sd);
    go->vwidth = gp->dwidth;
    go->vheight = gp->dheight + (int64_t)fabsf(gp->heli_offset / go->vx);
    go->concurrent = (int64_t)floorf((float)P / (float)gp->sit);
    const uint64_t width = (uint64_t)gp->dwidth / (uint64_t)M;
    const uint64_t height = (uint64_t)gp->dheight;
    /* the voxel grid (vx, orig) is single precision in both modes */
    v3f source_pos = {0.0f, 0.0f, 0.0f};
    v3f source_at = v3f_add(source_pos, (v3f){0.0f, 0.0f, gp->sd});
    v3f axis_proj = v3f_add(source_at, (v3f){-gp->sx + rx, -gp->sy, 0.0f});
    v3f object_center = v3f_add(source_pos, v3f_mul(v3f_norm(v3f_sub(axis_proj, source_pos)), gp->so));
    source_pos = v3f_sub(source_pos, object_center);
    source_at = v3f_sub(source_at, object_center);
    object_center = (v3f){0.0f, 0.0f, 0.0f};
    go->orig[0] = object_center.x + -0.5f * (float)go->vwidth * go->vx;
    go->orig[1] = object_center.y + -0.5f * (float)go->vheight * go->vx;
    go->orig[2] = object_center.z + -0.5f * (float)go->vwidth * go->vx;

    if (!fp64) {

        for (int64_t i = 0; i < P; ++i) {
            /* computeDetectorProjection (geometry.hpp:267-292) */
            float heli = (gp->heli_offset / (float)P) * (float)i - gp->heli_offset * 0.5f;
            float angle_deg = gp->angle_list ? gp->angle_list[i] : (float)i * (gp->angle / (float)P);
            v3f rsp = v3f_add(rotate_xyz_f(source_pos, object_center, 0.0f, angle_deg, 0.0f), (v3f){0.0f, heli, 0.0f});
            v3f rsa = v3f_add(rotate_xyz_f(source_at, object_center, 0.0f, angle_deg, 0.0f), (v3f){0.0f, heli, 0.0f});
            for (int64_t mod = 0; mod < M; ++mod) {
                /* detectorFromSource (geometry.hpp:244-265) */
                v3f vv = {0.0f, 1.0f, 0.0f};
                v3f dir = v3f_sub(rsa, rsp);
                v3f u = v3f_norm(v3f_cross(vv, dir));
                v3f nrm = v3f_norm(dir);
                v3f detector = v3f_sub(v3f_sub(rsa, v3f_mul(u, gp->sx)), v3f_mul(vv, gp->sy));
                if (gp->mod_offset) {
                    const float *o = gp->mod_offset + 3 * mod;
                    detector = v3f_add(detector, v3f_add(v3f_add(v3f_mul(u, o[0] * gp->px), v3f_mul(vv, o[1] * gp->px)),
                                                         v3f_mul(nrm, o[2] * gp->px)));
                }
                v3f ul = v3f_sub(v3f_sub(detector, v3f_mul(u, 0.5f * (float)width * gp->px)),
                                 v3f_mul(vv, 0.5f * (float)height * gp->px));
                v3f ur = v3f_add(ul, v3f_mul(u, (float)width * gp->px));
                v3f bl = v3f_add(ul, v3f_mul(vv, (float)height * gp->px));
                if (gp->mod_rpy) {
                    const float *a = gp->mod_rpy + 3 * mod; /* roll, pitch, yaw */
                    v3f *cs[3] = {&ul, &ur, &bl};
                    for (int c = 0; c < 3; ++c) {
                        v3f w = v3f_sub(*cs[c], detector);
                        w = rotate_axis_f(w, glm_radians_f(a[2]), u);
                        w = rotate_axis_f(w, glm_radians_f(a[1]), vv);
                        w = rotate_axis_f(w, glm_radians_f(a[0]), nrm);
                        *cs[c] = v3f_add(w, detector);
                    }
                }
                v3f center = detector;
                v3f mc = v3f_add(center, v3f_mul(v3f_norm(v3f_sub(rsp, rsa)), gp->sd - gp->module_center_offset_z));
                float dist = sqrtf(v3f_dot(v3f_sub(center, mc), v3f_sub(center, mc)));
                float mang = gp->module_angle_offset_set
                                 ? gp->module_angle_offset
                                 : glm_degrees_f(2.0f * atan2f((float)width * 0.5f * gp->px, dist));
                float mcur = mang * ((float)mod - floorf((float)M / 2.0f));
                v3f pa = rotate_xyz_f(ul, mc, 0.0f, mcur, 0.0f);
                v3f pb = rotate_xyz_f(ur, mc, 0.0f, mcur, 0.0f);
                v3f pc = rotate_xyz_f(bl, mc, 0.0f, mcur, 0.0f);
                float vpl = (float)(width * (uint64_t)mod), vpr = (float)(width * (uint64_t)(mod + 1));
                float vpb = 0.0f, vpt = (float)gp->dheight;
                m4f mvp = gen_proj_f(rsp, pa, pb, pc, vpl, vpr, vpb, vpt, gp->sd);
                orc_projdata *o = &out[i * M + mod];
                for (int c = 0; c < 4; ++c)
                    for (int r = 0; r < 4; ++r) o->mvp[c * 4 + r] = mvp.c[c][r];
                o->vp[0] = vpl; o->vp[1] = vpr; o->vp[2] = vpb; o->vp[3] = vpt;
            }
        }
    } else {
        double *dm = (double *)malloc(sizeof(double) * (size_t)(P * M * 16));
        double *dv = (double *)malloc(sizeof(double) * (size_t)(P * M * 4));
        geometry_f64(gp, P, M, width, height, dm, dv);
        for (int64_t k = 0; k < P * M; ++k) {
            for (int j = 0; j < 16; ++j) out[k].mvp[j] = (float)dm[k * 16 + j];
            for (int j = 0; j < 4; ++j) out[k].vp[j] = (float)dv[k * 4 + j];
        }
        free(dm);
        free(dv);
    }
    return 0;
}

/* point * mvp / w, y component (geometry.hpp:135-139; geometry_chunk.hpp:58-62) */
static float project_y(const orc_projdata *d, float x, float y, float z)
{
    const float *m = d->mvp;
    float py = ((m[4] * x + m[5] * y) + m[6] * z) + m[7] * 1.0f;
    float pw = ((m[12] * x + m[13] * y) + m[14] * z) + m[15] * 1.0f;
    return py / pw;
}

int orc_cull_layer(const orc_geom_params *gp, const orc_geom_out *go, const orc_projdata *all,
                   int64_t sit, int64_t layer, int per_module, uint16_t *mvp_idx, uint16_t *img_idx)
{
    const int64_t P = gp->projections, S = gp->sit, M = gp->module_number;
    const float ox = go->orig[0], oy = go->orig[1], oz = go->orig[2];
    const float bx[8] = {ox, -ox, ox, -ox, ox, -ox, ox, -ox};
    const float by[8] = {oy - 1.0f, oy - 1.0f, oy - 1.0f, oy - 1.0f, oy + 1.0f, oy + 1.0f, oy + 1.0f, oy + 1.0f};
    const float bz[8] = {-oz, -oz, oz, oz, -oz, -oz, oz, oz};
    int n = 0;
    uint16_t slot = 0;
    for (int64_t i = sit; i < P; i += S) {
        for (int64_t mod = 0; mod < M; ++mod) {
            const int64_t k = per_module ? i * M + mod : i;
            const orc_projdata *d = &all[k];
            /* minmaxLayerProj (geometry.hpp:334-355) */
            int64_t mn = go->vheight * 2, mx = -go->vheight;
            for (int j = 0; j < 8; ++j) {
                float y = by[j] + (float)(uint32_t)layer * go->vx;
                int64_t line = (int64_t)project_y(d, bx[j], y, bz[j]);
                if (line < mn) mn = line;
                if (line > mx) mx = line;
            }
            float fmn = (float)mn, fmx = (float)mx;
            if (!(fmn >= d->vp[3] && fmx >= d->vp[3]) && !(fmn < d->vp[2] && fmx < d->vp[2])) {
                mvp_idx[n] = (uint16_t)k;
                img_idx[n] = slot;
                ++n;
            }
        }
        ++slot;
    }
    return n;
}

/* ======================================================================== */
/* method_2 chunk planner (geometry_chunk.hpp:62-197)                       */
/* ======================================================================== */
typedef struct { int64_t vOffset, vSize, iOffset, iSize, vPadTop, vPadBot; } orc_chunk;

typedef struct {
    const orc_geom_params *gp;
    const orc_geom_out *go;
    float *ymin, *ymax;
    uint64_t avail, max_alloc;
    float overlap;
} chunk_ctx;

static void y_projection(const chunk_ctx *c, int64_t off, int64_t h, float *a, float *b)
{
    /* std::min / std::max of two floats */
    *a = std_min(c->ymin[off], c->ymin[off + h - 1]);
    *b = std_max(c->ymax[off], c->ymax[off + h - 1]);
}

static void update_image_viewport(const chunk_ctx *c, orc_chunk *ch)
{
    float a, b;
    y_projection(c, ch->vOffset, ch->vSize, &a, &b);
    ch->iOffset = (int64_t)std_max(floorf(a) - 1.0f, 0.0f);
    ch->iSize = (int64_t)std_max(std_min(ceilf(b - (float)ch->iOffset) + 2.0f,
                                         (float)(c->gp->dheight - ch->iOffset)), 0.0f);
}

static void update_volume_padding(const chunk_ctx *c, orc_chunk *ch)
{
    ch->vPadTop = 0;
    ch->vPadBot = 0;
    float a, b;
    while (ch->vOffset - ch->vPadTop > 0) {
        y_projection(c, ch->vOffset - ch->vPadTop, 1, &a, &b);
        if (!(b > (float)(ch->iOffset - 1))) break;
        ++ch->vPadTop;
    }
    while (ch->vOffset + ch->vSize + ch->vPadBot < c->go->vheight - 1) {
        y_projection(c, ch->vOffset + ch->vSize + ch->vPadBot, 1, &a, &b);
        if (!(a < (float)(ch->iOffset + ch->iSize + 1))) break;
        ++ch->vPadBot;
    }
    ch->vPadTop = (int64_t)ceilf((float)ch->vPadTop * c->overlap);
    ch->vPadBot = (int64_t)ceilf((float)ch->vPadBot * c->overlap);
}

static int fit_in_memory(const chunk_ctx *c, const orc_chunk *ch)
{
    const int64_t W = c->go->vwidth, layer = W * W, line = c->gp->dwidth, Pc = c->go->concurrent;
    uint64_t total = (uint64_t)(((ch->vSize + ch->vPadTop + ch->vPadBot) * layer + 2 * ch->iSize * line * Pc) * 4);
    uint64_t images = (uint64_t)(ch->iSize * line * Pc * 4);
    int64_t padmax = ch->vPadBot > ch->vPadTop ? ch->vPadBot : ch->vPadTop;
    uint64_t padding = (uint64_t)(padmax * layer * 4);
    return c->avail > total && c->max_alloc - 1 > images && c->max_alloc > padding;
}

int orc_plan_chunks(const orc_geom_params *gp, const orc_geom_out *go, const orc_projdata *all,
                    uint64_t avail_bytes, uint64_t max_alloc_bytes, float overlap_fct,
                    int64_t *chunks, int max_chunks)
{
    const int64_t H = go->vheight, PM = gp->projections * gp->module_number;
    chunk_ctx c = {gp, go, malloc(sizeof(float) * H), malloc(sizeof(float) * H), avail_bytes, max_alloc_bytes,
                   overlap_fct > 1.0f ? 1.0f : (overlap_fct < 0.01f ? 0.01f : overlap_fct)};
    const float ox = go->orig[0], oy = go->orig[1], oz = go->orig[2];
    const float bx[4] = {ox, -ox, ox, -ox}, bz[4] = {-oz, -oz, oz, oz};
    /* computeLayerYBounds (geometry_chunk.hpp:120-145) */
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < H; ++l) {
        float mn = INFINITY, mx = -INFINITY;
        const float yt = oy + (float)(int)l * go->vx;
        const float yb = oy + (float)(int)(l + 1) * go->vx;
        for (int64_t i = 0; i < PM; ++i)
            for (int j = 0; j < 4; ++j) {
                float a = project_y(&all[i], bx[j], yt, bz[j]);
                float b = project_y(&all[i], bx[j], yb, bz[j]);
                if (a < mn) mn = a;
                if (b < mn) mn = b;
                if (mx < a) mx = a;
                if (mx < b) mx = b;
            }
        c.ymin[l] = mn;
        c.ymax[l] = mx;
    }
    /* computeChunks (geometry_chunk.hpp:92-114) */
    int64_t first = 0, last = 0;
    while (first < H && !(0.0f < c.ymin[first])) ++first;
    while (last < H && !((float)(H - 1) < c.ymax[last])) ++last;
    int n = 1;
    orc_chunk *ch = (orc_chunk *)chunks;
    memset(&ch[0], 0, sizeof(orc_chunk));
    ch[0].vOffset = first;
    for (int64_t i = 0; i < last - first; ++i) {
        orc_chunk t = ch[n - 1];
        ++t.vSize;
        update_image_viewport(&c, &t);
        update_volume_padding(&c, &t);
        if (fit_in_memory(&c, &t)) {
            ch[n - 1] = t;
        } else {
            if (t.vSize <= 1 || n >= max_chunks) { n = -1; break; }
            memset(&ch[n], 0, sizeof(orc_chunk));
            ch[n].vOffset = ch[n - 1].vOffset + ch[n - 1].vSize;
            ++n;
        }
    }
    free(c.ymin);
    free(c.ymax);
    return n;
}

/* ======================================================================== */
/* whole reconstructions                                                    */
/* ======================================================================== */
static void jitter_origin(orc_mt19937 *g, const orc_geom_out *go, float o[3])
{
    for (int i = 0; i < 3; ++i) o[i] = go->orig[i] + orc_uniform_float(g, 0.0f, go->vx);
}

/* first Pc images of sub-iteration `sit`, packed (dataset.hpp:133-140), rows
 * [row0, row0 + rows) of each image */
static float *gather_subset(const orc_geom_params *gp, int64_t Pc, int64_t sit, const float *images,
                            int64_t row0, int64_t rows)
{
    const int64_t W = gp->dwidth, H = gp->dheight;
    float *o = (float *)malloc(sizeof(float) * (size_t)(Pc * W * rows) + 4);
    for (int64_t k = 0; k < Pc; ++k)
        memcpy(o + k * W * rows, images + (sit + k * gp->sit) * W * H + row0 * W, sizeof(float) * (size_t)(W * rows));
    return o;
}

int orc_recon_naive(const orc_geom_params *gp, const orc_recon_params *rp, const float *images, float *vol)
{
    orc_geom_out go;
    const int64_t P = gp->projections, M = gp->module_number, S = rp->sit;
    orc_geom_params g = *gp;
    g.sit = S;
    orc_projdata *all = (orc_projdata *)malloc(sizeof(orc_projdata) * (size_t)(P * M));
    orc_geometry(&g, 0, all, &go);
    const int64_t Pc = go.concurrent, W = go.vwidth, Hv = go.vheight, Wd = gp->dwidth, Hd = gp->dheight;
    if (Pc <= 0) { free(all); return -1; }
    /* per-subset ProjData (geometry.hpp:306-327): angles sit, sit+S, ... */
    orc_projdata *pd = (orc_projdata *)malloc(sizeof(orc_projdata) * (size_t)(S * Pc * M));
    for (int64_t s = 0; s < S; ++s)
        for (int64_t k = 0; k < Pc; ++k)
            for (int64_t mod = 0; mod < M; ++mod) pd[(s * Pc + k) * M + mod] = all[(s + k * S) * M + mod];
    const uint64_t n_sum = (uint64_t)(Pc * Wd * Hd);
    uint32_t *sum = (uint32_t *)malloc(sizeof(uint32_t) * n_sum);
    const uint64_t nvox = (uint64_t)(W * Hv * W);
    const uint64_t nbuf = rp->compat_pad ? orc_ndrange(nvox) : nvox;
    for (uint64_t i = 0; i < nbuf; ++i) vol[i] = 1.0f;          /* reconstruction_n.hpp:59 */
    for (uint64_t i = 0; i < n_sum; ++i) sum[i] = ORC_FIXED_ONE; /* :60 */
    orc_mt19937 gen;
    orc_mt_seed(&gen, rp->seed);
    orc_launch L;
    memset(&L, 0, sizeof(L));
    L.vmax[0] = (int32_t)W; L.vmax[1] = (int32_t)Hv; L.vmax[2] = (int32_t)W;
    L.voxel[0] = L.voxel[1] = L.voxel[2] = go.vx;
    L.det_w = (uint32_t)Wd; L.rows = (uint32_t)Hd; L.row_offset = 0;
    L.n_angles = (uint32_t)Pc; L.modules = (uint32_t)M;
    L.arith = rp->arith; L.compat_pad = rp->compat_pad;
    float weight = rp->weight;
    for (int64_t mit = 0; mit < rp->it; ++mit) {
        for (int64_t sit = 0; sit < S; ++sit) {
            jitter_origin(&gen, &go, L.origin);
            float *img = gather_subset(gp, Pc, sit, images, 0, Hd);
            const orc_projdata *spd = pd + sit * Pc * M;
            if (sit > 0 || mit > 0) orc_forward(vol, sum, spd, &L);
            orc_error(img, sum, n_sum, weight);
            orc_backward(vol, (const float *)sum, spd, &L);
            memset(sum, 0, sizeof(uint32_t) * n_sum);
            free(img);
        }
        weight *= rp->weight_factor;
    }
    free(sum);
    free(pd);
    free(all);
    return 0;
}

int orc_recon_1c(const orc_geom_params *gp, const orc_recon_params *rp, const float *images, float *vol)
{
    orc_geom_out go;
    const int64_t P = gp->projections, M = gp->module_number, S = rp->sit;
    orc_geom_params g = *gp;
    g.sit = S;
    orc_projdata *all = (orc_projdata *)malloc(sizeof(orc_projdata) * (size_t)(P * M));
    orc_geometry(&g, 0, all, &go);
    const int64_t Pc = go.concurrent, W = go.vwidth, Hv = go.vheight, Wd = gp->dwidth, Hd = gp->dheight;
    if (Pc <= 0) { free(all); return -1; }
    const int64_t slots = Pc + 1; /* reconstruction_lplh.hpp:41 */
    const uint64_t n_img = (uint64_t)(Wd * Hd);
    uint32_t *sum = (uint32_t *)calloc((size_t)(slots * n_img), sizeof(uint32_t));
    uint16_t *li = (uint16_t *)malloc(sizeof(uint16_t) * (size_t)(slots * M + 1));
    uint16_t *lm = (uint16_t *)malloc(sizeof(uint16_t) * (size_t)(slots * M + 1));
    orc_mt19937 gen;
    orc_mt_seed(&gen, rp->seed);
    orc_launch L;
    memset(&L, 0, sizeof(L));
    L.voxel[0] = L.voxel[1] = L.voxel[2] = go.vx;
    L.det_w = (uint32_t)Wd; L.rows = (uint32_t)Hd;
    L.modules = (uint32_t)M; L.arith = rp->arith;
    L.list_mvp = li; L.list_img = lm;
    float weight = rp->weight;
    const float init = 1.0f / (float)sqrt((double)(W * W)); /* :194 */
    for (int64_t mit = 0; mit < rp->it; ++mit) {
        for (int64_t sit = 0; sit < S; ++sit) {
            jitter_origin(&gen, &go, L.origin);
            const int first = (sit == 0 && mit == 0);
            memset(sum, 0, sizeof(uint32_t) * (size_t)(slots * n_img));
            if (!first) {
                for (int64_t l = 0; l < Hv; ++l) {
                    L.n_list = (uint32_t)orc_cull_layer(gp, &go, all, sit, l, M > 1, li, lm);
                    L.vmin[0] = 0; L.vmin[1] = (int32_t)l; L.vmin[2] = 0;
                    L.vmax[0] = (int32_t)W; L.vmax[1] = (int32_t)l + 1; L.vmax[2] = (int32_t)W;
                    L.nan_skip = 0;
                    orc_forward(vol + l * W * W, sum, all, &L);
                }
            }
            /* error on every image of the subset (:140-178) */
            for (int64_t j = sit, id = 0; j < P; j += S, ++id) {
                const float *ref = images + j * n_img;
                if (first) orc_error_first_1c(ref, (float *)(sum + id * n_img), n_img);
                else orc_error_1c(ref, sum + id * n_img, n_img, weight);
            }
            for (int64_t l = 0; l < Hv; ++l) {
                float *layer = vol + l * W * W;
                if (first)
                    for (int64_t i = 0; i < W * W; ++i) layer[i] = init;
                L.n_list = (uint32_t)orc_cull_layer(gp, &go, all, sit, l, M > 1, li, lm);
                L.vmin[0] = 0; L.vmin[1] = (int32_t)l; L.vmin[2] = 0;
                L.vmax[0] = (int32_t)W; L.vmax[1] = (int32_t)l + 1; L.vmax[2] = (int32_t)W;
                L.nan_skip = 1;
                orc_backward(layer, (const float *)sum, all, &L);
            }
        }
        weight *= rp->weight_factor;
    }
    free(li);
    free(lm);
    free(sum);
    free(all);
    return 0;
}

int orc_recon_chunks(const orc_geom_params *gp, const orc_recon_params *rp, const float *images,
                     const int64_t *chunks, int n_chunks, float *vol)
{
    orc_geom_out go;
    const int64_t P = gp->projections, M = gp->module_number, S = rp->sit;
    orc_geom_params g = *gp;
    g.sit = S;
    orc_projdata *all = (orc_projdata *)malloc(sizeof(orc_projdata) * (size_t)(P * M));
    orc_geometry(&g, 0, all, &go);
    const int64_t Pc = go.concurrent, W = go.vwidth, Wd = gp->dwidth;
    if (Pc <= 0) { free(all); return -1; }
    orc_projdata *pd = (orc_projdata *)malloc(sizeof(orc_projdata) * (size_t)(S * Pc * M));
    for (int64_t s = 0; s < S; ++s)
        for (int64_t k = 0; k < Pc; ++k)
            for (int64_t mod = 0; mod < M; ++mod) pd[(s * Pc + k) * M + mod] = all[(s + k * S) * M + mod];
    orc_mt19937 gen;
    orc_mt_seed(&gen, rp->seed);
    const orc_chunk *ch = (const orc_chunk *)chunks;
    for (int c = 0; c < n_chunks; ++c) {
        const orc_chunk k = ch[c];
        if (k.vSize <= 0) continue;
        /* one slab [vOffset - vPadTop, vOffset + vSize + vPadBot) initialised to 1
         * (reconstruction_chunk.hpp:57-72; the 6 sub-buffers only split launches) */
        const int64_t y0 = k.vOffset - k.vPadTop, ny = k.vPadTop + k.vSize + k.vPadBot;
        float *slab = (float *)malloc(sizeof(float) * (size_t)(ny * W * W));
        for (int64_t i = 0; i < ny * W * W; ++i) slab[i] = 1.0f;
        const uint64_t n_sum = (uint64_t)(Pc * Wd * k.iSize);
        uint32_t *sum = (uint32_t *)malloc(sizeof(uint32_t) * n_sum + 4);
        for (uint64_t i = 0; i < n_sum; ++i) sum[i] = ORC_FIXED_ONE;
        orc_launch L;
        memset(&L, 0, sizeof(L));
        L.vmin[0] = 0; L.vmin[1] = (int32_t)y0; L.vmin[2] = 0;
        L.vmax[0] = (int32_t)W; L.vmax[1] = (int32_t)(y0 + ny); L.vmax[2] = (int32_t)W;
        L.voxel[0] = L.voxel[1] = L.voxel[2] = go.vx;
        L.det_w = (uint32_t)Wd; L.rows = (uint32_t)k.iSize; L.row_offset = (int32_t)k.iOffset;
        L.n_angles = (uint32_t)Pc; L.modules = (uint32_t)M; L.arith = rp->arith;
        float weight = rp->weight;
        for (int64_t mit = 0; mit < rp->it; ++mit) {
            for (int64_t sit = 0; sit < S; ++sit) {
                jitter_origin(&gen, &go, L.origin);
                float *img = gather_subset(gp, Pc, sit, images, k.iOffset, k.iSize);
                const orc_projdata *spd = pd + sit * Pc * M;
                if (sit > 0 || mit > 0) orc_forward(slab, sum, spd, &L);
                orc_error(img, sum, n_sum, weight);
                orc_backward(slab, (const float *)sum, spd, &L);
                memset(sum, 0, sizeof(uint32_t) * n_sum);
                free(img);
            }
            weight *= rp->weight_factor;
        }
        memcpy(vol + k.vOffset * W * W, slab + k.vPadTop * W * W, sizeof(float) * (size_t)(k.vSize * W * W));
        free(sum);
        free(slab);
    }
    free(pd);
    free(all);
    return 0;
}

/* ======================================================================== */
/* FP64 oracle: the algorithm in double precision with no fixed point       */
/* ======================================================================== */
/* The precision reference for reduced-precision storage.  It keeps everything
 * that defines the algorithm -- the geometry of geometry.hpp (built and kept in
 * double), the same mt19937 jitter draws (uniform_real_distribution<float>, then
 * widened), the nearest-pixel rule with the viewport bounds, the clamps of the
 * error step (eps = 2^-22, KernelError.cl:8-24) and of the -log preprocessing
 * (data_loader.hpp:84-86), 0/0 -> NaN for voxels no projection reaches -- and drops
 * what only exists for single precision: the 22-bit fixed-point sums (double sums
 * instead) and the float roundings. */
int orc_geometry_f64(const orc_geom_params *gp, double *mvp, double *vp, orc_geom_out *go)
{
    const int64_t P = gp->projections, M = gp->module_number;
    orc_projdata *tmp = (orc_projdata *)malloc(sizeof(orc_projdata) * (size_t)(P * M));
    orc_geometry(gp, 1, tmp, go);
    free(tmp);
    geometry_f64(gp, P, M, (uint64_t)gp->dwidth / (uint64_t)M, (uint64_t)gp->dheight, mvp, vp);
    return 0;
}

static inline int pair_f64(const double *m, const double *vp, double px, double py, double pz, double rows,
                           int64_t *iu, int64_t *iv)
{
    const double nu = m[0] * px + m[1] * py + m[2] * pz + m[3];
    const double nv = m[4] * px + m[5] * py + m[6] * pz + m[7];
    const double nw = m[12] * px + m[13] * py + m[14] * pz + m[15];
    const double yu = nu / nw + 0.5, yv = nv / nw + 0.5;
    const int in = (yu >= vp[0]) && (yu < vp[1]) && (yv >= vp[2]) && (yv < vp[3]) && (yv < rows);
    if (in) {
        *iu = (int64_t)floor(yu);
        *iv = (int64_t)floor(yv);
    }
    return in;
}

void orc64_forward(const double *vol, double *sum, const double *mvp, const double *vp, int64_t n_entries,
                   int64_t modules, int64_t W, int64_t Hv, const double origin[3], double voxel, int64_t det_w,
                   int64_t rows)
{
    const int64_t n = W * Hv * W, stride = det_w * rows;
#pragma omp parallel for schedule(static, 4096)
    for (int64_t id = 0; id < n; ++id) {
        const int64_t y = id / (W * W), z = (id / W) % W, x = id % W;
        const double px = (double)x * voxel + origin[0], py = (double)y * voxel + origin[1],
                     pz = (double)z * voxel + origin[2];
        const double value = vol[id];
        if (value == 0.0) continue;
        for (int64_t e = 0; e < n_entries; ++e) {
            int64_t iu, iv;
            if (!pair_f64(mvp + 16 * e, vp + 4 * e, px, py, pz, (double)rows, &iu, &iv)) continue;
            double *dst = &sum[(e / modules) * stride + iv * det_w + iu];
#pragma omp atomic
            *dst += value;
        }
    }
}

void orc64_backward(double *vol, const double *ratio, const double *mvp, const double *vp, int64_t n_entries,
                    int64_t modules, int64_t W, int64_t Hv, const double origin[3], double voxel, int64_t det_w,
                    int64_t rows)
{
    const int64_t n = W * Hv * W, stride = det_w * rows;
#pragma omp parallel for schedule(static, 4096)
    for (int64_t id = 0; id < n; ++id) {
        const int64_t y = id / (W * W), z = (id / W) % W, x = id % W;
        const double px = (double)x * voxel + origin[0], py = (double)y * voxel + origin[1],
                     pz = (double)z * voxel + origin[2];
        double s = 0.0;
        int64_t cnt = 0;
        for (int64_t e = 0; e < n_entries; ++e) {
            int64_t iu, iv;
            if (!pair_f64(mvp + 16 * e, vp + 4 * e, px, py, pz, (double)rows, &iu, &iv)) continue;
            s += ratio[(e / modules) * stride + iv * det_w + iu];
            ++cnt;
        }
        vol[id] *= exp(s / (double)cnt);
    }
}

void orc64_preprocess(const float *raw, double *out, uint64_t n, int mlog)
{
    const double eps = 1.0 / 4194304.0;
#pragma omp parallel for schedule(static, 65536)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        double x = (double)raw[i];
        if (mlog) x = -log(fmax(fmin(x, 1.0 - eps), eps));
        out[i] = x;
    }
}

int orc64_recon_naive(const orc_geom_params *gp, const orc_recon_params *rp, const double *images, double *vol)
{
    orc_geom_out go;
    const int64_t P = gp->projections, M = gp->module_number, S = rp->sit;
    orc_geom_params g = *gp;
    g.sit = S;
    double *mvp = (double *)malloc(sizeof(double) * (size_t)(P * M * 16));
    double *vp = (double *)malloc(sizeof(double) * (size_t)(P * M * 4));
    orc_geometry_f64(&g, mvp, vp, &go);
    const int64_t Pc = go.concurrent, W = go.vwidth, Hv = go.vheight, Wd = gp->dwidth, Hd = gp->dheight;
    if (Pc <= 0) { free(mvp); free(vp); return -1; }
    const double eps = 1.0 / 4194304.0;
    const int64_t n_sum = Pc * Wd * Hd, nvox = W * Hv * W;
    double *sum = (double *)malloc(sizeof(double) * (size_t)n_sum);
    double *smvp = (double *)malloc(sizeof(double) * (size_t)(Pc * M * 16));
    double *svp = (double *)malloc(sizeof(double) * (size_t)(Pc * M * 4));
    for (int64_t i = 0; i < nvox; ++i) vol[i] = 1.0;
    orc_mt19937 gen;
    orc_mt_seed(&gen, rp->seed);
    double weight = rp->weight;
    for (int64_t mit = 0; mit < rp->it; ++mit) {
        for (int64_t sit = 0; sit < S; ++sit) {
            double origin[3];
            for (int i = 0; i < 3; ++i) origin[i] = (double)go.orig[i] + (double)orc_uniform_float(&gen, 0.0f, go.vx);
            for (int64_t k = 0; k < Pc; ++k)
                for (int64_t mod = 0; mod < M; ++mod) {
                    memcpy(smvp + (k * M + mod) * 16, mvp + ((sit + k * S) * M + mod) * 16, sizeof(double) * 16);
                    memcpy(svp + (k * M + mod) * 4, vp + ((sit + k * S) * M + mod) * 4, sizeof(double) * 4);
                }
            if (sit > 0 || mit > 0) {
                memset(sum, 0, sizeof(double) * (size_t)n_sum);
                orc64_forward(vol, sum, smvp, svp, Pc * M, M, W, Hv, origin, (double)go.vx, Wd, Hd);
            } else {
                for (int64_t i = 0; i < n_sum; ++i) sum[i] = 1.0;
            }
#pragma omp parallel for schedule(static, 65536)
            for (int64_t i = 0; i < n_sum; ++i) {
                const int64_t k = i / (Wd * Hd), r = i - k * Wd * Hd;
                const double ref = images[(sit + k * S) * Wd * Hd + r];
                sum[i] = log(fmax(ref / fmax(sum[i], eps), eps)) * weight;
            }
            orc64_backward(vol, sum, smvp, svp, Pc * M, M, W, Hv, origin, (double)go.vx, Wd, Hd);
        }
        weight *= rp->weight_factor;
    }
    free(sum); free(smvp); free(svp); free(mvp); free(vp);
    return 0;
}
