// xpr_math.cuh -- arithmetic contracts of the projector, shared by every kernel.
//
// Two contracts, both exactly reproducible on a CPU (the oracle restates them):
//
//   STRICT  the reference kernels (KernelForward.cl:25-36, KernelBackward.cl:23-37)
//           under IEEE-754 single precision: p = idx*vx + o (mul then add);
//           n_r = ((c.x*px + c.y*py) + c.z*pz) + c.w for r in {u, v, w};
//           u = n_u / n_w, v = n_v / n_w - line_offset; pixel = round half away
//           from zero, converted with saturation (NaN -> 0).
//   FAST    p = fma(idx, vx, o); C_r = fma(c.x, px, c.w) + c.z*pz for r in {u, v, w};
//           rw = 1/fma(c_w.y, py, C_w) (IEEE); yu = fma(py, c_u.y*rw, fma(C_u, rw, 0.5)),
//           yv = fma(py, c_v.y*rw, fma(C_v, rw, 0.5 - off)); pixel = (floor(yu), floor(yv)).
//           For an untilted detector c_u.y = c_w.y = 0 exactly, so along a vertical voxel
//           column u, w and 1/w are invariant and yv moves by one fma per voxel.
//
// Every operation is written with an explicit rounding intrinsic so that no
// compiler contraction can change a result.  exp / log are this project's own
// single-precision functions (Cody & Waite reduction with a degree-7 Taylor
// polynomial; the atanh series for log), bit-identical to the oracle's.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#ifdef __CUDACC__
#define XPR_HD __host__ __device__ __forceinline__
#else
#define XPR_HD inline
#endif

namespace xpr {

enum Arith : int { kStrict = 0, kFast = 1 };

constexpr uint32_t kFixedOne = 1u << 22;   // FIXED_FRAC_ONE (constants.cl:19)
constexpr float kEps = 1.0f / 4194304.0f;  // EPSILON = FIXED_TO_FLOAT(1) (constants.cl:23)

#ifdef __CUDA_ARCH__
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float frcp(float a) { return __frcp_rn(a); }
__device__ __forceinline__ uint32_t fbits(float f) { return __float_as_uint(f); }
__device__ __forceinline__ float bitsf(uint32_t u) { return __uint_as_float(u); }
#endif

// ------------------------------------------------------------------ portable exp / log
// 2^k for -126 <= k <= 127
__device__ __forceinline__ float pow2i(int k) { return __uint_as_float((uint32_t)(k + 127) << 23); }

__device__ __forceinline__ float p_expf(float x)
{
    if (x != x) return x;
    if (x > 0x1.62e42ep+6f) return __int_as_float(0x7f800000);
    if (x < -0x1.9fe368p+6f) return 0.0f;
    const float k = rintf(__fmul_rn(x, 0x1.715476p+0f));
    float r = __fmaf_rn(-k, 0x1.62e4p-1f, x);
    r = __fmaf_rn(-k, 0x1.7f7d1cp-20f, r);
    float p = 0x1.a01a02p-13f;
    p = __fmaf_rn(p, r, 0x1.6c16c2p-10f);
    p = __fmaf_rn(p, r, 0x1.111112p-7f);
    p = __fmaf_rn(p, r, 0x1.555556p-5f);
    p = __fmaf_rn(p, r, 0x1.555556p-3f);
    p = __fmaf_rn(p, r, 0.5f);
    p = __fmaf_rn(p, r, 1.0f);
    p = __fmaf_rn(p, r, 1.0f);
    const int ki = (int)k;
    const int k1 = ki / 2, k2 = ki - k1;
    return __fmul_rn(__fmul_rn(p, pow2i(k1)), pow2i(k2));
}

__device__ __forceinline__ float p_logf(float x)
{
    if (x != x || x < 0.0f) return __int_as_float(0x7fc00000);
    if (x == 0.0f) return __int_as_float(0xff800000);
    if (x == __int_as_float(0x7f800000)) return x;
    int adj = 0;
    if (x < 0x1p-126f) { x = __fmul_rn(x, 0x1p23f); adj = -23; }
    const uint32_t b = __float_as_uint(x);
    int e = (int)((b >> 23) & 0xffu) - 127 + adj;
    float m = __uint_as_float((b & 0x7fffffu) | 0x3f800000u);
    if (m > 0x1.6a09e6p+0f) { m = __fmul_rn(m, 0.5f); e += 1; }
    const float s = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
    const float z = __fmul_rn(s, s);
    float q = __fmaf_rn(z, 0x1.c71c72p-4f, 0x1.24924ap-3f);
    q = __fmaf_rn(q, z, 0x1.99999ap-3f);
    q = __fmaf_rn(q, z, 0x1.555556p-2f);
    const float t = __fadd_rn(s, s);
    const float lm = __fmaf_rn(t, __fmul_rn(z, q), t);
    const float fe = (float)e;
    return __fmaf_rn(fe, 0x1.62e4p-1f, __fmaf_rn(fe, 0x1.7f7d1cp-20f, lm));
}

// ------------------------------------------------------------------ fixed point
// FLOAT_TO_FIXED (constants.cl:22): truncation; the conversion saturates and maps NaN to 0.
__device__ __forceinline__ uint32_t float_to_fixed(float v) { return __float2uint_rz(__fmul_rn(v, 4194304.0f)); }
// FIXED_TO_FLOAT (constants.cl:21)
__device__ __forceinline__ float fixed_to_float(uint32_t x) { return __fdiv_rn(__uint2float_rn(x), 4194304.0f); }

// ------------------------------------------------------------------ storage types
enum DType : int { kF32 = 0, kBF16 = 1, kF16 = 2 };

}  // namespace xpr
