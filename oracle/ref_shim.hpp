/*
 * ref_shim.hpp -- OpenCL C built-ins for compiling the reference's own kernel
 * sources (src/reconstruction/gpu/kernels/*.cl of ebarjou/xpulse_recon) as C++
 * on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY: oracle/build_ref.py includes this header in front
 * of each kernel (after a textual pre-pass: include inlining as CMakeLists.txt:3-15
 * does, vector literals "(float2)(a, b)" -> "float2(a, b)", swizzles ".even" ->
 * ".even()"), and the result is built into oracle/_ref/libxpr_ref.so, which the
 * tests use to pin the oracle's restatement bit-for-bit.
 *
 * Semantics chosen for the operations OpenCL leaves to the implementation:
 *   - dot(a, b) = ((a.x*b.x + a.y*b.y) + a.z*b.z) + a.w*b.w, IEEE, not fused;
 *   - float / float2 arithmetic is IEEE single precision (the reference builds
 *     with -cl-fast-relaxed-math, whose exact results are unspecified);
 *   - convert_int*(): truncation, saturating, NaN -> 0; FLOAT_TO_FIXED is made
 *     saturating the same way (the plain C cast is undefined out of range);
 *   - exp / log: the oracle's portable single-precision functions;
 *   - max(float, float): fmax.
 */
#ifndef XPR_REF_SHIM_HPP
#define XPR_REF_SHIM_HPP

#include <stddef.h>
#include <stdint.h>

extern "C" float orc_expf(float);
extern "C" float orc_logf(float);

namespace oclshim {

typedef uint32_t uint;
typedef uint16_t ushort;

extern thread_local size_t g_gid;
inline size_t get_global_id(int) { return g_gid; }

struct float2 {
    float x, y;
    float2() = default;
    float2(float a, float b) : x(a), y(b) {}
    float lo() const { return x; }
    float hi() const { return y; }
    float even() const { return x; }
    float odd() const { return y; }
};
struct int2 {
    int x, y;
    int2() = default;
    int2(int a, int b) : x(a), y(b) {}
};
struct uint2 {
    uint x, y;
    uint2() = default;
    uint2(uint a, uint b) : x(a), y(b) {}
};
struct float3 {
    float x, y, z;
    float3() = default;
    float3(float a, float b, float c) : x(a), y(b), z(c) {}
};
struct uint3 {
    uint x, y, z;
    uint3() = default;
    uint3(uint a, uint b, uint c) : x(a), y(b), z(c) {}
};
/* members are mutable: KernelForwardH.cl:25 assigns .w of a const float4 */
struct float4 {
    mutable float x, y, z, w;
    float4() = default;
    float4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    float2 lo() const { return float2(x, y); }
    float2 hi() const { return float2(z, w); }
    float2 even() const { return float2(x, z); }
    float2 odd() const { return float2(y, w); }
};
struct uint4 {
    uint x, y, z, w;
    uint4() = default;
    uint4(uint a, uint b, uint c, uint d) : x(a), y(b), z(c), w(d) {}
    uint4(uint3 v, uint d) : x(v.x), y(v.y), z(v.z), w(d) {}
};

inline float2 operator-(float2 a, float2 b) { return float2(a.x - b.x, a.y - b.y); }
inline float2 operator+(float2 a, float2 b) { return float2(a.x + b.x, a.y + b.y); }
inline float2 operator/(float2 a, float s) { return float2(a.x / s, a.y / s); }
inline float3 operator-(float3 a, float3 b) { return float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(float3 a, float3 b) { return float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator/(float s, float3 v) { return float3(s / v.x, s / v.y, s / v.z); }
inline float4 operator*(float4 a, float4 b) { return float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
inline float4 operator*(float4 a, float s) { return float4(a.x * s, a.y * s, a.z * s, a.w * s); }
inline float4 operator+(float4 a, float4 b) { return float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline uint3 operator-(uint3 a, uint3 b) { return uint3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline uint4 operator+(uint4 a, uint4 b) { return uint4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }

/* relational built-ins on vectors return -1 (all bits set) for true */
inline int2 isgreaterequal(float2 a, float2 b) { return int2(a.x >= b.x ? -1 : 0, a.y >= b.y ? -1 : 0); }
inline int2 isless(float2 a, float2 b) { return int2(a.x < b.x ? -1 : 0, a.y < b.y ? -1 : 0); }
inline int2 operator&&(int2 a, int2 b) { return int2((a.x && b.x) ? -1 : 0, (a.y && b.y) ? -1 : 0); }
inline int all(int2 v) { return (v.x < 0) && (v.y < 0); }

inline float dot(float4 a, float4 b) { return ((a.x * b.x + a.y * b.y) + a.z * b.z) + a.w * b.w; }

inline int sat_f2i(float f)
{
    if (f != f) return 0;
    if (f >= 2147483648.0f) return INT32_MAX;
    if (f < -2147483648.0f) return INT32_MIN;
    return (int)f;
}
inline uint32_t float_to_fixed_sat(float v)
{
    float s = v * 4194304.0f;
    if (!(s > 0.0f)) return 0u;
    if (s >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)s;
}
inline float2 round(float2 v) { return float2(__builtin_roundf(v.x), __builtin_roundf(v.y)); }
inline int2 convert_int2(float2 v) { return int2(sat_f2i(v.x), sat_f2i(v.y)); }
inline float2 convert_float2(int2 v) { return float2((float)v.x, (float)v.y); }
inline float4 convert_float4(uint4 v) { return float4((float)v.x, (float)v.y, (float)v.z, (float)v.w); }

inline float exp(float x) { return orc_expf(x); }
inline float log(float x) { return orc_logf(x); }
inline float max(float a, float b) { return __builtin_fmaxf(a, b); }
inline float min(float a, float b) { return __builtin_fminf(a, b); }
inline float3 min(float3 a, float3 b) { return float3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline float3 max(float3 a, float3 b) { return float3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline bool isnan(float x) { return __builtin_isnan(x); }

inline uint atomic_add(volatile uint *p, uint v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }

}  // namespace oclshim

#ifndef MAXFLOAT
#define MAXFLOAT 3.402823466e+38F
#endif

#endif
