// xpr_kernels.cu -- sm_100a kernels of the iterative cone-beam hot path.
//
//   forward   (KernelForward.cl:10-55 / KernelForwardH.cl:8-37)   k_forward_tiled
//   backward  (KernelBackward.cl:8-40 / KernelBackwardH.cl:8-42) k_backward_tiled
//   error     (KernelError.cl:8-24, reconstruction_lplh.hpp:140-177) k_error
//   -log / normalise (data_loader.hpp:48-101)                     k_minmax, k_preprocess
//
// Design (B200): the path is a voxel-driven nearest-pixel splat / gather.  It
// is bound by FP32 issue and atomic throughput, not by HBM bytes, so the
// kernels are organised to cut atomics and redundant arithmetic:
//
//  * A forward CTA owns a brick of 32 x 8 x 32 voxels (x, y, z) for a run of
//    projections (a backward CTA one of 32 x 16 x 8).  The forward keeps the brick in shared memory as 22-bit
//    fixed point (loaded once, coalesced), projects its 8 corners per
//    projection to bound its detector footprint, splats into a shared-memory
//    tile of that footprint with shared atomics, and flushes the tile with one
//    coalesced global atomic per touched pixel.  Bricks whose footprint misses
//    the viewport are skipped; all-zero bricks are skipped.
//  * Each thread walks vertical voxel columns (along y).  For an untilted
//    detector a column lands in one detector column with one 1/w, so a voxel
//    costs one packed FMA and one round-toward-zero add for its row, one
//    multiply-add for its tile index, a quarter of a 128-bit shared load for
//    its value and one shared atomic.  The 32 lanes of a warp run across the ray
//    (x or z, chosen per projection), so they mostly hit distinct pixels.
//    Integer atomics commute, so the result is bit-identical to the reference's
//    voxel-per-work-item order.
//  * The backward keeps each voxel's running sum and count in registers and
//    visits projections in the reference's order, so the floating-point sum is
//    the reference's sum; detector gathers go through the read-only L1 path,
//    which the brick's small footprint keeps resident.
//  * Along a column the projective numerators are affine in y; the column
//    invariant part is computed once per column, and in the forward the lane
//    coordinate's share of it once per projection (see xpr_math.cuh for the
//    exact operation contracts).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <type_traits>
#include <cfloat>

#include "xpr_internal.h"
#include "xpr_math.cuh"

namespace xpr {

constexpr int BX = 32;          // brick extent along x
constexpr int BY = 8;           // forward brick extent along y (the column walked by a thread)
constexpr int BZ = 32;          // forward brick extent along z
constexpr int NT = 256;         // threads per CTA (8 warps)
constexpr int G = 4;            // projections whose tiles are in flight together
constexpr int TILE_CAP = 1024;  // pixels per shared-memory tile
constexpr int MCAP = 32;        // projections whose metadata a CTA prepares at once
static_assert(MCAP % G == 0 && MCAP / G <= NT / 32, "one group of G projections per warp");
constexpr int VSTRIDE = 132;    // padded row stride (words) of the brick value array: 32 x-positions of four
                                // layers interleaved, + 4 (128-bit reads bank-conflict free both ways)
constexpr int BWD_BY = 16;      // backward column length along y
constexpr int BWD_BZ = 8;       // backward brick extent along z (one warp per z)
constexpr uint32_t kMagic = 0x4B000000u;  // float bits of 2^23: bits(fadd_rz(y, 2^23)) - kMagic = floor(y)

enum Mode : int { kSkip = 0, kTile = 1, kDirect = 2 };

// Per-projection constants of one (brick, projection) pair, read by every thread as
// 16-byte vectors.  Rectangle [u0, u1) x [v0, v1) in buffer coordinates; a pixel
// (iu, iv) inside it goes to target index (iv - v0) * pitch + (iu - u0) + off, where
// the target is the shared-memory tile (pitch = tile width, off = 0) or the whole
// detector buffer (pitch = det_w, off = img_base + v0 * det_w + u0).
struct __align__(16) ProjMeta {
    float4 cu, cv, cw;                    // matrix rows for u, v, w (glm columns c0, c1, c3)
    uint4 fast;                           // {kMagic + u0, u1 - u0, kMagic + v0, v1 - v0}
    int4 rect;                            // {u0, u1 - u0, v0, v1 - v0}
    uint4 tgt;                            // {pitch, off, img_base, tile width}
    int4 flags;                           // {mode, lanes across z, column (bit 0: untilted, bit 1: and
                                          //  walk_exact's screen passed), inside (no bounds tests)}
    float T[16];                          // STRICT: c_v.y * py of the brick's layers (the reference's rounding)
};

// --------------------------------------------------------------------------------------
// per-projection metadata: one group of G entries, computed by warp 0
// lane = g * 8 + corner of the brick [x0, x0+ex) x [y0, y0+ey) x [z0, z0+ez)
// --------------------------------------------------------------------------------------
// align4: a tile is flushed by 16-byte bulk reductions, so it starts on a 4-pixel column
// boundary and its rows are padded to a multiple of 4 words (the detector width must then
// be a multiple of 4, which keeps the padded rows inside the image rows).
template <int ARITH, bool LIST, bool GATHER, int TCAP = TILE_CAP>
__device__ __forceinline__ void compute_meta(ProjMeta *s_meta, const xpr_projdata *__restrict__ pd,
                                             const LaunchArgs &a, int e0, int e_end, int bx0, int by0, int bz0,
                                             int ex, int ey, int ez, int lane, bool align4 = false)
{
    const int g = lane >> 3, c = lane & 7;
    const int entry = e0 + g;
    bool valid = entry < e_end;
    uint32_t pidx = 0, img = 0;
    if (valid) {
        pidx = LIST ? (uint32_t)__ldg(&a.list_mvp[entry]) : (uint32_t)entry;
        img = LIST ? (uint32_t)__ldg(&a.list_img[entry]) : (uint32_t)entry / a.modules;
        valid = pidx < a.n_pd && img < a.n_images;
    }
    const float *m = valid ? pd[pidx].mvp : pd[0].mvp;
    const float cu0 = __ldg(m + 0), cu1 = __ldg(m + 1), cu2 = __ldg(m + 2), cu3 = __ldg(m + 3);
    const float cv0 = __ldg(m + 4), cv1 = __ldg(m + 5), cv2 = __ldg(m + 6), cv3 = __ldg(m + 7);
    const float cw0 = __ldg(m + 12), cw1 = __ldg(m + 13), cw2 = __ldg(m + 14), cw3 = __ldg(m + 15);
    // corner voxel centres of the brick (nominal extent; partial bricks are covered)
    const int ix = a.vmin[0] + bx0 + ((c & 1) ? ex - 1 : 0);
    const int iy = a.vmin[1] + by0 + ((c & 2) ? ey - 1 : 0);
    const int iz = a.vmin[2] + bz0 + ((c & 4) ? ez - 1 : 0);
    const float px = __fmaf_rn((float)ix, a.voxel[0], a.origin[0]);
    const float py = __fmaf_rn((float)iy, a.voxel[1], a.origin[1]);
    const float pz = __fmaf_rn((float)iz, a.voxel[2], a.origin[2]);
    if (ARITH == kStrict) {
        // the products c_v.y * py of the STRICT numerator, two layers per lane, rounded as the
        // reference rounds them; walk_exact loads them, so no packed product feeds its sums
        // (the code generator contracts a packed multiply into the packed add that consumes it)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int k = 2 * c + h;
            if (k < ey)
                s_meta[g].T[k] = __fmul_rn(cv1, __fadd_rn(__fmul_rn(__uint2float_rn((uint32_t)(a.vmin[1] + by0 + k)),
                                                                     a.voxel[1]), a.origin[1]));
        }
    }
    const float nu = __fmaf_rn(cu0, px, __fmaf_rn(cu1, py, __fmaf_rn(cu2, pz, cu3)));
    const float nv = __fmaf_rn(cv0, px, __fmaf_rn(cv1, py, __fmaf_rn(cv2, pz, cv3)));
    const float nw = __fmaf_rn(cw0, px, __fmaf_rn(cw1, py, __fmaf_rn(cw2, pz, cw3)));
    const float u = __fdiv_rn(nu, nw);
    const float v = __fsub_rn(__fdiv_rn(nv, nw), a.row_off_f);
    int ok = (nw > 0.0f) && (fabsf(u) < 1.0e9f) && (fabsf(v) < 1.0e9f);
    // walk_exact's operand screen, with a factor 2 of margin for the STRICT positions'
    // rounding: the u and v numerators' terms below 2^99 in magnitude and n_w in
    // [2^-59, 2^59] with one sign at every corner (n_w is affine over the brick, so its
    // range is its corners'); NaN and inf fail every comparison
    const float bu = fabsf(cu0 * px) + fabsf(cu1 * py) + fabsf(cu2 * pz) + fabsf(cu3);
    const float bv = fabsf(cv0 * px) + fabsf(cv1 * py) + fabsf(cv2 * pz) + fabsf(cv3);
    int scr = (bu < 0x1p99f) && (bv < 0x1p99f) && (fabsf(nw) >= 0x1p-59f) && (fabsf(nw) <= 0x1p59f);
    int wpos = nw > 0.0f, wneg = nw < 0.0f;
    float umin = ok ? u : 0.0f, umax = umin, vmn = ok ? v : 0.0f, vmx = vmn;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
        umin = fminf(umin, __shfl_xor_sync(0xffffffffu, umin, o));
        umax = fmaxf(umax, __shfl_xor_sync(0xffffffffu, umax, o));
        vmn = fminf(vmn, __shfl_xor_sync(0xffffffffu, vmn, o));
        vmx = fmaxf(vmx, __shfl_xor_sync(0xffffffffu, vmx, o));
        ok &= __shfl_xor_sync(0xffffffffu, ok, o);
        scr &= __shfl_xor_sync(0xffffffffu, scr, o);
        wpos &= __shfl_xor_sync(0xffffffffu, wpos, o);
        wneg &= __shfl_xor_sync(0xffffffffu, wneg, o);
    }
    if (c == 0) {
        ProjMeta &M = s_meta[g];
        const float *vp = valid ? pd[pidx].vp : pd[0].vp;
        int l = max((int)ceilf(fmaxf(__ldg(vp + 0), -1.0e9f)), 0);
        int r = min((int)ceilf(fminf(__ldg(vp + 1), 1.0e9f)), (int)a.det_w);
        int b = max((int)ceilf(fmaxf(__ldg(vp + 2), -1.0e9f)), 0);
        int t = min((int)ceilf(fminf(__ldg(vp + 3), 1.0e9f)), (int)a.rows);
        // inside: the brick's whole footprint (corner projections with a margin of 2
        // pixels, far above the rounding of any voxel's pixel) lies in the viewport, so
        // every voxel of the brick lands in the rectangle and needs no bounds test
        int inside = 0;
        if (ok) {
            const int fl = (int)floorf(umin) - 2, fr = (int)ceilf(umax) + 3;
            const int fb = (int)floorf(vmn) - 2, ft = (int)ceilf(vmx) + 3;
            inside = fl >= l && fr <= r && fb >= b && ft <= t;
            l = max(l, fl);
            r = min(r, fr);
            b = max(b, fb);
            t = min(t, ft);
        }
        const int lt = (align4 && !GATHER) ? (l & ~3) : l;             // the tile's first column
        const int wt = (align4 && !GATHER) ? ((r - lt + 3) & ~3) : r - lt;  // its row pitch
        const int area = wt * (t - b);
        const int mode = (!valid || r <= l || t <= b) ? kSkip : ((ok && area <= TCAP) ? kTile : kDirect);
        const uint32_t img_base = img * a.img_stride;
        const bool tile = (mode == kTile) && !GATHER;
        if (tile) l = lt;
        const uint32_t pitch = tile ? (uint32_t)wt : a.det_w;
        const uint32_t off = tile ? 0u : img_base + (uint32_t)b * a.det_w + (uint32_t)l;
        M.cu = make_float4(cu0, cu1, cu2, cu3);
        M.cv = make_float4(cv0, cv1, cv2, cv3);
        M.cw = make_float4(cw0, cw1, cw2, cw3);
        M.fast = make_uint4(kMagic + (uint32_t)l, (uint32_t)(r - l), kMagic + (uint32_t)b, (uint32_t)(t - b));
        M.rect = make_int4(l, r - l, b, t - b);
        M.tgt = make_uint4(pitch, off, img_base, (uint32_t)(r - l));
        const int column = (cu1 == 0.0f) && (cw1 == 0.0f);
        M.flags = make_int4(mode, fabsf(cw0) > fabsf(cw2), column ? (1 | ((scr && (wpos || wneg)) << 1)) : 0, inside);
    }
}

// --------------------------------------------------------------------------------------
// positions and column-invariant numerators in each contract
// --------------------------------------------------------------------------------------
template <int ARITH>
__device__ __forceinline__ float pos(int idx, float vox, float org)
{
    if (ARITH == kFast) return __fmaf_rn((float)idx, vox, org);
    return __fadd_rn(__fmul_rn(__uint2float_rn((uint32_t)idx), vox), org);
}

// FAST: C = fma(c.x, px, c.w) + c.z*pz
__device__ __forceinline__ float col_fast(float4 c, float px, float pz)
{
    return __fadd_rn(__fmaf_rn(c.x, px, c.w), __fmul_rn(c.z, pz));
}

// STRICT: n = ((c.x*px + c.y*py) + c.z*pz) + c.w
__device__ __forceinline__ float num_strict(float4 c, float px, float py, float pz)
{
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(c.x, px), __fmul_rn(c.y, py)), __fmul_rn(c.z, pz)), c.w);
}

// bits of fadd_rz(y, 2^23) minus `base`: for 0 <= y < 2^22 this is floor(y) - (base - kMagic);
// every other y (negative, >= 2^22, inf, NaN) gives a value >= 2^23 as unsigned, so
// "d < range" with range <= 2^22 is exactly "base' <= y < base' + range".
__device__ __forceinline__ uint32_t fdist(float y, uint32_t base)
{
    return __float_as_uint(__fadd_rz(y, 8388608.0f)) - base;
}

// Two lanes of IEEE single-precision arithmetic in one instruction (sm_100 packed f32x2):
// each half is rounded exactly as the scalar operation, so results are unchanged.
// Scalar-operand forms (each call pairs its operands); the forward's walk uses these.
__device__ __forceinline__ void fma_rn2(float &d0, float &d1, float a0, float a1, float b, float c)
{
    asm("{.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %4};\n\t"
        "mov.b64 rc, {%5, %5};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\t"
        "mov.b64 {%0, %1}, rd;}"
        : "=f"(d0), "=f"(d1)
        : "f"(a0), "f"(a1), "f"(b), "f"(c));
}
__device__ __forceinline__ void add_rz2(float &d0, float &d1, float a0, float a1, float b)
{
    asm("{.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %4};\n\t"
        "add.rz.f32x2 rd, ra, rb;\n\t"
        "mov.b64 {%0, %1}, rd;}"
        : "=f"(d0), "=f"(d1)
        : "f"(a0), "f"(a1), "f"(b));
}
__device__ __forceinline__ void fma_rn2v(float &d0, float &d1, float a0, float a1, float b0, float b1, float c0,
                                         float c1)
{
    asm("{.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\t"
        "mov.b64 {%0, %1}, rd;}"
        : "=f"(d0), "=f"(d1)
        : "f"(a0), "f"(a1), "f"(b0), "f"(b1), "f"(c0), "f"(c1));
}
__device__ __forceinline__ void mul_rn2v(float &d0, float &d1, float a0, float a1, float b0, float b1)
{
    asm("{.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\t"
        "mov.b64 {%0, %1}, rd;}"
        : "=f"(d0), "=f"(d1)
        : "f"(a0), "f"(a1), "f"(b0), "f"(b1));
}
// FAST contract for two voxels of a tilted column: the pixel coordinates' bits
// fadd_rz(y, 2^23) for u (bu0, bu1) and v (bv0, bv1), with
// rw = 1/fma(c_w.y, py, C_w), yu = fma(py, c_u.y*rw, fma(C_u, rw, 1/2)),
// yv = fma(py, c_v.y*rw, fma(C_v, rw, 1/2 - off)).
__device__ __forceinline__ void tilted_pair(float py0, float py1, float4 cu, float4 cv, float4 cw, float Cu, float Cv,
                                            float Cw, float hv, uint32_t &bu0, uint32_t &bu1, uint32_t &bv0,
                                            uint32_t &bv1)
{
    float w0, w1, t0, t1, i0, i1, y0, y1, b0, b1;
    fma_rn2v(w0, w1, cw.y, cw.y, py0, py1, Cw, Cw);
    const float rw0 = __frcp_rn(w0), rw1 = __frcp_rn(w1);
    mul_rn2v(t0, t1, cu.y, cu.y, rw0, rw1);
    fma_rn2v(i0, i1, Cu, Cu, rw0, rw1, 0.5f, 0.5f);
    fma_rn2v(y0, y1, py0, py1, t0, t1, i0, i1);
    add_rz2(b0, b1, y0, y1, 8388608.0f);
    bu0 = __float_as_uint(b0);
    bu1 = __float_as_uint(b1);
    mul_rn2v(t0, t1, cv.y, cv.y, rw0, rw1);
    fma_rn2v(i0, i1, Cv, Cv, rw0, rw1, hv, hv);
    fma_rn2v(y0, y1, py0, py1, t0, t1, i0, i1);
    add_rz2(b0, b1, y0, y1, 8388608.0f);
    bv0 = __float_as_uint(b0);
    bv1 = __float_as_uint(b1);
}

// Register-pair forms: the operands are 64-bit pairs {lo, hi}, and values that stay packed
// across a column (the y positions, the column constants) are paired once, not per
// instruction; the backward's walk uses these.
// an add to a shared-memory word by its 32-bit shared-window address
__device__ __forceinline__ void red_shared_add(uint32_t saddr, uint32_t v)
{
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(saddr), "r"(v) : "memory");
}

// Bulk reduction of `bytes` (a multiple of 16) of u32 words from shared memory into global
// memory (both addresses 16-byte aligned), performed by the TMA unit: each word is added to
// its destination atomically (modulo 2^32), as a red.global.add of it would.  Tracked by the
// issuing thread's bulk async-group.
__device__ __forceinline__ void bulk_add_u32(uint32_t *gdst, const uint32_t *ssrc, uint32_t bytes)
{
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.u32 [%0], [%1], %2;"
                 ::"l"(gdst), "r"((uint32_t)__cvta_generic_to_shared(ssrc)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the thread's bulk operations have read their shared-memory sources
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// the thread's bulk operations are complete
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// orders this thread's shared-memory writes before later reads of them by the TMA unit
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ uint64_t f2pack(float lo, float hi)
{
    uint64_t d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ void f2unpack(uint64_t v, float &lo, float &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ void u2unpack(uint64_t v, uint32_t &lo, uint32_t &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=r"(lo), "=r"(hi) : "l"(v));
}
__device__ __forceinline__ float f2lo(uint64_t v)
{
    float lo, hi;
    f2unpack(v, lo, hi);
    return lo;
}
__device__ __forceinline__ float f2hi(uint64_t v)
{
    float lo, hi;
    f2unpack(v, lo, hi);
    return hi;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c)
{
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b)
{
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t addrz2(uint64_t a, uint64_t b)
{
    uint64_t d;
    asm("add.rz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b)
{
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Correctly rounded quotient a / b (IEEE round to nearest) for a divisor shared by many
// dividends, from y = RN(1/b) and ylo = RN(RN(1 - b*y) * y), computed once per divisor.
// y + ylo approximates 1/b to about 2^-47, so q0 = RN(a*y + RN(a*ylo)) lies within one ulp
// of a/b; the residual a - b*q0 is then exact (one fma), and RN(q0 + r*y) is the correctly
// rounded quotient (Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990).  The argument needs a, b, the
// quotient and the residual away from overflow; callers screen |b| in [2^-60, 2^60] and
// |a| < 2^102.  A quotient in the subnormal range may be off in its last bits, which no
// pixel decision can see (|a/b| < 2^-100 rounds to pixel 0 either way).
__device__ __forceinline__ float div_exact(float a, float nb, float y, float ylo)  // nb = -b
{
    const float q0 = __fmaf_rn(a, y, __fmul_rn(a, ylo));
    return __fmaf_rn(__fmaf_rn(nb, q0, a), y, q0);
}
// the same for two dividends (register pair) and one divisor
__device__ __forceinline__ uint64_t div_exact2(uint64_t a, uint64_t nb, uint64_t y, uint64_t ylo)
{
    const uint64_t q0 = fma2(a, y, mul2(a, ylo));
    return fma2(fma2(nb, q0, a), y, q0);
}
// Pixel of a STRICT coordinate q (the reference rounds half away from zero, then
// subtracts nothing (u) or an integer row offset first (v)): bits(RZ(RZ(q + 1/2) + 2^23))
// - base with base = 2^23's bits + off + lo is the buffer pixel minus lo for every q
// whose pixel can be in [lo, lo + n) (n <= 2^22), and >= 2^22 as unsigned otherwise,
// except q = off - 1/2 exactly (the reference gives -1 there, this gives 0).  For
// in-bounds pixels q - off is exact (|q - off| <= |q| and both are on q's ulp grid),
// and floor(RZ(x)) = floor(x) for x >= 0 because the integers below 2^24 are floats.
__device__ __forceinline__ uint64_t pix_bits2(uint64_t q, uint64_t half, uint64_t magic)
{
    return addrz2(addrz2(q, half), magic);
}
__device__ __forceinline__ uint32_t pix_bits(float q)
{
    return __float_as_uint(__fadd_rz(__fadd_rz(q, 0.5f), 8388608.0f));
}
// y position of layer k of a column, from its pairs or from a plain array
template <int N>
__device__ __forceinline__ float ypos(const uint64_t (&py2)[N], int k)
{
    return (k & 1) ? f2hi(py2[k >> 1]) : f2lo(py2[k >> 1]);
}
template <int N>
__device__ __forceinline__ float ypos(const float (&py)[N], int k)
{
    return py[k];
}

// Column constants of the FAST contract, each duplicated into both halves of a pair.
struct Packed {
    uint64_t magic;           // {2^23, 2^23}
    uint64_t cuy, cvy, cwy;   // c.y of the u, v, w rows
    uint64_t Cu, Cv, Cw;      // column numerators
    uint64_t half, hv;        // {1/2, 1/2}, {1/2 - off, 1/2 - off}
};

// FAST contract for two voxels (py pair P) of a tilted column: the pixel coordinates'
// bits fadd_rz(y, 2^23) for u (bu) and v (bv), each as {voxel 0, voxel 1}, with
// rw = 1/fma(c_w.y, py, C_w), yu = fma(py, c_u.y*rw, fma(C_u, rw, 1/2)),
// yv = fma(py, c_v.y*rw, fma(C_v, rw, 1/2 - off)).
__device__ __forceinline__ void tilted_pair(uint64_t P, const Packed &k, uint64_t &bu, uint64_t &bv)
{
    float w0, w1;
    f2unpack(fma2(k.cwy, P, k.Cw), w0, w1);
    const uint64_t rw = f2pack(__frcp_rn(w0), __frcp_rn(w1));
    bu = addrz2(fma2(P, mul2(k.cuy, rw), fma2(k.Cu, rw, k.half)), k.magic);
    bv = addrz2(fma2(P, mul2(k.cvy, rw), fma2(k.Cv, rw, k.hv)), k.magic);
}

// FAST-contract part of the column walker (below), from the column's numerators
// C_u, C_v, C_w = fma(c.x, px, c.w) + c.z * pz; same calls and return value.  Two forms
// of the same arithmetic: y positions as floats (this one, the forward's: measured faster
// there) or in register pairs (the next one, the backward's: measured faster there).
// isc / ib: f receives the target index as idx * isc + ib (mod 2^32); a shared-memory tile
// passes its element size and its shared-window address, so the walk's one multiply-add
// per voxel forms the atomic's address (isc = 1, ib = 0: the plain index).
template <int LEN, typename F>
__device__ __forceinline__ int walk_fast(const ProjMeta &M, const LaunchArgs &a, float Cu, float Cv, float Cw,
                                         const float (&py)[LEN], F &&f, uint32_t isc = 1u, uint32_t ib = 0u)
{
    const float4 cu = M.cu, cv = M.cv, cw = M.cw;
    const uint4 tgt = M.tgt;
    const uint32_t pitch = tgt.x;
    const uint4 fb = M.fast;
    const float hv = a.half_minus_off;
    if (M.flags.w) {
        // dv = bits(fadd_rz(yv, 2^23)) - fb.z is in [0, rows) for every voxel, so the
        // index dv * pitch + du + off is bits * pitch + (du + off - fb.z * pitch) mod 2^32
        const uint32_t Kv = tgt.y - fb.z * pitch;
        if (M.flags.z) {
            const float rw = __frcp_rn(Cw);
            const uint32_t K = (fdist(__fmaf_rn(Cu, rw, 0.5f), fb.x) + Kv) * isc + ib;
            const uint32_t pitchS = pitch * isc;
            const float Qv = __fmul_rn(cv.y, rw), Rv = __fmaf_rn(Cv, rw, hv);
            static_assert(LEN % 2 == 0, "columns are walked two voxels at a time");
#pragma unroll
            for (int k = 0; k < LEN; k += 2) {
                float y0, y1, b0, b1;
                fma_rn2(y0, y1, py[k], py[k + 1], Qv, Rv);
                add_rz2(b0, b1, y0, y1, 8388608.0f);
                f(std::true_type{}, k, true, __float_as_uint(b0) * pitchS + K);
                f(std::true_type{}, k + 1, true, __float_as_uint(b1) * pitchS + K);
            }
        } else {
            const uint32_t Ku = Kv - fb.x;
#pragma unroll
            for (int k = 0; k < LEN; k += 2) {
                uint32_t bu0, bu1, bv0, bv1;
                tilted_pair(py[k], py[k + 1], cu, cv, cw, Cu, Cv, Cw, hv, bu0, bu1, bv0, bv1);
                f(std::true_type{}, k, true, (bv0 * pitch + bu0 + Ku) * isc + ib);
                f(std::true_type{}, k + 1, true, (bv1 * pitch + bu1 + Ku) * isc + ib);
            }
        }
        return 2;
    }
    if (M.flags.z) {
        const float rw = __frcp_rn(Cw);
        const uint32_t du = fdist(__fmaf_rn(Cu, rw, 0.5f), fb.x);
        const bool in_u = du < fb.y;
        if (!__any_sync(0xffffffffu, in_u)) return 0;
        const uint32_t K = (du + tgt.y) * isc + ib;
        const uint32_t pitchS = pitch * isc;
        const float Qv = __fmul_rn(cv.y, rw), Rv = __fmaf_rn(Cv, rw, hv);
#pragma unroll
        for (int k = 0; k < LEN; k += 2) {
            float y0, y1, b0, b1;
            fma_rn2(y0, y1, py[k], py[k + 1], Qv, Rv);
            add_rz2(b0, b1, y0, y1, 8388608.0f);
            const uint32_t dv0 = __float_as_uint(b0) - fb.z, dv1 = __float_as_uint(b1) - fb.z;
            f(std::false_type{}, k, in_u && (dv0 < fb.w), dv0 * pitchS + K);
            f(std::false_type{}, k + 1, in_u && (dv1 < fb.w), dv1 * pitchS + K);
        }
    } else {
#pragma unroll
        for (int k = 0; k < LEN; k += 2) {
            uint32_t bu0, bu1, bv0, bv1;
            tilted_pair(py[k], py[k + 1], cu, cv, cw, Cu, Cv, Cw, hv, bu0, bu1, bv0, bv1);
            const uint32_t du0 = bu0 - fb.x, du1 = bu1 - fb.x, dv0 = bv0 - fb.z, dv1 = bv1 - fb.z;
            f(std::false_type{}, k, (du0 < fb.y) && (dv0 < fb.w), (dv0 * pitch + du0 + tgt.y) * isc + ib);
            f(std::false_type{}, k + 1, (du1 < fb.y) && (dv1 < fb.w), (dv1 * pitch + du1 + tgt.y) * isc + ib);
        }
    }
    return 1;
}

// FAST-contract part of the column walker (below), from the column's numerators
// C_u, C_v, C_w = fma(c.x, px, c.w) + c.z * pz; same calls and return value.  py2 holds
// the column's y positions in pairs {py[2m], py[2m + 1]}.
template <int LEN, typename F>
__device__ __forceinline__ int walk_fast(const ProjMeta &M, const LaunchArgs &a, float Cu, float Cv, float Cw,
                                         const uint64_t (&py2)[LEN / 2], F &&f)
{
    static_assert(LEN % 2 == 0, "columns are walked two voxels at a time");
    const uint4 tgt = M.tgt;
    const uint32_t pitch = tgt.x;
    const uint4 fb = M.fast;
    const float hv = a.half_minus_off;
    const uint64_t magic = f2pack(8388608.0f, 8388608.0f);
    if (M.flags.z) {
        // untilted: u, w and 1/w are column invariants, v = fma(py, Qv, Rv)
        const float rw = __frcp_rn(Cw);
        const float Qv = __fmul_rn(M.cv.y, rw), Rv = __fmaf_rn(Cv, rw, hv);
        const uint64_t Q2 = f2pack(Qv, Qv), R2 = f2pack(Rv, Rv);
        const uint32_t du = fdist(__fmaf_rn(Cu, rw, 0.5f), fb.x);
        if (M.flags.w) {
            // dv = bits(fadd_rz(yv, 2^23)) - fb.z is in [0, rows) for every voxel, so the
            // index dv * pitch + du + off is bits * pitch + (du + off - fb.z * pitch) mod 2^32
            const uint32_t K = du + tgt.y - fb.z * pitch;
#pragma unroll
            for (int k = 0; k < LEN; k += 2) {
                uint32_t b0, b1;
                u2unpack(addrz2(fma2(py2[k >> 1], Q2, R2), magic), b0, b1);
                f(std::true_type{}, k, true, b0 * pitch + K);
                f(std::true_type{}, k + 1, true, b1 * pitch + K);
            }
            return 2;
        }
        const bool in_u = du < fb.y;
        if (!__any_sync(0xffffffffu, in_u)) return 0;
        const uint32_t K = du + tgt.y;
#pragma unroll
        for (int k = 0; k < LEN; k += 2) {
            uint32_t b0, b1;
            u2unpack(addrz2(fma2(py2[k >> 1], Q2, R2), magic), b0, b1);
            const uint32_t dv0 = b0 - fb.z, dv1 = b1 - fb.z;
            f(std::false_type{}, k, in_u && (dv0 < fb.w), dv0 * pitch + K);
            f(std::false_type{}, k + 1, in_u && (dv1 < fb.w), dv1 * pitch + K);
        }
        return 1;
    }
    Packed kp;
    kp.magic = magic;
    kp.cuy = f2pack(M.cu.y, M.cu.y);
    kp.cvy = f2pack(M.cv.y, M.cv.y);
    kp.cwy = f2pack(M.cw.y, M.cw.y);
    kp.Cu = f2pack(Cu, Cu);
    kp.Cv = f2pack(Cv, Cv);
    kp.Cw = f2pack(Cw, Cw);
    kp.half = f2pack(0.5f, 0.5f);
    kp.hv = f2pack(hv, hv);
    if (M.flags.w) {
        const uint32_t Ku = tgt.y - fb.z * pitch - fb.x;
#pragma unroll
        for (int k = 0; k < LEN; k += 2) {
            uint64_t bu, bv;
            tilted_pair(py2[k >> 1], kp, bu, bv);
            uint32_t bu0, bu1, bv0, bv1;
            u2unpack(bu, bu0, bu1);
            u2unpack(bv, bv0, bv1);
            f(std::true_type{}, k, true, bv0 * pitch + bu0 + Ku);
            f(std::true_type{}, k + 1, true, bv1 * pitch + bu1 + Ku);
        }
        return 2;
    }
#pragma unroll
    for (int k = 0; k < LEN; k += 2) {
        uint64_t bu, bv;
        tilted_pair(py2[k >> 1], kp, bu, bv);
        uint32_t bu0, bu1, bv0, bv1;
        u2unpack(bu, bu0, bu1);
        u2unpack(bv, bv0, bv1);
        const uint32_t du0 = bu0 - fb.x, du1 = bu1 - fb.x, dv0 = bv0 - fb.z, dv1 = bv1 - fb.z;
        f(std::false_type{}, k, (du0 < fb.y) && (dv0 < fb.w), dv0 * pitch + du0 + tgt.y);
        f(std::false_type{}, k + 1, (du1 < fb.y) && (dv1 < fb.w), dv1 * pitch + du1 + tgt.y);
    }
    return 1;
}

// STRICT-contract walk of an untilted column (same calls and return value as walk_fast),
// bit-identical to the reference's per-voxel division: n_v = ((c.x*px + c.y*py) + c.z*pz)
// + c.w in the reference's order (c.y*py = Tk[k], formed by compute_meta), v = n_v / n_w by
// div_exact with the column's n_w, and the pixel by pix_bits2.  Returns -1, without calling f, when the projection's operands
// failed div_exact's screen over the brick (compute_meta; the caller then divides per
// voxel).
// CHUNK < LEN walks the column as LEN / CHUNK unrolled chunks in a rolled loop (fewer
// values live at once); f then sees k whose low bits are compile-time constants.
// isc / ib as in walk_fast: f receives idx * isc + ib.
template <int LEN, int CHUNK = LEN, typename F>
__device__ __forceinline__ int walk_exact(const ProjMeta &M, const LaunchArgs &a, float nu, float nw, float Pv,
                                          float Rv, const float *__restrict__ Tk, F &&f, uint32_t isc = 1u,
                                          uint32_t ib = 0u)
{
    static_assert(LEN % 2 == 0 && CHUNK % 4 == 0 && LEN % CHUNK == 0, "columns are walked two voxels at a time");
    const float4 cv = M.cv;
    const int4 rc = M.rect;
    const uint4 tgt = M.tgt;
    const uint32_t pitch = tgt.x, pitchS = pitch * isc;
    if (!(M.flags.z & 2)) return -1;  // uniform over the projection
    const float y = __frcp_rn(nw);
    const float ylo = __fmul_rn(__fmaf_rn(-nw, y, 1.0f), y);
    const float qu = div_exact(nu, -nw, y, ylo);
    const uint32_t du = pix_bits(qu) - (kMagic + (uint32_t)rc.x);
    const uint64_t P2 = f2pack(Pv, Pv), R2 = f2pack(Rv, Rv), W2 = f2pack(cv.w, cv.w);
    const uint64_t Y2 = f2pack(y, y), YL2 = f2pack(ylo, ylo), NB2 = f2pack(-nw, -nw);
    const uint64_t half = f2pack(0.5f, 0.5f), magic = f2pack(8388608.0f, 8388608.0f);
    const uint32_t base_v = kMagic + (uint32_t)a.row_off_f + (uint32_t)rc.z;
    auto qv = [&](int m) {  // Tk: shared memory, {T[2m], T[2m + 1]} as one 64-bit load
        const uint64_t nv = add2(add2(add2(P2, reinterpret_cast<const uint64_t *>(Tk)[m]), R2), W2);
        return div_exact2(nv, NB2, Y2, YL2);
    };
    if (M.flags.w) {
        // inside: every pixel is in the rectangle, idx = bits * pitch + K (mod 2^32)
        const uint32_t K = (du + tgt.y - base_v * pitch) * isc + ib;
#pragma unroll 1
        for (int c0 = 0; c0 < LEN; c0 += CHUNK) {
#pragma unroll
            for (int kk = 0; kk < CHUNK; kk += 2) {
                const int k = c0 + kk;
                uint32_t b0, b1;
                u2unpack(pix_bits2(qv(k >> 1), half, magic), b0, b1);
                f(std::true_type{}, k, true, b0 * pitchS + K);
                f(std::true_type{}, k + 1, true, b1 * pitchS + K);
            }
        }
        return 2;
    }
    const bool in_u = (du < (uint32_t)rc.y) && (qu != -0.5f);
    if (!__any_sync(0xffffffffu, in_u)) return 0;
    const uint32_t K = (du + tgt.y) * isc + ib;
    const float ex = __fsub_rn(a.row_off_f, 0.5f);  // pix_bits2's one exception
#pragma unroll 1
    for (int c0 = 0; c0 < LEN; c0 += CHUNK) {
#pragma unroll
        for (int kk = 0; kk < CHUNK; kk += 2) {
            const int k = c0 + kk;
            const uint64_t q = qv(k >> 1);
            uint32_t b0, b1;
            float q0, q1;
            u2unpack(pix_bits2(q, half, magic), b0, b1);
            f2unpack(q, q0, q1);
            const uint32_t dv0 = b0 - base_v, dv1 = b1 - base_v;
            f(std::false_type{}, k, in_u && (dv0 < (uint32_t)rc.w) && (q0 != ex), dv0 * pitchS + K);
            f(std::false_type{}, k + 1, in_u && (dv1 < (uint32_t)rc.w) && (q1 != ex), dv1 * pitchS + K);
        }
    }
    return 1;
}

// Column walker.  For the voxel column (ax, az) and y-positions py[0..LEN) (in pairs
// py2[m] = {py[2m], py[2m + 1]}), calls
// f(inside, k, in, idx) with idx the target index of ProjMeta.  Untilted projections
// (flags.z) hoist u, w and 1/w out of the column; the others evaluate the full
// contract per voxel.  In the FAST contract a brick whose footprint lies inside the
// viewport (flags.w) skips the bounds tests: `inside` is then std::true_type and
// `in` is true for every voxel.  Returns 0, without calling f, when no column of the
// warp meets the projection's u range; 2 when the inside path ran; 1 otherwise.
// CHUNK < LEN: the STRICT walks run as LEN / CHUNK unrolled chunks in a rolled loop (as in
// walk_exact); py2 must then be indexable at run time (the shared-memory pairs).
template <int ARITH, int LEN, int CHUNK = LEN, typename PY, typename F>
__device__ __forceinline__ int walk_column(const ProjMeta &M, const LaunchArgs &a, int ax, int az, const PY &py2,
                                           const float *__restrict__ Tk, F &&f)
{
    const float4 cu = M.cu, cv = M.cv, cw = M.cw;
    const uint4 tgt = M.tgt;
    const float px = pos<ARITH>(ax, a.voxel[0], a.origin[0]);
    const float pz = pos<ARITH>(az, a.voxel[2], a.origin[2]);
    const uint32_t pitch = tgt.x;
    if (ARITH == kFast)
        return walk_fast<LEN>(M, a, col_fast(cu, px, pz), col_fast(cv, px, pz), col_fast(cw, px, pz), py2, f);
    {  // STRICT
        const int4 rc = M.rect;
        const float off = a.row_off_f;
        if (M.flags.z) {
            // c.y == 0 in the u and w rows: c.y*py is a zero for every voxel of the column,
            // so n_u and n_w (up to the sign of a zero, which never changes a pixel) are
            // column invariants
            const float nu = num_strict(cu, px, 0.0f, pz);
            const float nw = num_strict(cw, px, 0.0f, pz);
            const int w = walk_exact<LEN, CHUNK>(M, a, nu, nw, __fmul_rn(cv.x, px), __fmul_rn(cv.z, pz), Tk, f);
            if (w >= 0) return w;
            const uint32_t du = (uint32_t)(__float2int_rz(roundf(__fdiv_rn(nu, nw))) - rc.x);
            const bool in_u = du < (uint32_t)rc.y;
            if (!__any_sync(0xffffffffu, in_u)) return 0;
            const uint32_t K = du + tgt.y;
            const float Pv = __fmul_rn(cv.x, px), Rv = __fmul_rn(cv.z, pz);
#pragma unroll 1
            for (int c0 = 0; c0 < LEN; c0 += CHUNK) {
#pragma unroll
                for (int kk = 0; kk < CHUNK; ++kk) {
                    const int k = c0 + kk;
                    const float nv = __fadd_rn(__fadd_rn(__fadd_rn(Pv, __fmul_rn(cv.y, ypos(py2, k))), Rv), cv.w);
                    const uint32_t dv = (uint32_t)(__float2int_rz(roundf(__fsub_rn(__fdiv_rn(nv, nw), off))) - rc.z);
                    f(std::false_type{}, k, in_u && (dv < (uint32_t)rc.w), dv * pitch + K);
                }
            }
        } else {
#pragma unroll 1
            for (int c0 = 0; c0 < LEN; c0 += CHUNK)
#pragma unroll
            for (int kk = 0; kk < CHUNK; ++kk) {
                const int k = c0 + kk;
                const float py = ypos(py2, k);
                const float nu = num_strict(cu, px, py, pz);
                const float nv = num_strict(cv, px, py, pz);
                const float nw = num_strict(cw, px, py, pz);
                const uint32_t du = (uint32_t)(__float2int_rz(roundf(__fdiv_rn(nu, nw))) - rc.x);
                const uint32_t dv = (uint32_t)(__float2int_rz(roundf(__fsub_rn(__fdiv_rn(nv, nw), off))) - rc.z);
                f(std::false_type{}, k, (du < (uint32_t)rc.y) && (dv < (uint32_t)rc.w), dv * pitch + du + tgt.y);
            }
        }
    }
    return 1;
}

// --------------------------------------------------------------------------------------
// forward
// --------------------------------------------------------------------------------------
// Forward brick shapes: 32 x by x 32 voxels, nt threads (cols = 1024 / nt columns of by
// layers per thread), G shared-memory tiles of `tile` pixels.  The narrow shape serves the
// FAST contract and the batched kernels; the STRICT contract's per-column work (reciprocal,
// u pixel, the packing of the column's constants) is a larger share of a voxel's, so its
// single-problem forward walks 16-layer columns (the tall shape) to halve that share.
template <int BY_, int NT_, int TC_>
struct FwdShape {
    static constexpr int by = BY_, nt = NT_, tile = TC_, warps = NT_ / 32, cols = BX * BZ / NT_;
    static constexpr size_t smem = (size_t)(BY_ / 4 * BZ * VSTRIDE + G * TC_) * sizeof(uint32_t);
    static_assert(BY_ % 4 == 0 && BY_ <= 16 && BX * BZ % NT_ == 0, "forward brick shape");
};
using FwdNarrow = FwdShape<BY, NT, TILE_CAP>;
using FwdTall = FwdShape<16, 512, 2048>;
constexpr size_t kFwdSmem = FwdNarrow::smem;

// One forward work unit: brick `brick` (x fastest, then z, then y) against the
// projection run `split` (entries [split * per_split, (split + 1) * per_split)).
// Called by every thread of the CTA; returns with the CTA converged.
template <int ARITH, bool LIST, typename SH = FwdNarrow>
__device__ __forceinline__ void forward_unit(const float *__restrict__ vol, uint32_t *__restrict__ sum,
                                             const xpr_projdata *__restrict__ pd, const LaunchArgs &a,
                                             uint32_t brick, uint32_t split, int bricks_x, int bricks_z,
                                             uint32_t *smem, ProjMeta *s_meta)
{
    constexpr int BYF = SH::by, NTF = SH::nt, TCF = SH::tile, NW = SH::warps, CPT = SH::cols;
    // fixed-point values [BYF / 4][BZ][VSTRIDE]: layers 4m .. 4m + 3 of (x, z) are adjacent
    // words, so a thread reads four of its column's voxels with one 128-bit load
    uint32_t *s_val = smem;
    uint32_t *s_tile = smem + BYF / 4 * BZ * VSTRIDE;   // [G][TCF]

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int b = (int)brick;
    const int bxi = b % bricks_x;
    b /= bricks_x;
    const int bzi = b % bricks_z;
    const int byi = b / bricks_z;
    const int x0 = bxi * BX, y0 = byi * BYF, z0 = bzi * BZ;
    const int sx = a.size[0], sy = a.size[1], sz = a.size[2];

    bool any = false;
    for (int i = threadIdx.x; i < BX * BYF * BZ; i += NTF) {
        const int x = i & 31, z = (i >> 5) & 31, y = i >> 10;
        const int gx = x0 + x, gy = y0 + y, gz = z0 + z;
        uint32_t v = 0;
        if (gx < sx && gy < sy && gz < sz) v = float_to_fixed(__ldg(&vol[((size_t)gy * sz + gz) * sx + gx]));
        s_val[((y >> 2) * BZ + z) * VSTRIDE + 4 * x + (y & 3)] = v;
        any |= (v != 0u);
    }
    for (int i = threadIdx.x; i < G * TCF; i += NTF) s_tile[i] = 0u;
    // the column's y positions: registers for 8-layer columns; for 16-layer columns (STRICT,
    // whose exact walk reads only the c_v.y*py products) in shared memory as pairs, for the
    // per-voxel fallback
    constexpr bool PYREG = BYF <= 8;
    float py[PYREG ? BYF : 2];
    __shared__ __align__(16) uint64_t s_py2[8];
    if (PYREG) {
#pragma unroll
        for (int k = 0; k < BYF; ++k) py[k] = pos<ARITH>(a.vmin[1] + y0 + k, a.voxel[1], a.origin[1]);
    } else if (threadIdx.x < BYF / 2) {
        const int k = 2 * (int)threadIdx.x;
        s_py2[threadIdx.x] = f2pack(pos<ARITH>(a.vmin[1] + y0 + k, a.voxel[1], a.origin[1]),
                                    pos<ARITH>(a.vmin[1] + y0 + k + 1, a.voxel[1], a.origin[1]));
    }
    auto with_py = [&](auto &&fn) {
        if constexpr (PYREG) fn(py);
        else fn(s_py2);
    };
    // the metadata of up to MCAP projections at a time (s_meta holds MCAP entries), one group
    // of G per warp, all warps at once: the first chunk's before the barrier that tests the
    // brick.  A group then takes two barriers (tiles complete, tiles flushed).
    const int e_begin = (int)split * (int)a.per_split;
    const int e_end = min((int)a.n_entries, e_begin + (int)a.per_split);
    // tiles are flushed by bulk reductions (the TMA unit adds each tile row to the sums)
    // when every row can start on a 16-byte boundary in both memories; else by threads
    const bool bulk = !(reinterpret_cast<uintptr_t>(sum) & 15u) && !(a.det_w & 3u) && !(a.img_stride & 3u);
    auto prepare = [&](int c0, int c1) {
        for (int w = warp; w * G < c1 - c0; w += NW)
            compute_meta<ARITH, LIST, false, TCF>(s_meta + w * G, pd, a, c0 + w * G, c1, x0, y0, z0, BX, BYF, BZ,
                                                  lane, bulk);
    };
    prepare(e_begin, min(e_end, e_begin + MCAP));
    if (!__syncthreads_or(any)) return;   // an all-zero brick adds nothing

    for (int e0 = e_begin; e0 < e_end; e0 += G) {
        const int buf = (e0 - e_begin) % MCAP;
        if (buf == 0 && e0 > e_begin) {
            prepare(e0, min(e_end, e0 + MCAP));
            __syncthreads();
        }
#pragma unroll 1
        for (int g = 0; g < G; ++g) {
            // a register copy: the walk's shared-memory atomics would otherwise force the
            // metadata to be re-read from shared memory for every column
            const ProjMeta M = s_meta[buf + g];
            const int4 fl = M.flags;
            if (fl.x == kSkip) continue;
            uint32_t *tile = s_tile + g * TCF;
            // the tile's shared-window address: the tile walks below hand f the atomic's
            // address (4 * index + tile_s), formed by their one multiply-add per voxel
            const uint32_t tile_s = (uint32_t)__cvta_generic_to_shared(tile);
            const bool orx = fl.y;
            if constexpr (ARITH == kFast) if (fl.x == kTile) {
                // FAST into a tile: one lane coordinate is the thread's for all of its columns,
                // so its share of the column numerators C = fma(c.x, px, c.w) + c.z * pz is
                // computed once per projection
                const float4 cu = M.cu, cv = M.cv, cw = M.cw;
                auto splat = [&](const uint4 *vals, float Cu, float Cv, float Cw) {
                    uint4 quad;
                    // a zero adds nothing to a shared-memory tile; no test for it
                    walk_fast<BYF>(M, a, Cu, Cv, Cw, py, [&](auto, int k, bool in, uint32_t saddr) {
                        if (!(k & 3)) quad = vals[(k >> 2) * (BZ * VSTRIDE / 4)];
                        const uint32_t v = (k & 2) ? ((k & 1) ? quad.w : quad.z) : ((k & 1) ? quad.y : quad.x);
                        if (in) red_shared_add(saddr, v);
                    }, 4u, tile_s);
                };
                if (orx) {
                    const float pz = pos<kFast>(a.vmin[2] + z0 + lane, a.voxel[2], a.origin[2]);
                    const float Pu = __fmul_rn(cu.z, pz), Pv = __fmul_rn(cv.z, pz), Pw = __fmul_rn(cw.z, pz);
#pragma unroll 1
                    for (int j = 0; j < CPT; ++j) {
                        const int cx = warp + NW * j;
                        const float px = pos<kFast>(a.vmin[0] + x0 + cx, a.voxel[0], a.origin[0]);
                        splat(reinterpret_cast<const uint4 *>(s_val + lane * VSTRIDE + 4 * cx),
                              __fadd_rn(__fmaf_rn(cu.x, px, cu.w), Pu), __fadd_rn(__fmaf_rn(cv.x, px, cv.w), Pv),
                              __fadd_rn(__fmaf_rn(cw.x, px, cw.w), Pw));
                    }
                } else {
                    const float px = pos<kFast>(a.vmin[0] + x0 + lane, a.voxel[0], a.origin[0]);
                    const float Au = __fmaf_rn(cu.x, px, cu.w), Av = __fmaf_rn(cv.x, px, cv.w),
                                Aw = __fmaf_rn(cw.x, px, cw.w);
#pragma unroll 1
                    for (int j = 0; j < CPT; ++j) {
                        const int cz = warp + NW * j;
                        const float pz = pos<kFast>(a.vmin[2] + z0 + cz, a.voxel[2], a.origin[2]);
                        splat(reinterpret_cast<const uint4 *>(s_val + cz * VSTRIDE + 4 * lane),
                              __fadd_rn(Au, __fmul_rn(cu.z, pz)), __fadd_rn(Av, __fmul_rn(cv.z, pz)),
                              __fadd_rn(Aw, __fmul_rn(cw.z, pz)));
                    }
                }
                continue;
            }
            if constexpr (ARITH == kStrict) if (fl.x == kTile && (fl.z & 2)) {
                // STRICT into a tile, untilted and screened: n_u and n_w are (c.x*px + c.z*pz) + c.w
                // (c.y*py is a zero), so the lane coordinate's product in every row is formed once
                // per projection; walk_exact divides per voxel with the column's reciprocal
                const float4 cu = M.cu, cv = M.cv, cw = M.cw;
                auto splat = [&](const uint4 *vals, float nu, float nw, float Pv, float Rv) {
                    uint4 quad;
                    // a zero adds nothing to a shared-memory tile; no test for it
                    walk_exact<BYF, 8>(M, a, nu, nw, Pv, Rv, s_meta[buf + g].T, [&](auto, int k, bool in, uint32_t saddr) {
                        if (!(k & 3)) quad = vals[(k >> 2) * (BZ * VSTRIDE / 4)];
                        const uint32_t v = (k & 2) ? ((k & 1) ? quad.w : quad.z) : ((k & 1) ? quad.y : quad.x);
                        if (in) red_shared_add(saddr, v);
                    }, 4u, tile_s);
                };
                if (orx) {
                    const float pz = pos<kStrict>(a.vmin[2] + z0 + lane, a.voxel[2], a.origin[2]);
                    const float Bu = __fmul_rn(cu.z, pz), Bw = __fmul_rn(cw.z, pz), Rv = __fmul_rn(cv.z, pz);
#pragma unroll 1
                    for (int j = 0; j < CPT; ++j) {
                        const int cx = warp + NW * j;
                        const float px = pos<kStrict>(a.vmin[0] + x0 + cx, a.voxel[0], a.origin[0]);
                        splat(reinterpret_cast<const uint4 *>(s_val + lane * VSTRIDE + 4 * cx),
                              __fadd_rn(__fadd_rn(__fmul_rn(cu.x, px), Bu), cu.w),
                              __fadd_rn(__fadd_rn(__fmul_rn(cw.x, px), Bw), cw.w), __fmul_rn(cv.x, px), Rv);
                    }
                } else {
                    const float px = pos<kStrict>(a.vmin[0] + x0 + lane, a.voxel[0], a.origin[0]);
                    const float Au = __fmul_rn(cu.x, px), Aw = __fmul_rn(cw.x, px), Pv = __fmul_rn(cv.x, px);
#pragma unroll 1
                    for (int j = 0; j < CPT; ++j) {
                        const int cz = warp + NW * j;
                        const float pz = pos<kStrict>(a.vmin[2] + z0 + cz, a.voxel[2], a.origin[2]);
                        splat(reinterpret_cast<const uint4 *>(s_val + cz * VSTRIDE + 4 * lane),
                              __fadd_rn(__fadd_rn(Au, __fmul_rn(cu.z, pz)), cu.w),
                              __fadd_rn(__fadd_rn(Aw, __fmul_rn(cw.z, pz)), cw.w), Pv, __fmul_rn(cv.z, pz));
                    }
                }
                continue;
            }
            // CPT columns per thread; lanes run across the ray so a warp hits distinct pixels
#pragma unroll 1
            for (int j = 0; j < CPT; ++j) {
                const int cx = orx ? warp + NW * j : lane;
                const int cz = orx ? lane : warp + NW * j;
                const uint4 *vals = reinterpret_cast<const uint4 *>(s_val + cz * VSTRIDE + 4 * cx);
                uint4 quad;
                const int ax = a.vmin[0] + x0 + cx, az = a.vmin[2] + z0 + cz;
                if (ARITH != kFast && fl.x == kTile) {
                    // a zero adds nothing to a shared-memory tile; no test for it
                    with_py([&](const auto &pyv) {
                        walk_column<ARITH, BYF, (BYF > 8 ? 8 : BYF)>(M, a, ax, az, pyv, s_meta[buf + g].T, [&](auto, int k, bool in, uint32_t idx) {
                            if (!(k & 3)) quad = vals[(k >> 2) * (BZ * VSTRIDE / 4)];
                            const uint32_t v = (k & 2) ? ((k & 1) ? quad.w : quad.z) : ((k & 1) ? quad.y : quad.x);
                            if (in) atomicAdd(&tile[idx], v);
                        });
                    });
                } else {
                    with_py([&](const auto &pyv) {
                        walk_column<ARITH, BYF, (BYF > 8 ? 8 : BYF)>(M, a, ax, az, pyv, s_meta[buf + g].T, [&](auto, int k, bool in, uint32_t idx) {
                            if (!(k & 3)) quad = vals[(k >> 2) * (BZ * VSTRIDE / 4)];
                            const uint32_t v = (k & 2) ? ((k & 1) ? quad.w : quad.z) : ((k & 1) ? quad.y : quad.x);
                            if (in & (v != 0u)) atomicAdd(&sum[idx], v);
                        });
                    });
                }
            }
        }
        if (bulk) fence_async_smem();  // the tiles' atomics before the TMA unit reads them
        __syncthreads();
        if (bulk) {
            // warp g flushes tile g: lane q adds rows q, q + 32, ... to the sums with one bulk
            // reduction each (rows of `pitch` words from column rect.x, inside the image row),
            // waits until the TMA unit has read them, then the warp zeroes the tile
            if (warp < G) {
                const ProjMeta &M = s_meta[buf + warp];
                if (M.flags.x == kTile) {
                    uint32_t *tile = s_tile + warp * TCF;
                    const int4 rc = M.rect;
                    const uint32_t pitch = M.tgt.x;
                    for (int r = lane; r < rc.w; r += 32)
                        bulk_add_u32(sum + M.tgt.z + (uint32_t)(rc.z + r) * a.det_w + (uint32_t)rc.x, tile + r * pitch,
                                     pitch * 4u);
                    bulk_commit();
                    bulk_wait_read();
                    __syncwarp();
                    uint4 *t4 = reinterpret_cast<uint4 *>(tile);
                    for (uint32_t i = lane; i < pitch * (uint32_t)rc.w / 4u; i += 32) t4[i] = make_uint4(0u, 0u, 0u, 0u);
                }
            }
        } else {
            // flush the tiles: one global atomic per touched pixel, coalesced along rows
#pragma unroll 1
            for (int g = 0; g < G; ++g) {
                const ProjMeta &M = s_meta[buf + g];
                if (M.flags.x != kTile) continue;
                uint32_t *tile = s_tile + g * TCF;
                const int4 rc = M.rect;
                const int tw = rc.y, th = rc.w;
                for (int r = warp; r < th; r += NW) {
                    uint32_t *dst = sum + M.tgt.z + (uint32_t)(rc.z + r) * a.det_w + (uint32_t)rc.x;
                    for (int c = lane; c < tw; c += 32) {
                        const uint32_t v = tile[r * tw + c];
                        if (v) {
                            tile[r * tw + c] = 0u;
                            atomicAdd(dst + c, v);
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    if (bulk && warp < G) bulk_wait_all();  // the unit's reductions complete before it ends
}

template <int ARITH, bool LIST, typename SH>
__global__ void __launch_bounds__(SH::nt, 1024 / SH::nt)
    k_forward_tiled(const float *__restrict__ vol, uint32_t *__restrict__ sum, const xpr_projdata *__restrict__ pd,
                    const LaunchArgs a, int bricks_x, int bricks_z)
{
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ ProjMeta s_meta[MCAP];
    forward_unit<ARITH, LIST, SH>(vol, sum, pd, a, blockIdx.x, blockIdx.y, bricks_x, bricks_z, smem, s_meta);
}

// the forward shape of each contract's single-problem kernel
template <int ARITH>
using FwdShapeOf = typename std::conditional<ARITH == kStrict, FwdTall, FwdNarrow>::type;

// Work-items of the reference NDRange padding (kernel.hpp:73-81, H5): one thread each,
// voxel coordinates from to3D() (utils.cl:39-45), all projections, global atomics.
template <int ARITH, bool LIST, bool FWD, bool NANSKIP, int DT>
__global__ void k_pad_items(float *vol, uint32_t *sum, const void *ratio, const xpr_projdata *__restrict__ pd,
                            const LaunchArgs a, uint64_t id_begin, uint64_t id_end)
{
    const uint64_t id = id_begin + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (id >= id_end) return;
    const uint64_t sx = (uint64_t)a.size[0], sz = (uint64_t)a.size[2];
    const uint64_t yy = id / (sx * sz), rem = id - yy * sx * sz;
    const int ax = a.vmin[0] + (int)(rem % sx), az = a.vmin[2] + (int)(rem / sx), ay = a.vmin[1] + (int)yy;
    float px, py, pz;
    if (ARITH == kFast) {
        px = __fmaf_rn((float)ax, a.voxel[0], a.origin[0]);
        py = __fmaf_rn((float)ay, a.voxel[1], a.origin[1]);
        pz = __fmaf_rn((float)az, a.voxel[2], a.origin[2]);
    } else {
        px = __fadd_rn(__fmul_rn(__uint2float_rn((uint32_t)ax), a.voxel[0]), a.origin[0]);
        py = __fadd_rn(__fmul_rn(__uint2float_rn((uint32_t)ay), a.voxel[1]), a.origin[1]);
        pz = __fadd_rn(__fmul_rn(__uint2float_rn((uint32_t)az), a.voxel[2]), a.origin[2]);
    }
    const uint32_t value = FWD ? float_to_fixed(vol[id]) : 0u;
    float s = 0.0f;
    uint32_t cnt = 0u;
    for (uint32_t e = 0; e < a.n_entries; ++e) {
        const uint32_t pidx = LIST ? (uint32_t)a.list_mvp[e] : e;
        const uint32_t img = LIST ? (uint32_t)a.list_img[e] : e / a.modules;
        if (pidx >= a.n_pd || img >= a.n_images) continue;
        const float *m = pd[pidx].mvp;
        const float *vp = pd[pidx].vp;
        const int l = max((int)ceilf(vp[0]), 0), r = min((int)ceilf(vp[1]), (int)a.det_w);
        const int bb = max((int)ceilf(vp[2]), 0), t = min((int)ceilf(vp[3]), (int)a.rows);
        int iu, iv;
        bool in;
        if (ARITH == kFast) {
            const float4 c0 = make_float4(m[0], m[1], m[2], m[3]), c1 = make_float4(m[4], m[5], m[6], m[7]);
            const float4 c3 = make_float4(m[12], m[13], m[14], m[15]);
            const float rw = __frcp_rn(__fmaf_rn(c3.y, py, col_fast(c3, px, pz)));
            const float yu = __fmaf_rn(py, __fmul_rn(c0.y, rw), __fmaf_rn(col_fast(c0, px, pz), rw, 0.5f));
            const float yv = __fmaf_rn(py, __fmul_rn(c1.y, rw), __fmaf_rn(col_fast(c1, px, pz), rw, a.half_minus_off));
            in = yu >= (float)l && yu < (float)r && yv >= (float)bb && yv < (float)t;
            iu = in ? (int)floorf(yu) : 0;
            iv = in ? (int)floorf(yv) : 0;
        } else {
            const float nu = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], px), __fmul_rn(m[1], py)), __fmul_rn(m[2], pz)), m[3]);
            const float nv = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[4], px), __fmul_rn(m[5], py)), __fmul_rn(m[6], pz)), m[7]);
            const float nw = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[12], px), __fmul_rn(m[13], py)), __fmul_rn(m[14], pz)), m[15]);
            iu = __float2int_rz(roundf(__fdiv_rn(nu, nw)));
            iv = __float2int_rz(roundf(__fsub_rn(__fdiv_rn(nv, nw), a.row_off_f)));
            in = iu >= l && iu < r && iv >= bb && iv < t;
        }
        if (!in) continue;
        const uint32_t gi = img * a.img_stride + (uint32_t)iv * a.det_w + (uint32_t)iu;
        if (FWD) {
            atomicAdd(&sum[gi], value);
        } else {
            float rr;
            if (DT == kF32) rr = ((const float *)ratio)[gi];
            else if (DT == kBF16) rr = __bfloat162float(((const __nv_bfloat16 *)ratio)[gi]);
            else rr = __half2float(((const __half *)ratio)[gi]);
            if (NANSKIP && rr != rr) continue;
            s = __fadd_rn(s, rr);
            cnt += 1u;
        }
    }
    if (!FWD) vol[id] = __fmul_rn(vol[id], p_expf(__fdiv_rn(s, __uint2float_rn(cnt))));
}

// --------------------------------------------------------------------------------------
// backward
// --------------------------------------------------------------------------------------
// The stored bits of ratio element i (zero-extended for the 16-bit types) and their
// value: a gather returns raw bits so that an out-of-bounds pair can keep 0 (the bits
// of +0.0 in every type) without a select after the conversion.
template <int DT>
__device__ __forceinline__ uint32_t load_ratio_bits(const void *ratio, uint32_t i)
{
    if (DT == kF32) return __float_as_uint(__ldg((const float *)ratio + i));
    return (uint32_t)__ldg((const unsigned short *)ratio + i);
}
// a quiet NaN in each storage type's bits
template <int DT>
constexpr uint32_t kNaNBits = DT == kF32 ? 0x7fc00000u : (DT == kBF16 ? 0x7fc0u : 0x7e00u);

template <int DT>
__device__ __forceinline__ float ratio_from_bits(uint32_t b)
{
    if (DT == kF32) return __uint_as_float(b);
    if (DT == kBF16) return __uint_as_float(b << 16);  // bf16 is the high half of an f32
    return __half2float(__ushort_as_half((unsigned short)b));
}

// One backward work unit: the brick of 32 x CB x 8 voxels `brick` (x fastest, then z,
// then y); every thread owns one voxel column of CB layers.  CB (16 or 8) trades
// registers for fewer projection-metadata passes per voxel.
template <int ARITH, bool LIST, bool NANSKIP, int DT, int CB>
__device__ __forceinline__ void backward_unit(float *__restrict__ vol, const void *__restrict__ ratio,
                                              const xpr_projdata *__restrict__ pd, const LaunchArgs &a,
                                              uint32_t brick, int bricks_x, int bricks_z, ProjMeta *s_meta)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int b = (int)brick;
    const int bxi = b % bricks_x;
    b /= bricks_x;
    const int bzi = b % bricks_z;
    const int byi = b / bricks_z;
    const int x0 = bxi * BX, y0 = byi * CB, z0 = bzi * BWD_BZ;
    // thread = the voxel column (x0 + lane, z0 + warp), layers y0 .. y0 + CB
    const int ax = a.vmin[0] + x0 + lane, az = a.vmin[2] + z0 + warp;

    // the column's y positions are the same for every thread: kept in shared memory
    // (read as broadcasts), which leaves the registers to the sums and the gathers in flight
    __shared__ __align__(16) uint64_t py[CB / 2];  // in pairs {py[2m], py[2m + 1]}
    float s[CB];
    uint32_t n2[CB / 2];  // in-bounds counts, two 16-bit halves per word (k even: low, odd: high)
    uint32_t n_inside = 0;  // projections walked on the inside path: every voxel of the column counted
    if (threadIdx.x < CB / 2) {
        const int k = 2 * (int)threadIdx.x;
        py[threadIdx.x] = f2pack(pos<ARITH>(a.vmin[1] + y0 + k, a.voxel[1], a.origin[1]),
                                 pos<ARITH>(a.vmin[1] + y0 + k + 1, a.voxel[1], a.origin[1]));
    }
#pragma unroll
    for (int k = 0; k < CB; ++k) s[k] = 0.0f;
#pragma unroll
    for (int k = 0; k < CB / 2; ++k) n2[k] = 0u;

    // the metadata of up to MCAP projections at a time (s_meta holds MCAP entries), one group
    // of G per warp, all warps at once; the walk only reads it, so a chunk takes two barriers
    const int n_entries = (int)a.n_entries;
    constexpr int NWB = NT / 32;
    for (int c0 = 0; c0 < n_entries; c0 += MCAP) {
        const int c1 = min(n_entries, c0 + MCAP);
        if (c0 > 0) __syncthreads();  // the previous chunk's metadata read by every warp
        for (int w = warp; w * G < c1 - c0; w += NWB)
            compute_meta<ARITH, LIST, true>(s_meta + w * G, pd, a, c0 + w * G, c1, x0, y0, z0, BX, CB, BWD_BZ, lane);
        __syncthreads();
#pragma unroll 1
        for (int e = 0; e < c1 - c0; ++e) {
            const ProjMeta &M = s_meta[e];
            if (M.flags.x == kSkip) continue;
            // the column's gathers are issued before any is consumed (all in flight together);
            // an out-of-bounds pair contributes r = 0, and s + 0 == s exactly (s is never -0).
            // Raw bits first, values after: the loads of the column stay independent of
            // any conversion, so they are all in flight together in every storage type.
            // consumed in two halves of CB / 2 gathers (each half all in flight), which keeps
            // the registers of the gathers in flight to CB / 2
            uint32_t rb[CB];
            auto consume = [&](int k0) {
#pragma unroll
                for (int k = k0; k < k0 + CB / 2; ++k) {
                    const float r = ratio_from_bits<DT>(rb[k]);
                    if (NANSKIP) {
                        if (r == r) {
                            s[k] = __fadd_rn(s[k], r);
                            n2[k >> 1] += (k & 1) ? 0x10000u : 1u;
                        }
                    } else {
                        s[k] = __fadd_rn(s[k], r);
                    }
                }
            };
            const int walked = walk_column<ARITH, CB>(M, a, ax, az, py, M.T, [&](auto inside, int k, bool in, uint32_t idx) {
                rb[k] = 0u;
                if (in) rb[k] = load_ratio_bits<DT>(ratio, idx);
                if constexpr (!decltype(inside)::value) {
                    if (!NANSKIP && in) n2[k >> 1] += (k & 1) ? 0x10000u : 1u;
                    if (NANSKIP && !in) rb[k] = kNaNBits<DT>;
                }
                if (k == CB / 2 - 1) consume(0);
            });
            if (!walked) continue;  // warp-uniform
            if (!NANSKIP && walked == 2) ++n_inside;
            consume(CB / 2);
        }
    }
    const int sx = a.size[0], sy = a.size[1], sz = a.size[2];
    const int x = x0 + lane, z = z0 + warp;
    if (x >= sx || z >= sz) return;  // after the last barrier of the unit
#pragma unroll
    for (int k = 0; k < CB; ++k) {
        const int y = y0 + k;
        if (y < sy) {
            const uint32_t cnt = ((k & 1) ? (n2[k >> 1] >> 16) : (n2[k >> 1] & 0xffffu)) + n_inside;
            float *p = vol + ((size_t)y * sz + z) * sx + x;
            *p = __fmul_rn(*p, p_expf(__fdiv_rn(s[k], __uint2float_rn(cnt))));
        }
    }
}


template <int ARITH, bool LIST, bool NANSKIP, int DT, int CB>
__global__ void __launch_bounds__(NT, 4)
    k_backward_tiled(float *__restrict__ vol, const void *__restrict__ ratio, const xpr_projdata *__restrict__ pd,
                     const LaunchArgs a, int bricks_x, int bricks_z)
{
    __shared__ ProjMeta s_meta[MCAP];
    backward_unit<ARITH, LIST, NANSKIP, DT, CB>(vol, ratio, pd, a, blockIdx.x, bricks_x, bricks_z, s_meta);
}

// --------------------------------------------------------------------------------------
// error, preprocessing, fill
// --------------------------------------------------------------------------------------
template <int DT>
__device__ __forceinline__ float load_any(const void *p, uint64_t i)
{
    if (DT == kF32) return ((const float *)p)[i];
    if (DT == kBF16) return __bfloat162float(((const __nv_bfloat16 *)p)[i]);
    return __half2float(((const __half *)p)[i]);
}
template <int DT>
__device__ __forceinline__ void store_any(void *p, uint64_t i, float v)
{
    if (DT == kF32) ((float *)p)[i] = v;
    else if (DT == kBF16) ((__nv_bfloat16 *)p)[i] = __float2bfloat16_rn(v);
    else ((__half *)p)[i] = __float2half_rn(v);
}
__device__ __forceinline__ float std_max(float a, float b) { return (a < b) ? b : a; }

template <int MODE, int IDT, int RDT, bool ZERO, bool RESID>
__global__ void k_error(const void *__restrict__ images, uint32_t *sum, void *ratio, uint64_t n, float w,
                        double *residual)
{
    double acc = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float ref = load_any<IDT>(images, i);
        const float got = fixed_to_float(sum[i]);
        float r;
        if (MODE == XPR_ERROR_STD) r = __fmul_rn(p_logf(fmaxf(__fdiv_rn(ref, fmaxf(got, kEps)), kEps)), w);
        else if (MODE == XPR_ERROR_FIRST_1C) r = p_logf(std_max(ref, kEps));
        else r = __fmul_rn(p_logf(std_max(__fdiv_rn(ref, std_max(got, kEps)), kEps)), w);
        store_any<RDT>(ratio, i, r);
        if (ZERO) sum[i] = 0u;
        if (RESID) acc += (double)r * (double)r;
    }
    if (RESID) {
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(residual, acc);
    }
}

// order-preserving float <-> int map for atomic min / max
__device__ __forceinline__ int ford(float f)
{
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float fordinv(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__device__ __forceinline__ bool is_normal(float v)
{
    const uint32_t e = (__float_as_uint(v) >> 23) & 0xffu;
    return e != 0u && e != 0xffu;
}

__global__ void k_minmax(const float *__restrict__ x, uint64_t n, float *minmax)
{
    float mn = FLT_MAX, mx = -FLT_MAX;
    bool anyv = false;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float v = x[i];
        if (is_normal(v)) {
            mn = fminf(mn, v);
            mx = fmaxf(mx, v);
            anyv = true;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    anyv = __any_sync(0xffffffffu, anyv);
    if ((threadIdx.x & 31) == 0 && anyv) {
        atomicMin((int *)&minmax[0], ford(mn));
        atomicMax((int *)&minmax[1], ford(mx));
    }
}

// minmax[] holds ford()-encoded values while the reduction runs
__global__ void k_minmax_encode(float *minmax, bool decode)
{
    if (threadIdx.x == 0) {
        if (!decode) {
            const int a = ford(minmax[0]), b = ford(minmax[1]);
            ((int *)minmax)[0] = a;
            ((int *)minmax)[1] = b;
        } else {
            const float a = fordinv(((int *)minmax)[0]), b = fordinv(((int *)minmax)[1]);
            minmax[0] = a;
            minmax[1] = b;
        }
    }
}

template <int ODT>
__global__ void k_preprocess(const float *__restrict__ x, void *out, uint64_t n, int normalize,
                             const float *__restrict__ minmax, int mlog)
{
    const float mn = normalize ? minmax[0] : 0.0f, mx = normalize ? minmax[1] : 0.0f;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        float v = x[i];
        if (normalize) v = is_normal(v) ? __fdiv_rn(__fsub_rn(v, mn), __fsub_rn(mx, mn)) : __fdiv_rn(__fadd_rn(mx, mn), 2.0f);
        if (mlog) {
            const float lo = 1.0f - kEps;
            float c = (lo < v) ? lo : v;          // std::min(v, 1 - eps)
            c = (c < kEps) ? kEps : c;            // std::max(., eps)
            v = -p_logf(c);
        }
        store_any<ODT>(out, i, v);
    }
}

// The preprocessing of k_preprocess applied to images [0, n_img) of W*H pixels in
// acquisition order, each written to its subset-major slot (j mod S) * Pc + j / S
// (dataset.hpp:133-140): one launch for a whole request's images.
template <int ODT>
__global__ void k_preprocess_reorder(const float *__restrict__ x, void *out, uint64_t wh, uint32_t n_img, uint32_t S,
                                     uint32_t Pc, int normalize, const float *__restrict__ minmax, int mlog)
{
    const float mn = normalize ? minmax[0] : 0.0f, mx = normalize ? minmax[1] : 0.0f;
    const uint64_t n = wh * n_img;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t j = i / wh, px = i - j * wh;
        const uint64_t slot = (j % S) * Pc + j / S;
        float v = x[i];
        if (normalize) v = is_normal(v) ? __fdiv_rn(__fsub_rn(v, mn), __fsub_rn(mx, mn)) : __fdiv_rn(__fadd_rn(mx, mn), 2.0f);
        if (mlog) {
            const float lo = 1.0f - kEps;
            float c = (lo < v) ? lo : v;          // std::min(v, 1 - eps)
            c = (c < kEps) ? kEps : c;            // std::max(., eps)
            v = -p_logf(c);
        }
        store_any<ODT>(out, slot * wh + px, v);
    }
}

__global__ void k_fill_u32(uint32_t *dst, uint32_t value, uint64_t count)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = value;
}

template <int ODT>
__global__ void k_convert(const float *__restrict__ x, void *out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        store_any<ODT>(out, i, x[i]);
}

// ======================================================================================
// batched (persistent) kernels: many independent problems per launch
// ======================================================================================
// A CTA claims work units from ticket[0] until they run out; the last CTA to leave
// (ticket[1] counts departures) puts both words back to zero for the next launch, so
// a batch's launches need no reset between them and capture into a graph as is.
__device__ __forceinline__ int find_item(const uint32_t *begins, size_t stride, int n_items, uint32_t unit)
{
    int lo = 0, hi = n_items - 1;  // last item with begin <= unit
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg((const uint32_t *)((const char *)begins + (size_t)mid * stride)) <= unit) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void ticket_depart(uint32_t *ticket)
{
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ticket[1], 1u) == gridDim.x - 1) {
            atomicExch(&ticket[0], 0u);
            atomicExch(&ticket[1], 0u);
        }
    }
}

template <int ARITH, typename SH = FwdNarrow>
__global__ void __launch_bounds__(SH::nt, 1024 / SH::nt)
    k_forward_batched(const BatchFwdItem *__restrict__ items, int n_items, uint32_t total_units, uint32_t *ticket)
{
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ ProjMeta s_meta[MCAP];
    __shared__ LaunchArgs s_a;
    __shared__ uint32_t s_unit;
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t u = atomicAdd(&ticket[0], 1u);
            int it = 0;
            if (u < total_units) {
                it = find_item(&items[0].unit_begin, sizeof(BatchFwdItem), n_items, u);
                s_a = items[it].a;
            }
            s_unit = u;
            s_item = it;
        }
        __syncthreads();
        const uint32_t u = s_unit;
        if (u >= total_units) break;
        const BatchFwdItem &I = items[s_item];
        const uint32_t local = u - I.unit_begin, splits = I.splits;
        forward_unit<ARITH, false, SH>(I.vol, I.sum, I.pd, s_a, local / splits, local % splits, I.bricks_x,
                                       I.bricks_z, smem, s_meta);
        __syncthreads();
    }
    ticket_depart(ticket);
}

template <int ARITH, int DT, int CB>
__global__ void __launch_bounds__(NT, 4)
    k_backward_batched(const BatchBwdItem *__restrict__ items, int n_items, uint32_t total_units, uint32_t *ticket)
{
    __shared__ ProjMeta s_meta[MCAP];
    __shared__ LaunchArgs s_a;
    __shared__ uint32_t s_unit;
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t u = atomicAdd(&ticket[0], 1u);
            int it = 0;
            if (u < total_units) {
                it = find_item(&items[0].unit_begin, sizeof(BatchBwdItem), n_items, u);
                s_a = items[it].a;
            }
            s_unit = u;
            s_item = it;
        }
        __syncthreads();
        const uint32_t u = s_unit;
        if (u >= total_units) break;
        const BatchBwdItem &I = items[s_item];
        backward_unit<ARITH, false, false, DT, CB>(I.vol, I.ratio, I.pd, s_a, u - I.unit_begin, I.bricks_x,
                                                   I.bricks_z, s_meta);
        __syncthreads();
    }
    ticket_depart(ticket);
}

// grid (x: chunks of an item, y: item)
template <int IDT, int RDT>
__global__ void k_error_batched(const BatchErrItem *__restrict__ items)
{
    const BatchErrItem I = items[blockIdx.y];
    double acc = 0.0;
    const bool resid = I.residual != nullptr;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < I.n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float ref = load_any<IDT>(I.images, i);
        const float got = I.first ? 1.0f : fixed_to_float(I.sum[i]);
        const float r = __fmul_rn(p_logf(fmaxf(__fdiv_rn(ref, fmaxf(got, kEps)), kEps)), I.weight);
        store_any<RDT>(I.ratio, i, r);
        I.sum[i] = 0u;
        if (resid) acc += (double)r * (double)r;
    }
    if (resid) {
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(I.residual, acc);
    }
}

__global__ void k_fill_batched(const BatchFillItem *__restrict__ items)
{
    const BatchFillItem I = items[blockIdx.y];
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < I.n; i += (uint64_t)gridDim.x * blockDim.x)
        I.dst[i] = I.value;
}

// ======================================================================================
// launchers
// ======================================================================================
static inline unsigned stream_grid(uint64_t n, const DeviceInfo &dev)
{
    const uint64_t want = (n + 255) / 256;
    const uint64_t cap = (uint64_t)dev.sm_count * 8;
    return (unsigned)std::max<uint64_t>(1, std::min(want, cap));
}

const char *make_launch_args(const xpr_launch *L, uint32_t n_pd, LaunchArgs *a)
{
    if (!L) return "launch descriptor is NULL";
    for (int i = 0; i < 3; ++i) {
        if (L->vmin[i] < 0 || L->vmax[i] <= L->vmin[i]) return "volume box must satisfy 0 <= vmin < vmax";
        a->vmin[i] = L->vmin[i];
        a->size[i] = L->vmax[i] - L->vmin[i];
        a->origin[i] = L->origin[i];
        a->voxel[i] = L->voxel[i];
    }
    if (L->det_w == 0 || L->rows == 0) return "detector width and rows must be positive";
    if (L->det_w > (1u << 22) || L->rows > (1u << 22)) return "detector width / rows exceed 2^22";
    if (L->row_offset < 0 || L->row_offset > (1 << 22)) return "row_offset must be in [0, 2^22]";
    if (L->arith != XPR_ARITH_STRICT && L->arith != XPR_ARITH_FAST) return "unknown arith mode";
    if (n_pd == 0) return "no ProjData";
    const uint32_t M = L->modules ? L->modules : 1u;
    a->det_w = L->det_w;
    a->rows = L->rows;
    a->row_off_f = (float)(uint32_t)L->row_offset;
    a->half_minus_off = 0.5f - (float)L->row_offset;
    a->modules = M;
    a->n_pd = n_pd;
    a->img_stride = L->det_w * L->rows;
    if (L->list_mvp || L->list_img) {
        if (!L->list_mvp || !L->list_img) return "both index lists are required";
        a->list_mvp = L->list_mvp;
        a->list_img = L->list_img;
        a->n_entries = L->n_list;
        a->n_images = L->n_angles;
    } else {
        a->list_mvp = nullptr;
        a->list_img = nullptr;
        if ((uint64_t)L->n_angles * M > n_pd) return "n_angles * modules exceeds the ProjData count";
        a->n_entries = L->n_angles * M;
        a->n_images = L->n_angles;
    }
    if ((uint64_t)a->img_stride * a->n_images >= (1ull << 32)) return "detector buffer exceeds 2^32 elements";
    if (a->n_entries > 65535u) return "more than 65535 (angle, module) entries in one launch";
    const uint64_t nvox = (uint64_t)a->size[0] * a->size[1] * a->size[2];
    if (nvox + 64 >= (1ull << 40)) return "volume box too large";
    a->per_split = a->n_entries;
    return nullptr;
}

static bool g_attr_done[64];

cudaError_t prepare_device_kernels()
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && g_attr_done[dev]) return cudaSuccess;
    const int smem = (int)kFwdSmem;
    using FwdFn = void (*)(const float *, uint32_t *, const xpr_projdata *, const LaunchArgs, int, int);
    const struct { FwdFn f; size_t smem; } fns[] = {
        {k_forward_tiled<kStrict, false, FwdShapeOf<kStrict>>, FwdShapeOf<kStrict>::smem},
        {k_forward_tiled<kStrict, true, FwdShapeOf<kStrict>>, FwdShapeOf<kStrict>::smem},
        {k_forward_tiled<kFast, false, FwdShapeOf<kFast>>, FwdShapeOf<kFast>::smem},
        {k_forward_tiled<kFast, true, FwdShapeOf<kFast>>, FwdShapeOf<kFast>::smem}};
    for (const auto &f : fns) {
        e = cudaFuncSetAttribute(f.f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f.smem);
        if (e != cudaSuccess) return e;
    }
    using BFwdFn = void (*)(const BatchFwdItem *, int, uint32_t, uint32_t *);
    const struct { BFwdFn f; size_t smem; } bfns[] = {{k_forward_batched<kStrict>, (size_t)smem},
                                                      {k_forward_batched<kFast>, (size_t)smem},
                                                      {k_forward_batched<kStrict, FwdTall>, FwdTall::smem}};
    for (const auto &f : bfns) {
        e = cudaFuncSetAttribute(f.f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f.smem);
        if (e != cudaSuccess) return e;
    }
    if (dev < 64) g_attr_done[dev] = true;
    return cudaSuccess;
}

// the single-problem forward of contract AR over its brick shape
template <int AR>
static cudaError_t forward_tiled(const float *vol, uint32_t *sum, const xpr_projdata *pd, LaunchArgs a,
                                 const DeviceInfo &dev, cudaStream_t s)
{
    using SH = FwdShapeOf<AR>;
    const int bx = (a.size[0] + BX - 1) / BX, by = (a.size[1] + SH::by - 1) / SH::by, bz = (a.size[2] + BZ - 1) / BZ;
    const uint64_t bricks = (uint64_t)bx * by * bz;
    // split the projection run across CTAs when the volume has too few bricks to fill the GPU
    const uint64_t target = (uint64_t)dev.sm_count * 3 * (1024 / SH::nt);
    uint32_t splits = 1;
    if (bricks < target && a.n_entries > (uint32_t)G) {
        splits = (uint32_t)std::min<uint64_t>((target + bricks - 1) / bricks, (a.n_entries + G - 1) / G);
        splits = std::max<uint32_t>(splits, 1);
    }
    // runs of whole metadata groups (equal runs that end in a part-filled group measured
    // slower: c1 forward 0.131 -> 0.136 ms, one more group per brick)
    a.per_split = (((a.n_entries + splits - 1) / splits) + G - 1) / G * G;
    splits = (a.n_entries + a.per_split - 1) / std::max<uint32_t>(a.per_split, 1);
    if (splits == 0) splits = 1;
    if (a.n_entries > 0 && bricks > 0) {
        dim3 grid((unsigned)bricks, splits);
        if (a.list_mvp != nullptr) k_forward_tiled<AR, true, SH><<<grid, SH::nt, SH::smem, s>>>(vol, sum, pd, a, bx, bz);
        else k_forward_tiled<AR, false, SH><<<grid, SH::nt, SH::smem, s>>>(vol, sum, pd, a, bx, bz);
        return cudaGetLastError();
    }
    return cudaSuccess;
}

cudaError_t launch_forward(const float *vol, uint32_t *sum, const xpr_projdata *pd, const LaunchArgs &a0, int arith,
                           int compat_pad, const DeviceInfo &dev, cudaStream_t s)
{
    cudaError_t e = prepare_device_kernels();
    if (e != cudaSuccess) return e;
    const LaunchArgs &a = a0;
    e = arith == kFast ? forward_tiled<kFast>(vol, sum, pd, a0, dev, s) : forward_tiled<kStrict>(vol, sum, pd, a0, dev, s);
    if (e != cudaSuccess) return e;
    if (compat_pad && a.n_entries > 0) {
        const uint64_t n = (uint64_t)a.size[0] * a.size[1] * a.size[2];
        const uint64_t end = n + (32u - n % 32u);
        const unsigned blocks = (unsigned)((end - n + 63) / 64);
        const bool list = a.list_mvp != nullptr;
#define XPR_PAD_FWD(AR, LI) k_pad_items<AR, LI, true, false, kF32><<<blocks, 64, 0, s>>>(const_cast<float *>(vol), sum, nullptr, pd, a, n, end)
        if (arith == kFast) { if (list) XPR_PAD_FWD(kFast, true); else XPR_PAD_FWD(kFast, false); }
        else { if (list) XPR_PAD_FWD(kStrict, true); else XPR_PAD_FWD(kStrict, false); }
#undef XPR_PAD_FWD
        e = cudaGetLastError();
    }
    return e;
}

template <int AR, bool LI, bool NS>
static void dispatch_bwd_dt(int dt, dim3 grid, cudaStream_t s, float *vol, const void *ratio, const xpr_projdata *pd,
                            const LaunchArgs &a, int bx, int bz)
{
    if (dt == kBF16) k_backward_tiled<AR, LI, NS, kBF16, BWD_BY><<<grid, NT, 0, s>>>(vol, ratio, pd, a, bx, bz);
    else if (dt == kF16) k_backward_tiled<AR, LI, NS, kF16, BWD_BY><<<grid, NT, 0, s>>>(vol, ratio, pd, a, bx, bz);
    else k_backward_tiled<AR, LI, NS, kF32, BWD_BY><<<grid, NT, 0, s>>>(vol, ratio, pd, a, bx, bz);
}

template <int AR, bool LI, bool NS>
static void dispatch_pad_bwd_dt(int dt, unsigned blocks, cudaStream_t s, float *vol, const void *ratio,
                                const xpr_projdata *pd, const LaunchArgs &a, uint64_t b, uint64_t e)
{
    if (dt == kBF16) k_pad_items<AR, LI, false, NS, kBF16><<<blocks, 64, 0, s>>>(vol, nullptr, ratio, pd, a, b, e);
    else if (dt == kF16) k_pad_items<AR, LI, false, NS, kF16><<<blocks, 64, 0, s>>>(vol, nullptr, ratio, pd, a, b, e);
    else k_pad_items<AR, LI, false, NS, kF32><<<blocks, 64, 0, s>>>(vol, nullptr, ratio, pd, a, b, e);
}

cudaError_t launch_backward(float *vol, const void *ratio, int dt, const xpr_projdata *pd, const LaunchArgs &a,
                            int arith, int compat_pad, int nan_skip, const DeviceInfo &dev, cudaStream_t s)
{
    (void)dev;
    const int bx = (a.size[0] + BX - 1) / BX, by = (a.size[1] + BWD_BY - 1) / BWD_BY,
              bz = (a.size[2] + BWD_BZ - 1) / BWD_BZ;
    const uint64_t bricks = (uint64_t)bx * by * bz;
    const bool list = a.list_mvp != nullptr;
    dim3 grid((unsigned)bricks);
    if (bricks > 0) {
#define XPR_BWD(AR, LI, NS) dispatch_bwd_dt<AR, LI, NS>(dt, grid, s, vol, ratio, pd, a, bx, bz)
        if (arith == kFast) {
            if (list) { if (nan_skip) XPR_BWD(kFast, true, true); else XPR_BWD(kFast, true, false); }
            else { if (nan_skip) XPR_BWD(kFast, false, true); else XPR_BWD(kFast, false, false); }
        } else {
            if (list) { if (nan_skip) XPR_BWD(kStrict, true, true); else XPR_BWD(kStrict, true, false); }
            else { if (nan_skip) XPR_BWD(kStrict, false, true); else XPR_BWD(kStrict, false, false); }
        }
#undef XPR_BWD
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (compat_pad) {
        const uint64_t n = (uint64_t)a.size[0] * a.size[1] * a.size[2];
        const uint64_t end = n + (32u - n % 32u);
        const unsigned blocks = (unsigned)((end - n + 63) / 64);
#define XPR_PADB(AR, LI, NS) dispatch_pad_bwd_dt<AR, LI, NS>(dt, blocks, s, vol, ratio, pd, a, n, end)
        if (arith == kFast) {
            if (list) { if (nan_skip) XPR_PADB(kFast, true, true); else XPR_PADB(kFast, true, false); }
            else { if (nan_skip) XPR_PADB(kFast, false, true); else XPR_PADB(kFast, false, false); }
        } else {
            if (list) { if (nan_skip) XPR_PADB(kStrict, true, true); else XPR_PADB(kStrict, true, false); }
            else { if (nan_skip) XPR_PADB(kStrict, false, true); else XPR_PADB(kStrict, false, false); }
        }
#undef XPR_PADB
        return cudaGetLastError();
    }
    return cudaSuccess;
}

template <int MODE, int IDT, int RDT>
static void dispatch_error3(unsigned grid, cudaStream_t s, const void *img, uint32_t *sum, void *ratio, uint64_t n,
                            float w, bool zero, double *res)
{
    if (zero) {
        if (res) k_error<MODE, IDT, RDT, true, true><<<grid, 256, 0, s>>>(img, sum, ratio, n, w, res);
        else k_error<MODE, IDT, RDT, true, false><<<grid, 256, 0, s>>>(img, sum, ratio, n, w, res);
    } else {
        if (res) k_error<MODE, IDT, RDT, false, true><<<grid, 256, 0, s>>>(img, sum, ratio, n, w, res);
        else k_error<MODE, IDT, RDT, false, false><<<grid, 256, 0, s>>>(img, sum, ratio, n, w, res);
    }
}

template <int MODE, int IDT>
static void dispatch_error2(int rdt, unsigned grid, cudaStream_t s, const void *img, uint32_t *sum, void *ratio,
                            uint64_t n, float w, bool zero, double *res)
{
    if (rdt == kBF16) dispatch_error3<MODE, IDT, kBF16>(grid, s, img, sum, ratio, n, w, zero, res);
    else if (rdt == kF16) dispatch_error3<MODE, IDT, kF16>(grid, s, img, sum, ratio, n, w, zero, res);
    else dispatch_error3<MODE, IDT, kF32>(grid, s, img, sum, ratio, n, w, zero, res);
}

template <int MODE>
static void dispatch_error1(int idt, int rdt, unsigned grid, cudaStream_t s, const void *img, uint32_t *sum,
                            void *ratio, uint64_t n, float w, bool zero, double *res)
{
    if (idt == kBF16) dispatch_error2<MODE, kBF16>(rdt, grid, s, img, sum, ratio, n, w, zero, res);
    else if (idt == kF16) dispatch_error2<MODE, kF16>(rdt, grid, s, img, sum, ratio, n, w, zero, res);
    else dispatch_error2<MODE, kF32>(rdt, grid, s, img, sum, ratio, n, w, zero, res);
}

cudaError_t launch_error(const void *images, int idt, uint32_t *sum, void *ratio, int rdt, uint64_t n, float weight,
                         int mode, int zero_sum, double *residual, const DeviceInfo &dev, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const unsigned grid = stream_grid(n, dev);
    const bool zero = zero_sum && ((void *)sum != ratio);
    if (mode == XPR_ERROR_FIRST_1C) dispatch_error1<XPR_ERROR_FIRST_1C>(idt, rdt, grid, s, images, sum, ratio, n, weight, zero, residual);
    else if (mode == XPR_ERROR_1C) dispatch_error1<XPR_ERROR_1C>(idt, rdt, grid, s, images, sum, ratio, n, weight, zero, residual);
    else dispatch_error1<XPR_ERROR_STD>(idt, rdt, grid, s, images, sum, ratio, n, weight, zero, residual);
    return cudaGetLastError();
}

cudaError_t launch_minmax(const float *images, uint64_t n, float *minmax, const DeviceInfo &dev, cudaStream_t s)
{
    k_minmax_encode<<<1, 32, 0, s>>>(minmax, false);
    if (n) k_minmax<<<stream_grid(n, dev), 256, 0, s>>>(images, n, minmax);
    k_minmax_encode<<<1, 32, 0, s>>>(minmax, true);
    return cudaGetLastError();
}

cudaError_t launch_preprocess(const float *images, void *out, int odt, uint64_t n, int normalize, const float *minmax,
                              int mlog, const DeviceInfo &dev, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const unsigned grid = stream_grid(n, dev);
    if (odt == kBF16) k_preprocess<kBF16><<<grid, 256, 0, s>>>(images, out, n, normalize, minmax, mlog);
    else if (odt == kF16) k_preprocess<kF16><<<grid, 256, 0, s>>>(images, out, n, normalize, minmax, mlog);
    else k_preprocess<kF32><<<grid, 256, 0, s>>>(images, out, n, normalize, minmax, mlog);
    return cudaGetLastError();
}

cudaError_t launch_preprocess_reorder(const float *images, void *out, int odt, uint64_t wh, uint32_t n_img, uint32_t S,
                                      uint32_t Pc, int normalize, const float *minmax, int mlog, const DeviceInfo &dev,
                                      cudaStream_t s)
{
    if (wh == 0 || n_img == 0) return cudaSuccess;
    if (S == 0 || Pc == 0 || n_img > S * Pc) return cudaErrorInvalidValue;
    const unsigned grid = stream_grid(wh * n_img, dev);
    if (odt == kBF16) k_preprocess_reorder<kBF16><<<grid, 256, 0, s>>>(images, out, wh, n_img, S, Pc, normalize, minmax, mlog);
    else if (odt == kF16) k_preprocess_reorder<kF16><<<grid, 256, 0, s>>>(images, out, wh, n_img, S, Pc, normalize, minmax, mlog);
    else k_preprocess_reorder<kF32><<<grid, 256, 0, s>>>(images, out, wh, n_img, S, Pc, normalize, minmax, mlog);
    return cudaGetLastError();
}

cudaError_t launch_fill_u32(void *dst, uint32_t value, uint64_t count, const DeviceInfo &dev, cudaStream_t s)
{
    if (count == 0) return cudaSuccess;
    if (value == 0u) return cudaMemsetAsync(dst, 0, count * 4, s);
    k_fill_u32<<<stream_grid(count, dev), 256, 0, s>>>((uint32_t *)dst, value, count);
    return cudaGetLastError();
}

cudaError_t launch_convert(const float *src, void *dst, int dtype, uint64_t n, const DeviceInfo &dev, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const unsigned grid = stream_grid(n, dev);
    if (dtype == kBF16) k_convert<kBF16><<<grid, 256, 0, s>>>(src, dst, n);
    else if (dtype == kF16) k_convert<kF16><<<grid, 256, 0, s>>>(src, dst, n);
    else return cudaMemcpyAsync(dst, src, n * 4, cudaMemcpyDeviceToDevice, s);
    return cudaGetLastError();
}

// ---- batched launchers ---------------------------------------------------------------
int forward_brick(int axis, int layers) { return axis == 0 ? BX : (axis == 1 ? layers : BZ); }
bool forward_layers_ok(int arith, int layers) { return layers == BY || (layers == FwdTall::by && arith == kStrict); }
int backward_brick(int axis, int cb) { return axis == 0 ? BX : (axis == 1 ? cb : BWD_BZ); }

template <int AR, int DT>
static void *bwd_batched_fn(int cb)
{
    return cb == 8 ? (void *)k_backward_batched<AR, DT, 8> : (void *)k_backward_batched<AR, DT, 16>;
}

// kind 0: the forward, cb its brick layers (8, or 16 in the STRICT contract); kind 1: the
// backward, cb its column length
static void *batched_fn(int kind, int arith, int dtype, int cb)
{
    if (kind == 0) {
        if (arith == kFast) return (void *)k_forward_batched<kFast>;
        return cb == FwdTall::by ? (void *)k_forward_batched<kStrict, FwdTall> : (void *)k_forward_batched<kStrict>;
    }
    if (arith == kFast) {
        if (dtype == kBF16) return bwd_batched_fn<kFast, kBF16>(cb);
        if (dtype == kF16) return bwd_batched_fn<kFast, kF16>(cb);
        return bwd_batched_fn<kFast, kF32>(cb);
    }
    if (dtype == kBF16) return bwd_batched_fn<kStrict, kBF16>(cb);
    if (dtype == kF16) return bwd_batched_fn<kStrict, kF16>(cb);
    return bwd_batched_fn<kStrict, kF32>(cb);
}

int batched_ctas_per_sm(int kind, int arith, int dtype, int cb)
{
    if (prepare_device_kernels() != cudaSuccess) return 0;
    int n = 0;
    const bool tall = kind == 0 && arith == kStrict && cb == FwdTall::by;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batched_fn(kind, arith, dtype, cb), tall ? FwdTall::nt : NT,
                                                      kind == 0 ? (tall ? FwdTall::smem : kFwdSmem) : 0) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

cudaError_t launch_forward_batched(const BatchFwdItem *items, int n_items, uint32_t total_units, uint32_t *ticket,
                                   int arith, int layers, unsigned ctas, cudaStream_t s)
{
    cudaError_t e = prepare_device_kernels();
    if (e != cudaSuccess) return e;
    if (!forward_layers_ok(arith, layers)) return cudaErrorInvalidValue;
    if (n_items <= 0 || total_units == 0) return cudaSuccess;
    ctas = std::max(1u, std::min(ctas, total_units));
    if (arith == kFast) k_forward_batched<kFast><<<ctas, NT, kFwdSmem, s>>>(items, n_items, total_units, ticket);
    else if (layers == FwdTall::by)
        k_forward_batched<kStrict, FwdTall><<<ctas, FwdTall::nt, FwdTall::smem, s>>>(items, n_items, total_units,
                                                                                     ticket);
    else k_forward_batched<kStrict><<<ctas, NT, kFwdSmem, s>>>(items, n_items, total_units, ticket);
    return cudaGetLastError();
}

template <int AR, int DT>
static void bwd_batched(int cb, unsigned ctas, cudaStream_t s, const BatchBwdItem *items, int n, uint32_t total,
                        uint32_t *ticket)
{
    if (cb == 8) k_backward_batched<AR, DT, 8><<<ctas, NT, 0, s>>>(items, n, total, ticket);
    else k_backward_batched<AR, DT, 16><<<ctas, NT, 0, s>>>(items, n, total, ticket);
}

cudaError_t launch_backward_batched(const BatchBwdItem *items, int n_items, uint32_t total_units, uint32_t *ticket,
                                    int arith, int dt, int cb, unsigned ctas, cudaStream_t s)
{
    if (n_items <= 0 || total_units == 0) return cudaSuccess;
    ctas = std::max(1u, std::min(ctas, total_units));
    if (arith == kFast) {
        if (dt == kBF16) bwd_batched<kFast, kBF16>(cb, ctas, s, items, n_items, total_units, ticket);
        else if (dt == kF16) bwd_batched<kFast, kF16>(cb, ctas, s, items, n_items, total_units, ticket);
        else bwd_batched<kFast, kF32>(cb, ctas, s, items, n_items, total_units, ticket);
    } else {
        if (dt == kBF16) bwd_batched<kStrict, kBF16>(cb, ctas, s, items, n_items, total_units, ticket);
        else if (dt == kF16) bwd_batched<kStrict, kF16>(cb, ctas, s, items, n_items, total_units, ticket);
        else bwd_batched<kStrict, kF32>(cb, ctas, s, items, n_items, total_units, ticket);
    }
    return cudaGetLastError();
}

template <int IDT>
static void err_batched(int rdt, dim3 grid, cudaStream_t s, const BatchErrItem *items)
{
    if (rdt == kBF16) k_error_batched<IDT, kBF16><<<grid, 256, 0, s>>>(items);
    else if (rdt == kF16) k_error_batched<IDT, kF16><<<grid, 256, 0, s>>>(items);
    else k_error_batched<IDT, kF32><<<grid, 256, 0, s>>>(items);
}

static dim3 batched_stream_grid(int n_items, uint64_t max_n, const DeviceInfo &dev)
{
    const uint64_t want = (max_n + 255) / 256;
    const uint64_t cap = std::max<uint64_t>(1, (uint64_t)dev.sm_count * 8 / (uint64_t)std::max(1, n_items));
    return dim3((unsigned)std::max<uint64_t>(1, std::min(want, std::max<uint64_t>(cap, 4))), (unsigned)n_items);
}

cudaError_t launch_error_batched(const BatchErrItem *items, int n_items, int idt, int rdt, uint64_t max_n,
                                 const DeviceInfo &dev, cudaStream_t s)
{
    if (n_items <= 0 || max_n == 0) return cudaSuccess;
    if (n_items > 65535) return cudaErrorInvalidValue;
    const dim3 grid = batched_stream_grid(n_items, max_n, dev);
    if (idt == kBF16) err_batched<kBF16>(rdt, grid, s, items);
    else if (idt == kF16) err_batched<kF16>(rdt, grid, s, items);
    else err_batched<kF32>(rdt, grid, s, items);
    return cudaGetLastError();
}

cudaError_t launch_fill_batched(const BatchFillItem *items, int n_items, uint64_t max_n, const DeviceInfo &dev,
                                cudaStream_t s)
{
    if (n_items <= 0 || max_n == 0) return cudaSuccess;
    if (n_items > 65535) return cudaErrorInvalidValue;
    k_fill_batched<<<batched_stream_grid(n_items, max_n, dev), 256, 0, s>>>(items);
    return cudaGetLastError();
}

}  // namespace xpr
