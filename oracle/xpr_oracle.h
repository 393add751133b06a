/*
 * xpr_oracle.h -- CPU oracle for the XPRecon iterative cone-beam hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links this library: it is
 * loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
 * leg, and only to compare the product's results with.  It restates, in plain C, the algorithm of
 * ebarjou/xpulse_recon ("XPRecon") for this path:
 *
 *   - geometry -> ProjData          src/reconstruction/dataset/geometry.hpp:35-76,182-328
 *   - Forward / ForwardH kernels    src/reconstruction/gpu/kernels/KernelForward.cl:10-55,
 *                                   KernelForwardH.cl:8-37 (+ utils.cl:26,39-47, constants.cl:17-28)
 *   - Error kernel                  KernelError.cl:8-24
 *   - Backward / BackwardH kernels  KernelBackward.cl:8-40, KernelBackwardH.cl:8-42
 *   - -log / normalise              src/reconstruction/dataset/data_loader.hpp:48-101
 *   - naive subset loop             src/reconstruction/reconstruction_n.hpp:27-88
 *   - method_1c loop                src/reconstruction/reconstruction_lplh.hpp:40-233
 *   - method_2 planner + loop       dataset/geometry_chunk.hpp:92-197, reconstruction_chunk.hpp:36-131
 *   - origin jitter                 src/reconstruction.hpp:268-272 (std::mt19937 +
 *                                   std::uniform_real_distribution<float>, restated)
 *
 * Parity pin: the kernel restatements (arith = XPR_ARITH_STRICT) are checked
 * bit-for-bit against the reference's own OpenCL kernel sources compiled for
 * the CPU (oracle/_ref, built by oracle/build.py).  The geometry depends on
 * glm, an un-vendored submodule with no pinned commit: it is restated from
 * glm's published semantics and its parity is unpinned at that boundary.
 *
 * Arithmetic contracts (both are exactly reproducible on the GPU):
 *   XPR_ARITH_STRICT  the reference kernels under IEEE-754 single precision:
 *                     p = idx*vx + o (mul, add); u = dot(c0,p)/dot(c3,p) with
 *                     dot = ((x*x'+y*y')+z*z')+w*w'; v likewise minus the line
 *                     offset; round half away from zero; saturating float->int.
 *   XPR_ARITH_FAST    p = fma(idx, vx, o); C_r = fma(c_r.x, px, c_r.w) + c_r.z*pz
 *                     for the rows r = u, v, w; rw = 1/fma(c_w.y, py, C_w) (IEEE);
 *                     yu = fma(py, c_u.y*rw, fma(C_u, rw, 0.5));
 *                     yv = fma(py, c_v.y*rw, fma(C_v, rw, 0.5 - line_offset));
 *                     in-bounds iff l <= yu < r and b <= yv < min(t, rows);
 *                     pixel = (floor(yu), floor(yv)).  Along a voxel column of an
 *                     untilted detector (c_u.y = c_w.y = 0) only yv varies, by one fma.
 * exp/log are this project's own portable single-precision functions (Cody-Waite
 * reduction + Taylor polynomial; atanh series), identical on CPU and GPU.
 */
#ifndef XPR_ORACLE_H
#define XPR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_FIXED_FRAC_BITS 22
#define ORC_FIXED_ONE (1u << ORC_FIXED_FRAC_BITS)

enum { XPR_ARITH_STRICT = 0, XPR_ARITH_FAST = 1 };

/* 80-byte ProjData (constants.cl:25-28): glm columns c0..c3, then viewport {l, r, b, t}. */
typedef struct {
    float mvp[16];
    float vp[4];
} orc_projdata;

/* One forward / backward launch (the scalar kernel arguments of constants.cl:30-54,
 * plus the optional ForwardH/BackwardH index lists of constants.cl:62-88). */
typedef struct {
    int32_t vmin[3];        /* voxel box [vmin, vmax) in (x, y, z); buffer layout (y, z, x) */
    int32_t vmax[3];
    float origin[3];        /* volume origin in mm, jitter already added */
    float voxel[3];         /* voxel size in mm */
    uint32_t det_w;         /* detector width (size.x) */
    uint32_t rows;          /* image rows held per image in the buffer (lineOffsetY.y) */
    int32_t row_offset;     /* first detector row held in the buffer (lineOffsetY.x) */
    uint32_t n_angles;      /* angles in the subset (angleNumber) */
    uint32_t modules;       /* modules per angle (modulePerAngle) */
    const uint16_t *list_mvp; /* optional: ProjData index per entry (ForwardH "indexes") */
    const uint16_t *list_img; /* optional: image slot per entry (ForwardH "img_indexes") */
    uint32_t n_list;
    int32_t arith;          /* XPR_ARITH_* */
    int32_t compat_pad;     /* also run the padding work-items of the reference NDRange */
    int32_t nan_skip;       /* BackwardH: skip NaN ratios */
} orc_launch;

/* ---- portable math ---------------------------------------------------- */
float orc_expf(float x);
float orc_logf(float x);

/* ---- std::mt19937 + uniform_real_distribution<float> (libstdc++) ----- */
typedef struct { uint32_t mt[624]; int idx; } orc_mt19937;
void orc_mt_seed(orc_mt19937 *g, uint32_t seed);
uint32_t orc_mt_next(orc_mt19937 *g);
float orc_uniform_float(orc_mt19937 *g, float a, float b);

/* ---- fixed point (constants.cl:17-23) -------------------------------- */
uint32_t orc_float_to_fixed(float x);
float orc_fixed_to_float(uint32_t x);

/* ---- kernels ----------------------------------------------------------- */
/* Number of work-items the reference NDRange launches for n items (kernel.hpp:73-81). */
uint64_t orc_ndrange(uint64_t n);
void orc_forward(const float *vol, uint32_t *sum, const orc_projdata *pd, const orc_launch *L);
void orc_backward(float *vol, const float *ratio, const orc_projdata *pd, const orc_launch *L);
/* Error kernel: ratio bits are written in place over the fixed-point sums. */
void orc_error(const float *images, uint32_t *sum_ratio, uint64_t n, float weight);
/* method_1c first sub-iteration: ratio = log(max(ref, eps)), unweighted
 * (reconstruction_lplh.hpp:164-177). */
void orc_error_first_1c(const float *images, float *ratio, uint64_t n);
/* method_1c CPU error: ratio = log(max(ref / max(fixed->float(sum), eps), eps)) * w
 * (reconstruction_lplh.hpp:140-163) */
void orc_error_1c(const float *images, uint32_t *sum_ratio, uint64_t n, float weight);

/* ---- preprocessing (data_loader.hpp:48-101) ---------------------------- */
/* min / max over the "normal" values (std::isnormal) of n floats; *mn / *mx are
 * running values (initialise with FLT_MAX and FLT_MIN as the reference does). */
void orc_minmax_normal(const float *v, uint64_t n, float *mn, float *mx);
void orc_preprocess(float *v, uint64_t n, int normalize, float mn, float mx, int mlog);

/* ---- geometry (geometry.hpp) ------------------------------------------ */
typedef struct {
    float so, sd, angle, heli_offset;
    float px, rx_px, sx, sy;          /* rx in pixels as in the JSON (converted to mm here) */
    int64_t module_number;
    int32_t module_angle_offset_set;
    float module_angle_offset;
    float module_center_offset_z;
    int64_t dwidth, dheight, projections, sit;
    const float *angle_list;          /* optional, `projections` entries (degrees) */
    /* per-module extension (absent from the reference): offsets in pixels, angles in degrees */
    const float *mod_offset;          /* optional, 3 per module */
    const float *mod_rpy;             /* optional, 3 per module: roll, pitch, yaw */
} orc_geom_params;

typedef struct {
    float vx;
    int64_t vwidth, vheight;
    float orig[3];
    int64_t concurrent;               /* floor(P / sit) */
} orc_geom_out;

/* ProjData for all projections*modules, in angle-major order (index i*M + module).
 * fp64 != 0 builds the matrices in double and rounds once at the end.  Returns 0. */
int orc_geometry(const orc_geom_params *gp, int fp64, orc_projdata *out, orc_geom_out *go);

/* method_1c per-layer culling (geometry.hpp:141-171, 334-355): for sub-iteration
 * `sit` and layer `l`, writes the ProjData indexes and image slots that may touch
 * the layer; returns the count.  `per_module` != 0 indexes ProjData by i*M+module
 * (the reference uses the angle index i, valid for one module only). */
int orc_cull_layer(const orc_geom_params *gp, const orc_geom_out *go, const orc_projdata *all,
                   int64_t sit, int64_t layer, int per_module, uint16_t *mvp_idx, uint16_t *img_idx);

/* method_2 chunk planner (geometry_chunk.hpp:62-197).  chunk rows are
 * {vOffset, vSize, iOffset, iSize, vPadTop, vPadBot}.  Returns the chunk count,
 * or -1 when a single layer does not fit. */
int orc_plan_chunks(const orc_geom_params *gp, const orc_geom_out *go, const orc_projdata *all,
                    uint64_t avail_bytes, uint64_t max_alloc_bytes, float overlap_fct,
                    int64_t *chunks, int max_chunks);

/* ---- whole reconstructions --------------------------------------------- */
typedef struct {
    int64_t it, sit;
    float weight, weight_factor;
    uint32_t seed;
    int32_t arith;
    int32_t compat_pad;
} orc_recon_params;

/* naive method (reconstruction_n.hpp:27-88).  images: P preprocessed images in
 * file order (P*W*H floats).  vol: W*H*W floats (+ the padding of the reference
 * buffer when compat_pad; orc_ndrange(W*H*W) floats). */
int orc_recon_naive(const orc_geom_params *gp, const orc_recon_params *rp,
                    const float *images, float *vol);
/* method_1c (reconstruction_lplh.hpp:40-219), one GPU "thread" semantics. */
int orc_recon_1c(const orc_geom_params *gp, const orc_recon_params *rp,
                 const float *images, float *vol);
/* method_2 (reconstruction_chunk.hpp:36-131) with a given chunk plan. */
int orc_recon_chunks(const orc_geom_params *gp, const orc_recon_params *rp,
                     const float *images, const int64_t *chunks, int n_chunks, float *vol);

/* ---- FP64 oracle: the same algorithm in double, no fixed point ----------
 * The precision reference for reduced-precision storage (xpr_oracle.c). */
int orc_geometry_f64(const orc_geom_params *gp, double *mvp, double *vp, orc_geom_out *go);
void orc64_forward(const double *vol, double *sum, const double *mvp, const double *vp, int64_t n_entries,
                   int64_t modules, int64_t W, int64_t Hv, const double origin[3], double voxel, int64_t det_w,
                   int64_t rows);
void orc64_backward(double *vol, const double *ratio, const double *mvp, const double *vp, int64_t n_entries,
                    int64_t modules, int64_t W, int64_t Hv, const double origin[3], double voxel, int64_t det_w,
                    int64_t rows);
void orc64_preprocess(const float *raw, double *out, uint64_t n, int mlog);
/* naive method in double: images = P preprocessed images in file order,
 * vol = W*H*W doubles */
int orc64_recon_naive(const orc_geom_params *gp, const orc_recon_params *rp, const double *images, double *vol);

#ifdef __cplusplus
}
#endif
#endif
