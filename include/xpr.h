/*
 * xpr.h -- C ABI of the B200 backend for the XPRecon iterative cone-beam path.
 *
 * The reference (ebarjou/xpulse_recon) has no library boundary: its operator
 * seam is the protected API of class Reconstruction (src/reconstruction.hpp:
 * 166-312) driving five OpenCL kernels through gpu::Context / gpu::Kernel
 * (src/reconstruction/gpu/context.hpp, kernel.hpp).  This header is the plain-C
 * replacement for that seam: plain pointers and sizes, status codes instead of
 * exceptions, explicit streams instead of the three in-order OpenCL queues.
 *
 * Conventions
 *   - Every function returns XPR_OK (0) or a positive XPR_ERR_* code; the
 *     message of the last failure on the calling thread is xpr_last_error().
 *   - "device" pointers are CUDA device memory of the context's GPU; "host"
 *     pointers are ordinary or pinned host memory.
 *   - `stream` is a cudaStream_t passed as void* (NULL = the legacy default stream).
 *     Operator calls are asynchronous with respect to the host.
 *   - Volumes are laid out (y, z, x) with x fastest: index = (y*Z + z)*X + x,
 *     the layout of utils.cl:39-45 (to3D).  Detector images are (image, row,
 *     column): index = img*(W*rows) + v*W + u (utils.cl:47).
 *   - Forward sums are 22-bit-fraction unsigned fixed point (constants.cl:17-23),
 *     accumulated modulo 2^32.
 */
#ifndef XPR_H
#define XPR_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XPR_ABI_VERSION 1

enum xpr_status {
    XPR_OK = 0,
    XPR_ERR_INVALID = 1,     /* bad argument */
    XPR_ERR_CUDA = 2,        /* CUDA runtime error */
    XPR_ERR_OOM = 3,         /* device or pinned allocation failed */
    XPR_ERR_CAP = 4,         /* request exceeds the context's device-memory cap, or the capacity of a
                                fixed-size scratch (xpr_subiteration_static) */
    XPR_ERR_IO = 5,          /* file read / write failure */
    XPR_ERR_PARAM = 6,       /* malformed or inconsistent parameters (JSON, geometry) */
    XPR_ERR_UNSUPPORTED = 7  /* valid request this build does not implement */
};

enum xpr_arith { XPR_ARITH_STRICT = 0, XPR_ARITH_FAST = 1 };
enum xpr_dtype { XPR_F32 = 0, XPR_BF16 = 1, XPR_F16 = 2 };
enum xpr_error_mode {
    XPR_ERROR_STD = 0,       /* KernelError.cl:8-24: log(max(ref/max(got,eps),eps))*w */
    XPR_ERROR_FIRST_1C = 1,  /* reconstruction_lplh.hpp:164-177: log(max(ref,eps)) */
    XPR_ERROR_1C = 2         /* reconstruction_lplh.hpp:140-163 (std::max semantics) */
};

/* ProjData (constants.cl:25-28): the 4 columns of the glm projection matrix,
 * then the viewport {l, r, b, t}.  80 bytes, the reference's layout.
 * Viewport bounds must be integers in [0, 2^22]. */
typedef struct xpr_projdata {
    float mvp[16];
    float vp[4];
} xpr_projdata;

/* One projector launch: the scalar arguments of Forward/Backward
 * (constants.cl:30-54, set by reconstruction.hpp:208-281) and the index lists
 * of ForwardH/BackwardH (constants.cl:62-88). */
typedef struct xpr_launch {
    int32_t vmin[3];          /* voxel box [vmin, vmax) in (x, y, z) (setVolumeParameters) */
    int32_t vmax[3];
    float origin[3];          /* volume origin in mm incl. jitter (setOrigin) */
    float voxel[3];           /* voxel size in mm */
    uint32_t det_w;           /* detector width (setImageParameters: size.x) */
    uint32_t rows;            /* rows held per image in the buffer (setImageOffset: y) */
    int32_t row_offset;       /* first detector row held (setImageOffset: x) */
    uint32_t n_angles;        /* angles in the subset (setAngleNumber) */
    uint32_t modules;         /* modules per angle */
    const uint16_t *list_mvp; /* optional device list: ProjData index per entry (ForwardH) */
    const uint16_t *list_img; /* optional device list: image slot per entry */
    uint32_t n_list;
    int32_t arith;            /* xpr_arith */
    int32_t compat_pad;       /* also run the reference NDRange padding work-items (kernel.hpp:73-81);
                                 the volume buffer must then hold xpr_ndrange(n) floats */
    int32_t nan_skip;         /* BackwardH: NaN ratios are skipped (KernelBackwardH.cl:36) */
} xpr_launch;

typedef struct xpr_ctx xpr_ctx;

/* ---------------------------------------------------------------- context */
/* Replaces gpu::Context() (context.hpp:36-113).  mem_cap_bytes = 0: no cap
 * beyond what cudaMemGetInfo reports (the reference's VRAM-filling probe,
 * context.hpp:90-104, is not reproduced). */
int xpr_create(int device, uint64_t mem_cap_bytes, xpr_ctx **out);
int xpr_destroy(xpr_ctx *ctx);
const char *xpr_last_error(void);
int xpr_abi_version(void);
/* usable device bytes: min(free memory, cap - bytes allocated through the context) */
int xpr_mem_available(xpr_ctx *ctx, uint64_t *bytes);
/* work-items of the reference NDRange for n items: n + (32 - n % 32) (kernel.hpp:73-81) */
uint64_t xpr_ndrange(uint64_t n);

/* ---------------------------------------------------------------- memory */
/* Replace Context::createBuffer / setBuffer / getBuffer (context.hpp:152-300). */
int xpr_alloc(xpr_ctx *ctx, uint64_t bytes, void **dptr);
int xpr_free(xpr_ctx *ctx, void *dptr);
/* Page-locked host memory for staging.  From 32 MB up the buffer is mapped with huge pages
 * requested, faulted in by several threads and registered with the driver (about 10x faster
 * to obtain than one cudaMallocHost of the same size); release it with xpr_free_pinned only. */
int xpr_alloc_pinned(xpr_ctx *ctx, uint64_t bytes, void **hptr);
int xpr_free_pinned(xpr_ctx *ctx, void *hptr);
int xpr_upload(xpr_ctx *ctx, void *dst, const void *src, uint64_t bytes, void *stream);
int xpr_download(xpr_ctx *ctx, void *dst, const void *src, uint64_t bytes, void *stream);
/* fill `count` 32-bit words (enqueueFillBuffer; 1.0f is 0x3f800000) */
int xpr_fill_u32(xpr_ctx *ctx, void *dst, uint32_t value, uint64_t count, void *stream);
int xpr_synchronize(xpr_ctx *ctx, void *stream);

/* ---------------------------------------------------------------- operators */
/* Forward projection (Reconstruction::forward, reconstruction.hpp:294-296;
 * KernelForward.cl:10-55, KernelForwardH.cl:8-37 when L->list_mvp is set):
 * sum[img][v][u] += fixed(vol[voxel]) for every in-bounds (voxel, ProjData) pair.
 * pd: n_pd device ProjData; without a list, entries 0 .. n_angles*modules-1 are
 * used and image slot = entry / modules. */
int xpr_forward(xpr_ctx *ctx, const float *vol, uint32_t *sum, const xpr_projdata *pd, uint32_t n_pd,
                const xpr_launch *L, void *stream);

/* Back projection with the multiplicative update (Reconstruction::backward,
 * reconstruction.hpp:310-312; KernelBackward.cl:8-40, KernelBackwardH.cl:8-42):
 * vol *= exp(sum of in-bounds ratios / their count).  ratio has ratio_dtype. */
int xpr_backward(xpr_ctx *ctx, float *vol, const void *ratio, int ratio_dtype, const xpr_projdata *pd,
                 uint32_t n_pd, const xpr_launch *L, void *stream);

/* Error step (Reconstruction::error, reconstruction.hpp:302-304; KernelError.cl:8-24).
 * images: n measured values of image_dtype.  sum: n fixed-point sums.  ratio:
 * output of ratio_dtype; ratio == sum with XPR_F32 writes in place as the
 * reference does.  When zero_sum != 0 (and ratio != sum) the sums are reset to 0
 * in the same pass.  residual: optional device double, += sum of ratio^2 (FP64). */
int xpr_error(xpr_ctx *ctx, const void *images, int image_dtype, uint32_t *sum, void *ratio, int ratio_dtype,
              uint64_t n, float weight, int mode, int zero_sum, double *residual, void *stream);

/* -log / normalise preprocessing (data_loader.hpp:48-101) on the device.
 * minmax: device float[2] running {min, max} of the std::isnormal values,
 * initialise to {FLT_MAX, FLT_MIN} as data_loader.hpp:12-13 does. */
int xpr_preprocess_minmax(xpr_ctx *ctx, const float *images, uint64_t n, float *minmax, void *stream);
/* v = normalize ? (isnormal(v) ? (v-min)/(max-min) : (max+min)/2) : v;
 * v = mlog ? -log(clamp(v, eps, 1-eps)) : v; written as out_dtype into out
 * (out may equal images for XPR_F32). */
int xpr_preprocess_apply(xpr_ctx *ctx, const float *images, void *out, int out_dtype, uint64_t n, int normalize,
                         const float *minmax, int mlog, void *stream);

/* One sub-iteration of reconstruction_n.hpp:65-76: [forward] -> error -> backward,
 * then the sums reset to 0.  first != 0 skips the forward (the sums must then
 * hold FIXED_ONE, as after reconstruction_n.hpp:60).  ratio may equal sum (FP32
 * in place) or be a separate buffer of ratio_dtype. */
int xpr_subiteration(xpr_ctx *ctx, float *vol, uint32_t *sum, const void *images, int image_dtype, void *ratio,
                     int ratio_dtype, const xpr_projdata *pd, uint32_t n_pd, const xpr_launch *L, float weight,
                     int first, double *residual, void *stream);

/* One sub-iteration as xpr_subiteration, for callers that cannot allocate device
 * memory while they run (a host application that owns the device budget and passes
 * only its inputs and outputs; a frame loop that must not stall on, or fail in, an
 * allocation).  No counterpart in the reference.  The detector scratch (fixed-point
 * sums, overwritten in place by the FP32 ratio) lives in a fixed device array of
 * xpr_subiteration_static_capacity() 32-bit words, held by every GPU that loads the
 * library until the process exits; larger sub-iterations (n_angles * det_w * rows
 * words) are rejected with XPR_ERR_CAP.  The call neither allocates nor frees.  It
 * starts from FIXED_ONE sums when first != 0 (forward skipped) and from zero sums
 * otherwise, so no state carries over between calls; the ratio is FP32.  The first
 * call on a device looks up the array's device address; make that first call before
 * any stream capture.  All calls share the one array: calls that overlap on the GPU
 * (other streams, other threads) race on it. */
int xpr_subiteration_static(xpr_ctx *ctx, float *vol, const void *images, int image_dtype, const xpr_projdata *pd,
                            uint32_t n_pd, const xpr_launch *L, float weight, int first, void *stream);
uint64_t xpr_subiteration_static_capacity(void);

/* ---------------------------------------------------------------- batched reconstructions */
/* Many independent naive reconstructions (reconstruction_n.hpp:27-88 each) advanced in
 * lock-step.  A sub-iteration step of all problems is three persistent launches (forward,
 * error, backward) whose CTAs claim work units from one list spanning every problem;
 * a whole run can be captured once into a CUDA graph and replayed.  No counterpart in
 * the reference, which runs one reconstruction per process.  Each problem's volume is
 * bit-identical to the same reconstruction run alone through xpr_subiteration (same
 * seed, contract and storage), whatever the batch, schedule or tuning. */
typedef struct xpr_batch_problem {
    float *vol;                   /* device, vwidth * vheight * vwidth floats (x fastest, then z, then y) */
    const void *images;           /* device, sit * per_subset preprocessed images of det_w * det_h in the batch's
                                     image storage type, subset-major: subset s holds acquisitions s, s + sit, ... */
    const xpr_projdata *projdata; /* device, sit * per_subset * modules entries in the same order */
    uint32_t det_w, det_h;
    uint32_t per_subset;          /* projections per sub-iteration: floor(projections / sit) */
    uint32_t modules;
    uint32_t sit, it;
    uint32_t vwidth, vheight;     /* the reconstruction grid (geometry.hpp:55-60) */
    float voxel;                  /* vx */
    float orig[3];                /* grid origin before the jitter */
    uint32_t seed;                /* std::mt19937 seed of the origin jitter (3 draws per sub-iteration) */
    float weight, weight_factor;
    double *residual;             /* optional device array of it * sit doubles: sum of ratio^2 per sub-iteration */
} xpr_batch_problem;

typedef struct xpr_batch_opts {
    int32_t arith;                /* xpr_arith */
    int32_t storage;              /* xpr_dtype of the ratio scratch, and of the images unless
                                     image_storage_set */
    int32_t init_volume;          /* each run first sets every volume to 1.0 (reconstruction_n.hpp:59) */
    int32_t use_graph;            /* capture the whole run into one CUDA graph at the first run, replay after */
    int32_t autotune;             /* time the schedule candidates once (per batch shape, cached) */
    int32_t fwd_splits;           /* 0: automatic or tuned; else projection runs per forward brick */
    int32_t bwd_column;           /* 0: automatic or tuned; else 8 or 16 layers per backward voxel column */
    int32_t ctas_per_sm;          /* 0: the occupancy limit */
    int32_t image_storage_set;    /* 0: the measured images are stored in `storage` too */
    int32_t image_storage;        /* else their xpr_dtype, e.g. FP16 images with a BF16 ratio */
    int32_t fwd_layers;           /* 0: automatic or tuned; else the forward brick's layers: 8, or 16
                                     in the STRICT contract */
} xpr_batch_opts;

typedef struct xpr_batch xpr_batch;
/* Validates the problems, allocates their scratch (fixed-point sums and ratios) through
 * ctx and uploads every step's work lists.  With opts->autotune it runs the candidate
 * schedules on the problems' data (volumes are left as they were). */
int xpr_batch_create(xpr_ctx *ctx, const xpr_batch_problem *problems, uint32_t n, const xpr_batch_opts *opts,
                     void *stream, xpr_batch **out);
/* All it * sit sub-iterations of every problem (the longest problem sets the step count). */
int xpr_batch_run(xpr_batch *b, void *stream);
/* One step: sub-iteration `step` of every problem that has one (step < xpr_batch_steps). */
int xpr_batch_step(xpr_batch *b, uint32_t step, void *stream);
uint32_t xpr_batch_steps(const xpr_batch *b);
/* The schedule in use: projection runs per forward brick, the forward brick's layers,
 * backward column length, persistent forward CTAs per SM, and the tuned step time in ms
 * (0 when not tuned). */
int xpr_batch_schedule(const xpr_batch *b, int32_t *fwd_splits, int32_t *fwd_layers, int32_t *bwd_column,
                       int32_t *ctas_per_sm, double *tuned_ms);
int xpr_batch_destroy(xpr_batch *b);

/* ---------------------------------------------------------------- serving */
/* A request loop with continuous batching.  Each request is a naive reconstruction
 * (reconstruction_n.hpp:27-88) of raw projections held by the caller, with its
 * parameters in the XPRecon JSON schema (recon / geometry / detector; the detector size
 * and projection count come from the images).  A request is admitted when the device
 * memory it needs fits the server's budget (first come, first served); it then joins
 * the running batch at the next sub-iteration boundary and every active request advances
 * one sub-iteration per tick (one persistent forward, error and backward launch over all
 * of them).  Its volume, images and scratch stay resident until its last sub-iteration;
 * the volume is then copied to the caller's buffer and the memory freed.  Uploads and
 * downloads run on their own streams beside the compute.  A request's result is
 * bit-identical whatever else is being served (see xpr_batch).  No counterpart in the
 * reference.  recon.seed should be set: without it the jitter seed is random, as in the
 * reference. */
typedef struct xpr_serve_opts {
    int32_t arith;                /* xpr_arith for every request */
    int32_t storage;              /* xpr_dtype of the ratios of every request, and of its images unless
                                     image_storage_set */
    uint64_t mem_budget;          /* device bytes for resident requests; 0: 90% of the free memory */
    uint32_t max_active;          /* requests resident at once; 0: no limit */
    int32_t image_storage_set;    /* 0: images stored in `storage` */
    int32_t image_storage;        /* else the xpr_dtype of the preprocessed images */
} xpr_serve_opts;

enum xpr_request_state { XPR_REQ_QUEUED = 0, XPR_REQ_ACTIVE = 1, XPR_REQ_DONE = 2, XPR_REQ_FAILED = 3 };

typedef struct xpr_request_info {
    int32_t state;                /* xpr_request_state */
    int32_t error;                /* XPR_ERR_* of a failed request */
    double submit_s, admit_s, done_s;  /* seconds since the server started */
    uint64_t pairs;               /* voxel x projection pairs of the whole reconstruction */
    uint64_t device_bytes;        /* peak device memory held (the admission charge: the resident
                                     reconstruction plus its raw images until it joins the batch) */
} xpr_request_info;

typedef struct xpr_serve_stats {
    uint64_t submitted, completed, failed;
    uint64_t ticks;               /* batched sub-iteration steps launched */
    uint64_t pairs;               /* voxel x projection pairs processed */
    uint32_t active, queued;
    uint64_t bytes_in_use, peak_bytes;
} xpr_serve_stats;

typedef struct xpr_server xpr_server;
int xpr_serve_create(xpr_ctx *ctx, const xpr_serve_opts *opts, xpr_server **out);
/* raw: count images of height x width float32 intensities in acquisition order, read by
 * the server until the request completes; vol_out: host memory for vwidth * vheight *
 * vwidth floats, written before the request is reported done.  Malformed parameters or a
 * request larger than the whole budget fail here (XPR_ERR_PARAM / XPR_ERR_CAP). */
int xpr_serve_submit(xpr_server *s, const char *json, const float *raw, int64_t count, uint32_t width,
                     uint32_t height, float *vol_out, uint64_t vol_cap, uint64_t *ticket);
int xpr_serve_poll(xpr_server *s, uint64_t ticket, xpr_request_info *info);
/* Blocks until the request is done or failed, or timeout_s (< 0: no limit) passes;
 * returns XPR_OK with info->state set either way. */
int xpr_serve_wait(xpr_server *s, uint64_t ticket, double timeout_s, xpr_request_info *info);
int xpr_serve_stats_get(xpr_server *s, xpr_serve_stats *stats);
/* Waits for every submitted request, then stops the server and frees its resources. */
int xpr_serve_destroy(xpr_server *s);

/* ---------------------------------------------------------------- geometry (host) */
/* Geometry parameters (global_parameters.hpp:23-54, parameters.hpp:34-48). */
typedef struct xpr_geom_params {
    float so, sd, angle, heli_offset;
    float px, rx_px, sx, sy;            /* rx in pixels as in the JSON; sx, sy act in mm (geometry.hpp:61) */
    int64_t module_number;
    int32_t module_angle_offset_set;
    float module_angle_offset;
    float module_center_offset_z;
    int64_t dwidth, dheight, projections, sit;
    const float *angle_list;            /* optional, `projections` angles in degrees */
    const float *mod_offset;            /* optional extension: 3 per module, pixels */
    const float *mod_rpy;               /* optional extension: roll, pitch, yaw per module, degrees */
} xpr_geom_params;

typedef struct xpr_geom_out {
    float vx;
    int64_t vwidth, vheight;
    float orig[3];
    int64_t concurrent;                 /* floor(projections / sit) */
} xpr_geom_out;

/* Geometry() + computeMVPs() (geometry.hpp:35-76, 182-328): ProjData for every
 * (angle, module) in angle-major order (index angle*modules + module).
 * fp64 != 0 builds the matrices in double precision. */
int xpr_geometry(const xpr_geom_params *gp, int fp64, xpr_projdata *out, xpr_geom_out *go);

/* The origin jitter sequence: n draws of std::uniform_real_distribution<float>(0, vx)
 * from std::mt19937(seed) (reconstruction.hpp:268-272), 3 per sub-iteration. */
int xpr_jitter(uint32_t seed, uint64_t n, float vx, float *out);

/* method_2 chunk planner (GeometryChunk, geometry_chunk.hpp:92-197).  all: ProjData of
 * every (angle, module).  chunks: 6 int64 per chunk {vOffset, vSize, iOffset, iSize,
 * vPadTop, vPadBot}.  *n_chunks = -1 when one layer does not fit. */
int xpr_plan_chunks(const xpr_geom_params *gp, const xpr_geom_out *go, const xpr_projdata *all, uint64_t avail_bytes,
                    uint64_t max_alloc_bytes, float overlap_fct, int64_t *chunks, int max_chunks, int *n_chunks);
/* method_1c per-layer angle culling (Geometry::getMvpPerLayer, geometry.hpp:141-171).
 * per_module != 0 indexes ProjData by angle*modules + module (the reference indexes by
 * angle, which is right for one module only). */
int xpr_cull_layer(const xpr_geom_params *gp, const xpr_geom_out *go, const xpr_projdata *all, int64_t sit,
                   int64_t layer, int per_module, uint16_t *mvp_idx, uint16_t *img_idx, int *n);

/* ---------------------------------------------------------------- whole runs (host) */
/* The XPRecon command line (main.cpp:69-136) as a call: json_or_path is a parameter
 * file or inline JSON starting with '{'.  Runs the selected method (naive | method_1a |
 * method_1b | method_1c | method_2) on the TIFF stack of recon.input, writes
 * layer_%05d.tif to recon.output, then the simulation projections (p_%010d.tif) to
 * recon.proj_output when set.  Returns 0, -2 (bad parameters) or -3 (reconstruction
 * error), the reference's exit codes. */
int xpr_run(const char *json_or_path);
/* The default parameters as JSON (XPRecon -template).  Returns the length; writes at
 * most cap bytes (NUL-terminated) when buf is non-NULL. */
int64_t xpr_template_json(char *buf, uint64_t cap);
/* The parameters a run would use (defaults, aliases, initializeParameters applied), as JSON. */
int xpr_params_normalize(const char *json_or_path, char *buf, uint64_t cap, int64_t *len);
/* A whole reconstruction of in-memory projections (count images of height x width floats,
 * acquisition order) with the parameters of `json` (recon.input / output unused, no files
 * written).  vol_out receives vwidth * vheight * vwidth floats; layers a method does not
 * reconstruct (method_2 outside its chunks) are NaN.  *seconds: time of the iterations. */
int xpr_reconstruct_host(const char *json, const float *images, int64_t count, uint32_t width, uint32_t height,
                         float *vol_out, uint64_t vol_cap, double *seconds);
/* Single-channel float32 TIFF I/O (the reference uses TinyTIFF, data_loader.hpp:209-237). */
int xpr_tiff_write(const char *path, const float *data, uint32_t width, uint32_t height);
int xpr_tiff_read(const char *path, float *data, uint64_t cap, uint32_t *width, uint32_t *height);

#ifdef __cplusplus
}
#endif
#endif
