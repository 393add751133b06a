// xpr_internal.h -- internal C++ interface between the C ABI, the host
// schedulers and the CUDA kernels (not installed; include/xpr.h is the boundary).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "../../include/xpr.h"

namespace xpr {

// A named NVTX range around a phase (forward, error, backward, upload, download,
// preprocessing, a sub-iteration) for a profiler's timeline; it marks the host-side
// enqueue of asynchronous work.  Without a profiler attached push / pop cost a few ns.
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};

// Validated launch description shared by the forward / backward launchers.
struct LaunchArgs {
    int32_t vmin[3];
    int32_t size[3];          // vmax - vmin
    float origin[3];
    float voxel[3];
    uint32_t det_w, rows;
    float row_off_f;          // (float)row_offset (STRICT)
    float half_minus_off;     // 0.5f - (float)row_offset (FAST)
    uint32_t n_entries;       // list length, or n_angles * modules
    uint32_t modules;
    uint32_t n_images;        // image slots in the sum / ratio buffer
    uint32_t n_pd;
    uint32_t img_stride;      // det_w * rows
    const uint16_t *list_mvp;
    const uint16_t *list_img;
    uint32_t per_split;       // entries per CTA along grid.y (forward)
};

struct DeviceInfo {
    int device = 0;
    int sm_count = 148;
};

// Fills `a` from `L`; returns an error message or nullptr.
const char *make_launch_args(const xpr_launch *L, uint32_t n_pd, LaunchArgs *a);

cudaError_t launch_forward(const float *vol, uint32_t *sum, const xpr_projdata *pd, const LaunchArgs &a, int arith,
                           int compat_pad, const DeviceInfo &dev, cudaStream_t s);
cudaError_t launch_backward(float *vol, const void *ratio, int ratio_dtype, const xpr_projdata *pd,
                            const LaunchArgs &a, int arith, int compat_pad, int nan_skip, const DeviceInfo &dev,
                            cudaStream_t s);
cudaError_t launch_error(const void *images, int image_dtype, uint32_t *sum, void *ratio, int ratio_dtype, uint64_t n,
                         float weight, int mode, int zero_sum, double *residual, const DeviceInfo &dev,
                         cudaStream_t s);
cudaError_t launch_minmax(const float *images, uint64_t n, float *minmax, const DeviceInfo &dev, cudaStream_t s);
// images [0, n_img) of wh pixels (acquisition order) preprocessed into subset-major slots
// (j mod S) * Pc + j / S of `out`
cudaError_t launch_preprocess_reorder(const float *images, void *out, int out_dtype, uint64_t wh, uint32_t n_img,
                                      uint32_t S, uint32_t Pc, int normalize, const float *minmax, int mlog,
                                      const DeviceInfo &dev, cudaStream_t s);
cudaError_t launch_preprocess(const float *images, void *out, int out_dtype, uint64_t n, int normalize,
                              const float *minmax, int mlog, const DeviceInfo &dev, cudaStream_t s);
cudaError_t launch_fill_u32(void *dst, uint32_t value, uint64_t count, const DeviceInfo &dev, cudaStream_t s);
cudaError_t launch_convert(const float *src, void *dst, int dtype, uint64_t n, const DeviceInfo &dev, cudaStream_t s);

// One-time per-device kernel attributes (dynamic shared memory opt-in).
cudaError_t prepare_device_kernels();

// For entry points defined outside xpr_capi.cu: make ctx's device current and return
// its description (nullptr and a message on failure), and record an error message
// for xpr_last_error(); returns `code`.
const DeviceInfo *context_device(xpr_ctx *ctx);
int set_last_error(int code, const char *fmt, ...);

// ---- batched launches: many independent problems in one persistent launch ----------
// Device descriptors, one per problem; work units are numbered across the problems
// (unit_begin = prefix sum of the problems' unit counts), claimed by persistent CTAs
// from a self-resetting ticket (two words, zero before the first launch).
struct BatchFwdItem {
    LaunchArgs a;
    const float *vol;
    uint32_t *sum;
    const xpr_projdata *pd;
    int32_t bricks_x, bricks_z;
    uint32_t splits;          // projection runs per brick (a.per_split entries each)
    uint32_t unit_begin;
};
struct BatchBwdItem {
    LaunchArgs a;
    float *vol;
    const void *ratio;
    const xpr_projdata *pd;
    int32_t bricks_x, bricks_z;
    uint32_t unit_begin;
    uint32_t reserved;
};
struct BatchErrItem {
    const void *images;
    uint32_t *sum;            // zeroed after it is read
    void *ratio;
    double *residual;         // optional: += sum of r^2 (FP64)
    uint64_t n;
    float weight;
    int32_t first;            // 1: the first sub-iteration, sums taken as FIXED_ONE (no forward ran)
};
struct BatchFillItem {
    uint32_t *dst;
    uint64_t n;
    uint32_t value;
    uint32_t reserved;
};

// forward brick / backward brick extents (work-unit geometry for the host planner)
int forward_brick(int axis, int layers);   // 0: x, 1: y (the brick's layers: 8, or 16 in STRICT), 2: z
bool forward_layers_ok(int arith, int layers);
int backward_brick(int axis, int cb);
// kind 0: forward (cb = its brick layers), 1: backward (cb = its column length)
int batched_ctas_per_sm(int kind, int arith, int dtype, int cb);
cudaError_t launch_forward_batched(const BatchFwdItem *items, int n_items, uint32_t total_units, uint32_t *ticket,
                                   int arith, int layers, unsigned ctas, cudaStream_t s);
cudaError_t launch_backward_batched(const BatchBwdItem *items, int n_items, uint32_t total_units, uint32_t *ticket,
                                    int arith, int dtype, int cb, unsigned ctas, cudaStream_t s);
cudaError_t launch_error_batched(const BatchErrItem *items, int n_items, int image_dtype, int ratio_dtype,
                                 uint64_t max_n, const DeviceInfo &dev, cudaStream_t s);
cudaError_t launch_fill_batched(const BatchFillItem *items, int n_items, uint64_t max_n, const DeviceInfo &dev,
                                cudaStream_t s);

}  // namespace xpr
