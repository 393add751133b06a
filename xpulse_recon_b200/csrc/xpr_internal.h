// xpr_internal.h -- internal C++ interface between the C ABI, the host
// schedulers and the CUDA kernels (not installed; include/xpr.h is the boundary).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/xpr.h"

namespace xpr {

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

}  // namespace xpr
