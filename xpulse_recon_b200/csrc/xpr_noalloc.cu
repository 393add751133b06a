// xpr_noalloc.cu -- xpr_subiteration_static: one sub-iteration that allocates nothing.
//
// Some callers cannot allocate device memory while they run: a host application that
// owns the whole device budget and hands this library only its inputs and outputs, a
// frame loop that must never stall on cudaMalloc / cudaFree (both can synchronise the
// device) or fail on an allocation in the middle of a scan.  For them this entry point
// keeps the sub-iteration's scratch -- the fixed-point detector sums, overwritten in
// place by the FP32 ratio -- in a file-scope device array of fixed size instead of a
// caller- or library-allocated buffer.  The array exists on every GPU that loads the
// library, for the life of the process.
#include <mutex>

#include "xpr_internal.h"
#include "xpr_math.cuh"

namespace {

// 4 Mi 32-bit words (16 MiB): room for e.g. 18 projections of 384 x 576 pixels
constexpr uint64_t kScratchWords = 4ull << 20;
__device__ __align__(256) uint32_t g_subiteration_scratch[kScratchWords];

std::mutex g_mu;
uint32_t *g_scratch_addr[64];  // device address of g_subiteration_scratch, per device

}  // namespace

extern "C" {

uint64_t xpr_subiteration_static_capacity(void) { return kScratchWords; }

int xpr_subiteration_static(xpr_ctx *ctx, float *vol, const void *images, int image_dtype, const xpr_projdata *pd,
                            uint32_t n_pd, const xpr_launch *L, float weight, int first, void *stream)
{
    const xpr::DeviceInfo *di = xpr::context_device(ctx);
    if (!di) return XPR_ERR_INVALID;
    if (!vol || !images || !pd) return xpr::set_last_error(XPR_ERR_INVALID, "xpr_subiteration_static: NULL buffer");
    if (image_dtype != XPR_F32 && image_dtype != XPR_BF16 && image_dtype != XPR_F16)
        return xpr::set_last_error(XPR_ERR_INVALID, "xpr_subiteration_static: unknown image dtype %d", image_dtype);
    xpr::LaunchArgs a;
    if (const char *m = xpr::make_launch_args(L, n_pd, &a))
        return xpr::set_last_error(XPR_ERR_INVALID, "xpr_subiteration_static: %s", m);
    const uint64_t n = (uint64_t)a.img_stride * a.n_images;
    if (n > kScratchWords)
        return xpr::set_last_error(XPR_ERR_CAP,
                                   "xpr_subiteration_static: the sub-iteration needs %llu words of detector scratch "
                                   "(%u images of %u x %u pixels); the static scratch holds %llu",
                                   (unsigned long long)n, a.n_images, a.det_w, a.rows,
                                   (unsigned long long)kScratchWords);
    const int dev = di->device;
    if (dev < 0 || dev >= 64) return xpr::set_last_error(XPR_ERR_UNSUPPORTED, "device ordinal %d >= 64", dev);
    uint32_t *sum = nullptr;
    {
        // set-up, once per device, with that device current: the array's device address
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch_addr[dev]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_subiteration_scratch);
            if (e != cudaSuccess || !p)
                return xpr::set_last_error(XPR_ERR_CUDA, "xpr_subiteration_static: cudaGetSymbolAddress: %s",
                                           cudaGetErrorString(e));
            g_scratch_addr[dev] = (uint32_t *)p;
        }
        sum = g_scratch_addr[dev];
    }
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // the array keeps the previous call's contents: start from FIXED_ONE (the first
    // sub-iteration, reconstruction_n.hpp:60) or from zero sums
    cudaError_t e = xpr::launch_fill_u32(sum, first ? xpr::kFixedOne : 0u, n, *di, s);
    if (e == cudaSuccess && !first) e = xpr::launch_forward(vol, sum, pd, a, L->arith, L->compat_pad, *di, s);
    if (e == cudaSuccess)
        e = xpr::launch_error(images, image_dtype, sum, sum, XPR_F32, n, weight, XPR_ERROR_STD, 0, nullptr, *di, s);
    if (e == cudaSuccess)
        e = xpr::launch_backward(vol, sum, XPR_F32, pd, a, L->arith, L->compat_pad, L->nan_skip, *di, s);
    if (e != cudaSuccess)
        return xpr::set_last_error(XPR_ERR_CUDA, "xpr_subiteration_static: %s", cudaGetErrorString(e));
    return XPR_OK;
}

}  // extern "C"
