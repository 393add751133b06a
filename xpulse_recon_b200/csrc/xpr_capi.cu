// xpr_capi.cu -- the C ABI (include/xpr.h): context, memory, operator entry points.
//
// Replaces the reference's gpu::Context / gpu::Kernel plumbing
// (src/reconstruction/gpu/context.hpp, kernel.hpp) and the protected operator API
// of class Reconstruction (src/reconstruction.hpp:166-312).  No exception crosses
// the boundary: failures return a status and leave a thread-local message.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>

#include "host/pinned.h"
#include "xpr_internal.h"

struct xpr_ctx {
    int device = 0;
    uint64_t cap = 0;        // 0 = no cap
    uint64_t allocated = 0;  // device bytes allocated through this context
    xpr::DeviceInfo dev;
    std::mutex mu;
    std::unordered_map<void *, uint64_t> allocs;
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    return fail(e == cudaErrorMemoryAllocation ? XPR_ERR_OOM : XPR_ERR_CUDA, "%s: %s (%d)", what,
                cudaGetErrorString(e), (int)e);
}

#define XPR_CHECK_CTX(ctx)                                                  \
    do {                                                                    \
        if (!(ctx)) return fail(XPR_ERR_INVALID, "context is NULL");        \
        cudaError_t _e = cudaSetDevice((ctx)->device);                      \
        if (_e != cudaSuccess) return cuda_fail(_e, "cudaSetDevice");       \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

inline bool valid_dtype(int d) { return d == XPR_F32 || d == XPR_BF16 || d == XPR_F16; }

}  // namespace

namespace xpr {

const DeviceInfo *context_device(xpr_ctx *ctx)
{
    if (!ctx) {
        fail(XPR_ERR_INVALID, "context is NULL");
        return nullptr;
    }
    const cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) {
        cuda_fail(e, "cudaSetDevice");
        return nullptr;
    }
    return &ctx->dev;
}

int set_last_error(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

}  // namespace xpr

extern "C" {

const char *xpr_last_error(void) { return g_last_error.c_str(); }
int xpr_abi_version(void) { return XPR_ABI_VERSION; }
uint64_t xpr_ndrange(uint64_t n) { return n + (32u - n % 32u); }

int xpr_create(int device, uint64_t mem_cap_bytes, xpr_ctx **out)
{
    if (!out) return fail(XPR_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= count) return fail(XPR_ERR_INVALID, "device %d out of range (%d devices)", device, count);
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
    if (prop.major < 10) return fail(XPR_ERR_UNSUPPORTED, "device %d is sm_%d%d; this build targets sm_100a", device, prop.major, prop.minor);
    e = xpr::prepare_device_kernels();
    if (e != cudaSuccess) return cuda_fail(e, "kernel attributes");
    xpr_ctx *c = new xpr_ctx();
    c->device = device;
    c->cap = mem_cap_bytes;
    c->dev.device = device;
    c->dev.sm_count = prop.multiProcessorCount;
    *out = c;
    return XPR_OK;
}

int xpr_destroy(xpr_ctx *ctx)
{
    if (!ctx) return XPR_OK;
    cudaSetDevice(ctx->device);
    for (auto &kv : ctx->allocs) cudaFree(kv.first);
    delete ctx;
    return XPR_OK;
}

int xpr_mem_available(xpr_ctx *ctx, uint64_t *bytes)
{
    XPR_CHECK_CTX(ctx);
    if (!bytes) return fail(XPR_ERR_INVALID, "bytes is NULL");
    size_t fr = 0, tot = 0;
    cudaError_t e = cudaMemGetInfo(&fr, &tot);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemGetInfo");
    uint64_t avail = fr;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (ctx->cap) avail = std::min<uint64_t>(avail, ctx->cap > ctx->allocated ? ctx->cap - ctx->allocated : 0);
    *bytes = avail;
    return XPR_OK;
}

int xpr_alloc(xpr_ctx *ctx, uint64_t bytes, void **dptr)
{
    XPR_CHECK_CTX(ctx);
    if (!dptr) return fail(XPR_ERR_INVALID, "dptr is NULL");
    *dptr = nullptr;
    if (bytes == 0) bytes = 4;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        if (ctx->cap && ctx->allocated + bytes > ctx->cap)
            return fail(XPR_ERR_CAP, "allocation of %llu bytes exceeds the %llu-byte cap (%llu in use)",
                        (unsigned long long)bytes, (unsigned long long)ctx->cap, (unsigned long long)ctx->allocated);
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "cudaMalloc");
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->allocs[p] = bytes;
    ctx->allocated += bytes;
    *dptr = p;
    return XPR_OK;
}

int xpr_free(xpr_ctx *ctx, void *dptr)
{
    XPR_CHECK_CTX(ctx);
    if (!dptr) return XPR_OK;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->allocs.find(dptr);
        if (it == ctx->allocs.end()) return fail(XPR_ERR_INVALID, "pointer was not allocated by this context");
        ctx->allocated -= it->second;
        ctx->allocs.erase(it);
    }
    cudaError_t e = cudaFree(dptr);
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "cudaFree");
}

int xpr_alloc_pinned(xpr_ctx *ctx, uint64_t bytes, void **hptr)
{
    XPR_CHECK_CTX(ctx);
    if (!hptr) return fail(XPR_ERR_INVALID, "hptr is NULL");
    cudaError_t e = xpr::pinned_alloc(hptr, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *hptr = nullptr;
        return cuda_fail(e, "page-locked host allocation");
    }
    return XPR_OK;
}

int xpr_free_pinned(xpr_ctx *ctx, void *hptr)
{
    XPR_CHECK_CTX(ctx);
    if (!hptr) return XPR_OK;
    cudaError_t e = xpr::pinned_free(hptr);
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "page-locked host release");
}

int xpr_upload(xpr_ctx *ctx, void *dst, const void *src, uint64_t bytes, void *stream)
{
    xpr::Range nvtx("xpr.upload");
    XPR_CHECK_CTX(ctx);
    if (!bytes) return XPR_OK;
    if (!dst || !src) return fail(XPR_ERR_INVALID, "NULL pointer");
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, as_stream(stream));
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "upload");
}

int xpr_download(xpr_ctx *ctx, void *dst, const void *src, uint64_t bytes, void *stream)
{
    xpr::Range nvtx("xpr.download");
    XPR_CHECK_CTX(ctx);
    if (!bytes) return XPR_OK;
    if (!dst || !src) return fail(XPR_ERR_INVALID, "NULL pointer");
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, as_stream(stream));
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "download");
}

int xpr_fill_u32(xpr_ctx *ctx, void *dst, uint32_t value, uint64_t count, void *stream)
{
    XPR_CHECK_CTX(ctx);
    if (!count) return XPR_OK;
    if (!dst) return fail(XPR_ERR_INVALID, "dst is NULL");
    cudaError_t e = xpr::launch_fill_u32(dst, value, count, ctx->dev, as_stream(stream));
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "fill");
}

int xpr_synchronize(xpr_ctx *ctx, void *stream)
{
    XPR_CHECK_CTX(ctx);
    cudaError_t e = stream ? cudaStreamSynchronize(as_stream(stream)) : cudaDeviceSynchronize();
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "synchronize");
}

int xpr_forward(xpr_ctx *ctx, const float *vol, uint32_t *sum, const xpr_projdata *pd, uint32_t n_pd,
                const xpr_launch *L, void *stream)
{
    xpr::Range nvtx("xpr.forward");
    XPR_CHECK_CTX(ctx);
    if (!vol || !sum || !pd) return fail(XPR_ERR_INVALID, "NULL buffer");
    xpr::LaunchArgs a;
    if (const char *m = xpr::make_launch_args(L, n_pd, &a)) return fail(XPR_ERR_INVALID, "forward: %s", m);
    cudaError_t e = xpr::launch_forward(vol, sum, pd, a, L->arith, L->compat_pad, ctx->dev, as_stream(stream));
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "forward launch");
}

int xpr_backward(xpr_ctx *ctx, float *vol, const void *ratio, int ratio_dtype, const xpr_projdata *pd, uint32_t n_pd,
                 const xpr_launch *L, void *stream)
{
    xpr::Range nvtx("xpr.backward");
    XPR_CHECK_CTX(ctx);
    if (!vol || !ratio || !pd) return fail(XPR_ERR_INVALID, "NULL buffer");
    if (!valid_dtype(ratio_dtype)) return fail(XPR_ERR_INVALID, "unknown ratio dtype %d", ratio_dtype);
    xpr::LaunchArgs a;
    if (const char *m = xpr::make_launch_args(L, n_pd, &a)) return fail(XPR_ERR_INVALID, "backward: %s", m);
    cudaError_t e = xpr::launch_backward(vol, ratio, ratio_dtype, pd, a, L->arith, L->compat_pad, L->nan_skip, ctx->dev,
                                         as_stream(stream));
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "backward launch");
}

int xpr_error(xpr_ctx *ctx, const void *images, int image_dtype, uint32_t *sum, void *ratio, int ratio_dtype,
              uint64_t n, float weight, int mode, int zero_sum, double *residual, void *stream)
{
    xpr::Range nvtx("xpr.error");
    XPR_CHECK_CTX(ctx);
    if (!images || !sum || !ratio) return fail(XPR_ERR_INVALID, "NULL buffer");
    if (!valid_dtype(image_dtype) || !valid_dtype(ratio_dtype)) return fail(XPR_ERR_INVALID, "unknown dtype");
    if ((void *)sum == ratio && ratio_dtype != XPR_F32) return fail(XPR_ERR_INVALID, "in-place ratio must be F32");
    if (mode < XPR_ERROR_STD || mode > XPR_ERROR_1C) return fail(XPR_ERR_INVALID, "unknown error mode %d", mode);
    cudaError_t e = xpr::launch_error(images, image_dtype, sum, ratio, ratio_dtype, n, weight, mode, zero_sum, residual,
                                      ctx->dev, as_stream(stream));
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "error launch");
}

int xpr_preprocess_minmax(xpr_ctx *ctx, const float *images, uint64_t n, float *minmax, void *stream)
{
    xpr::Range nvtx("xpr.preprocess_minmax");
    XPR_CHECK_CTX(ctx);
    if (!minmax || (n && !images)) return fail(XPR_ERR_INVALID, "NULL buffer");
    cudaError_t e = xpr::launch_minmax(images, n, minmax, ctx->dev, as_stream(stream));
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "minmax launch");
}

int xpr_preprocess_apply(xpr_ctx *ctx, const float *images, void *out, int out_dtype, uint64_t n, int normalize,
                         const float *minmax, int mlog, void *stream)
{
    xpr::Range nvtx("xpr.preprocess");
    XPR_CHECK_CTX(ctx);
    if (n && (!images || !out)) return fail(XPR_ERR_INVALID, "NULL buffer");
    if (normalize && !minmax) return fail(XPR_ERR_INVALID, "normalize needs minmax");
    if (!valid_dtype(out_dtype)) return fail(XPR_ERR_INVALID, "unknown dtype");
    if ((const void *)images == out && out_dtype != XPR_F32) return fail(XPR_ERR_INVALID, "in-place output must be F32");
    cudaError_t e = xpr::launch_preprocess(images, out, out_dtype, n, normalize, minmax, mlog, ctx->dev, as_stream(stream));
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "preprocess launch");
}

int xpr_subiteration(xpr_ctx *ctx, float *vol, uint32_t *sum, const void *images, int image_dtype, void *ratio,
                     int ratio_dtype, const xpr_projdata *pd, uint32_t n_pd, const xpr_launch *L, float weight,
                     int first, double *residual, void *stream)
{
    xpr::Range nvtx("xpr.subiteration");
    XPR_CHECK_CTX(ctx);
    if (!vol || !sum || !images || !ratio || !pd) return fail(XPR_ERR_INVALID, "NULL buffer");
    if (!valid_dtype(image_dtype) || !valid_dtype(ratio_dtype)) return fail(XPR_ERR_INVALID, "unknown dtype");
    if ((void *)sum == ratio && ratio_dtype != XPR_F32) return fail(XPR_ERR_INVALID, "in-place ratio must be F32");
    xpr::LaunchArgs a;
    if (const char *m = xpr::make_launch_args(L, n_pd, &a)) return fail(XPR_ERR_INVALID, "subiteration: %s", m);
    const uint64_t n = (uint64_t)a.img_stride * a.n_images;
    cudaStream_t s = as_stream(stream);
    cudaError_t e = cudaSuccess;
    if (!first) e = xpr::launch_forward(vol, sum, pd, a, L->arith, L->compat_pad, ctx->dev, s);
    if (e == cudaSuccess)
        e = xpr::launch_error(images, image_dtype, sum, ratio, ratio_dtype, n, weight, XPR_ERROR_STD, 1, residual,
                              ctx->dev, s);
    if (e == cudaSuccess)
        e = xpr::launch_backward(vol, ratio, ratio_dtype, pd, a, L->arith, L->compat_pad, L->nan_skip, ctx->dev, s);
    if (e == cudaSuccess && (void *)sum == ratio) e = cudaMemsetAsync(sum, 0, n * 4, s);
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "subiteration");
}

}  // extern "C"
