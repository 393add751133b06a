// engine.cpp -- see engine.h
#include "engine.h"
#include "hostcopy.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <functional>
#include <iostream>
#include <sstream>
#include <stdexcept>

#include "planner.h"
#include "tiff.h"

namespace fs = std::filesystem;

namespace xpr {

namespace {

void check(int status, const char *what)
{
    if (status != XPR_OK) throw std::runtime_error(std::string(what) + ": " + xpr_last_error());
}
void check_cuda(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// device allocation owned by a context
struct DevBuf {
    xpr_ctx *c = nullptr;
    void *p = nullptr;
    uint64_t bytes = 0;
    DevBuf() = default;
    DevBuf(xpr_ctx *ctx, uint64_t n) : c(ctx), bytes(n) { check(xpr_alloc(ctx, n ? n : 4, &p), "device allocation"); }
    DevBuf(DevBuf &&o) noexcept : c(o.c), p(o.p), bytes(o.bytes) { o.p = nullptr; }
    DevBuf &operator=(DevBuf &&o) noexcept
    {
        reset();
        c = o.c; p = o.p; bytes = o.bytes; o.p = nullptr;
        return *this;
    }
    ~DevBuf() { reset(); }
    void reset()
    {
        if (p) xpr_free(c, p);
        p = nullptr;
    }
    template <class T> T *as() const { return (T *)p; }
    char *at(uint64_t off) const { return (char *)p + off; }
};

// pinned host allocation
struct PinBuf {
    xpr_ctx *c = nullptr;
    void *p = nullptr;
    uint64_t bytes = 0;
    PinBuf() = default;
    PinBuf(xpr_ctx *ctx, uint64_t n) : c(ctx), bytes(n) { check(xpr_alloc_pinned(ctx, n ? n : 4, &p), "pinned allocation"); }
    ~PinBuf()
    {
        if (p) xpr_free_pinned(c, p);
    }
    PinBuf(const PinBuf &) = delete;
    template <class T> T *as() const { return (T *)p; }
    char *at(uint64_t off) const { return (char *)p + off; }
};

struct Stream {
    cudaStream_t s = nullptr;
    Stream() { check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate"); }
    ~Stream()
    {
        if (s) cudaStreamDestroy(s);
    }
    void *v() const { return (void *)s; }
    void sync() const { check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize"); }
};

struct Event {
    cudaEvent_t e = nullptr;
    Event() { check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate"); }
    ~Event()
    {
        if (e) cudaEventDestroy(e);
    }
    void record(const Stream &s) { check_cuda(cudaEventRecord(e, s.s), "cudaEventRecord"); }
    void wait_in(const Stream &s) { check_cuda(cudaStreamWaitEvent(s.s, e, 0), "cudaStreamWaitEvent"); }
};

class DirImages : public ImageSource {
public:
    explicit DirImages(const std::string &dir)
    {
        std::error_code ec;
        if (!fs::is_directory(dir, ec)) throw std::runtime_error("No valid TIFF file found in the directory.");
        std::vector<std::string> all;
        for (const auto &e : fs::directory_iterator(dir, ec)) {
            if (!e.is_regular_file()) continue;
            const std::string ext = e.path().extension().string();
            if (ext == ".tif" || ext == ".tiff") all.push_back(e.path().string());
        }
        std::sort(all.begin(), all.end());
        for (const auto &f : all) {
            TiffInfo ti;
            std::string err;
            if (!tiff_info(f, &ti, &err)) continue;
            if (ti.sample_format != 3 || ti.bits != 32)
                throw std::runtime_error("Trying to load a tiff with an incompatble format (should be floating-point 32bits)");
            if (ti.width == 0 || ti.height == 0) throw std::runtime_error("Trying to load a tiff with an incorrect size.");
            if (w_ == 0 && h_ == 0) { w_ = ti.width; h_ = ti.height; }
            if (ti.width == w_ && ti.height == h_) files_.push_back(f);  // dataset.hpp:259-266
        }
        if (files_.empty()) throw std::runtime_error("No valid TIFF file found in the directory.");
    }
    int64_t count() const override { return (int64_t)files_.size(); }
    uint32_t width() const override { return w_; }
    uint32_t height() const override { return h_; }
    void read(int64_t i, float *dst) override
    {
        uint32_t w, h;
        std::vector<float> v = tiff_read_f32(files_[(size_t)i], &w, &h);
        if (w != w_ || h != h_) throw std::runtime_error("image size changed: " + files_[(size_t)i]);
        std::memcpy(dst, v.data(), v.size() * sizeof(float));
    }

private:
    std::vector<std::string> files_;
    uint32_t w_ = 0, h_ = 0;
};

class MemImages : public ImageSource {
public:
    MemImages(const float *d, int64_t n, uint32_t w, uint32_t h) : d_(d), n_(n), w_(w), h_(h) {}
    int64_t count() const override { return n_; }
    uint32_t width() const override { return w_; }
    uint32_t height() const override { return h_; }
    void read(int64_t i, float *dst) override { par_memcpy(dst, d_ + (size_t)i * w_ * h_, sizeof(float) * w_ * h_); }

private:
    const float *d_;
    int64_t n_;
    uint32_t w_, h_;
};

std::string layer_path(const std::string &dir, int64_t l)
{
    char b[32];
    snprintf(b, sizeof b, "layer_%05lld.tif", (long long)l);
    return (fs::path(dir) / b).string();
}
std::string proj_path(const std::string &dir, int64_t l)
{
    char b[32];
    snprintf(b, sizeof b, "p_%010lld.tif", (long long)l);
    return (fs::path(dir) / b).string();
}

double now()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

std::unique_ptr<ImageSource> directory_images(const std::string &dir) { return std::make_unique<DirImages>(dir); }
std::unique_ptr<ImageSource> memory_images(const float *data, int64_t count, uint32_t width, uint32_t height)
{
    return std::make_unique<MemImages>(data, count, width, height);
}

struct Engine::Impl {
    xpr_ctx *ctx = nullptr;
    std::unique_ptr<ImageSource> src;
    bool write = false;
    std::vector<xpr_projdata> pd_all;
    std::vector<float> mod_offset, mod_rpy;
    std::mt19937 rng;
    int arith = XPR_ARITH_FAST, idt = XPR_F32, rdt = XPR_F32;  // image / ratio storage
    uint64_t iesize = 4, rsize = 4;                            // their element sizes
    int64_t P = 0, S = 0, Pc = 0, M = 1, slots = 0, W = 0, Hv = 0, Wd = 0, Hd = 0;
    uint64_t WH = 0, N = 0;
    float nmin = FLT_MAX, nmax = FLT_MIN;
    std::unique_ptr<Stream> comp, up, down;

    ~Impl()
    {
        comp.reset();
        up.reset();
        down.reset();
        if (ctx) xpr_destroy(ctx);
    }

    uint64_t available() const
    {
        uint64_t b = 0;
        check(xpr_mem_available(ctx, &b), "xpr_mem_available");
        return b;
    }

    // reconstruction.hpp:268-272: origin + U[0, vx) per axis
    void jittered_origin(const xpr_geom_out &go, float out[3])
    {
        for (int i = 0; i < 3; ++i) out[i] = go.orig[i] + std::uniform_real_distribution<float>(0.0f, go.vx)(rng);
    }

    // image i of the acquisition lives in subset slot (i % S) * slots + i / S
    int64_t slot_of(int64_t i) const { return (i % S) * slots + i / S; }
    int64_t angles_in(int64_t sit) const { return (P - sit + S - 1) / S; }

    // Reads every image, preprocesses it on the device (data_loader.hpp:48-101) and hands the
    // preprocessed image (storage dtype, device) to sink(i, ptr) on the compute stream.
    // The images one by one through two page-locked staging buffers: reading image i + 1
    // on the host overlaps the upload and preprocessing of image i on the stream; `sink`
    // enqueues its copy of the preprocessed image on the same stream.
    void preprocess(const Params &p, const std::function<void(int64_t, const void *)> &sink)
    {
        DevBuf raw[2] = {DevBuf(ctx, WH * 4), DevBuf(ctx, WH * 4)};
        DevBuf out[2] = {DevBuf(ctx, WH * iesize), DevBuf(ctx, WH * iesize)};
        DevBuf mm(ctx, 8);
        PinBuf stage0(ctx, WH * 4), stage1(ctx, WH * 4);
        PinBuf *stage[2] = {&stage0, &stage1};
        Event used[2];
        bool pending[2] = {false, false};
        auto next = [&](int64_t i) {  // image i into staging buffer i % 2, uploaded to raw[i % 2]
            const int b = (int)(i & 1);
            if (pending[b]) check_cuda(cudaEventSynchronize(used[b].e), "staging");
            src->read(i, stage[b]->as<float>());
            check(xpr_upload(ctx, raw[b].p, stage[b]->p, WH * 4, comp->v()), "upload");
            return b;
        };
        const float init[2] = {FLT_MAX, FLT_MIN};  // data_loader.hpp:12-13
        if (p.normalize) {
            check(xpr_upload(ctx, mm.p, init, 8, comp->v()), "upload");
            for (int64_t i = 0; i < P; ++i) {
                const int b = next(i);
                check(xpr_preprocess_minmax(ctx, raw[b].as<float>(), WH, mm.as<float>(), comp->v()), "minmax");
                used[b].record(*comp);
                pending[b] = true;
            }
            float h[2];
            check(xpr_download(ctx, h, mm.p, 8, comp->v()), "download");
            comp->sync();
            nmin = h[0];
            nmax = h[1];
        }
        for (int64_t i = 0; i < P; ++i) {
            const int b = next(i);
            check(xpr_preprocess_apply(ctx, raw[b].as<float>(), out[b].p, idt, WH, p.normalize ? 1 : 0,
                                       mm.as<float>(), p.mlog ? 1 : 0, comp->v()), "preprocess");
            sink(i, out[b].p);
            used[b].record(*comp);
            pending[b] = true;
        }
        comp->sync();
    }

    // n bytes of device memory to host memory: straight into page-locked memory, otherwise
    // through two page-locked chunks whose host copies overlap the next chunk's transfer
    void download_host(void *dst, const void *dsrc, uint64_t n)
    {
        cudaPointerAttributes at{};
        const bool pinned = cudaPointerGetAttributes(&at, dst) == cudaSuccess && at.type == cudaMemoryTypeHost;
        cudaGetLastError();
        if (pinned || n <= (8u << 20)) {
            check(xpr_download(ctx, dst, dsrc, n, comp->v()), "download");
            comp->sync();
            return;
        }
        const uint64_t chunk = 64u << 20;
        PinBuf c0(ctx, chunk), c1(ctx, chunk);
        PinBuf *cb[2] = {&c0, &c1};
        Event done[2];
        uint64_t pend[2] = {0, 0}, pend_off[2] = {0, 0};
        int b = 0;
        for (uint64_t off = 0; off < n; off += chunk, b ^= 1) {
            if (pend[b]) {
                check_cuda(cudaEventSynchronize(done[b].e), "download");
                par_memcpy((char *)dst + pend_off[b], cb[b]->p, pend[b]);
            }
            const uint64_t m = std::min(chunk, n - off);
            check(xpr_download(ctx, cb[b]->p, (const char *)dsrc + off, m, comp->v()), "download");
            done[b].record(*comp);
            pend[b] = m;
            pend_off[b] = off;
        }
        for (int k = 0; k < 2; ++k, b ^= 1) {
            if (!pend[b]) continue;
            check_cuda(cudaEventSynchronize(done[b].e), "download");
            par_memcpy((char *)dst + pend_off[b], cb[b]->p, pend[b]);
        }
    }

    xpr_launch launch(int32_t y0, int32_t y1, const float origin[3], float vx, uint32_t rows, int32_t row_offset,
                      uint32_t n_angles, int compat_pad) const
    {
        xpr_launch L;
        std::memset(&L, 0, sizeof L);
        L.vmin[0] = 0; L.vmin[1] = y0; L.vmin[2] = 0;
        L.vmax[0] = (int32_t)W; L.vmax[1] = y1; L.vmax[2] = (int32_t)W;
        for (int i = 0; i < 3; ++i) { L.origin[i] = origin[i]; L.voxel[i] = vx; }
        L.det_w = (uint32_t)Wd;
        L.rows = rows;
        L.row_offset = row_offset;
        L.n_angles = n_angles;
        L.modules = (uint32_t)M;
        L.arith = arith;
        L.compat_pad = compat_pad;
        return L;
    }

    // ProjData of the first Pc angles of every sub-iteration, packed per subset (geometry.hpp:306-327)
    std::vector<xpr_projdata> subset_projdata() const
    {
        std::vector<xpr_projdata> v((size_t)(S * Pc * M));
        for (int64_t s = 0; s < S; ++s)
            for (int64_t k = 0; k < Pc; ++k)
                for (int64_t m = 0; m < M; ++m) v[(size_t)((s * Pc + k) * M + m)] = pd_all[(size_t)((s + k * S) * M + m)];
        return v;
    }

    // recon.resume: layers [y0, y1) of a previous result's stack into dst (W x W each); saved
    // layers carry the normalisation's (max - min) factor, divided out here
    void load_layers(const Params &p, float *dst, int64_t y0, int64_t y1)
    {
        for (int64_t l = y0; l < y1; ++l) {
            uint32_t w = 0, h = 0;
            std::vector<float> layer = tiff_read_f32(layer_path(p.resume, l), &w, &h);
            if (w != (uint32_t)W || h != (uint32_t)W)
                throw std::runtime_error("recon.resume: layer size mismatch: " + layer_path(p.resume, l));
            if (p.normalize)
                for (auto &v : layer) v = v / (nmax - nmin);
            std::memcpy(dst + (size_t)(l - y0) * W * W, layer.data(), sizeof(float) * W * W);
        }
    }

    // recon.first_iteration k: iteration k's weight (the schedule's float products) and the
    // origin-jitter draws of iterations 0 .. k - 1 taken and dropped
    float start_weight(const Params &p) const
    {
        float w = p.weight;
        for (int64_t k = 0; k < p.first_iteration; ++k) w *= p.weight_factor;
        return w;
    }
    void skip_jitter(const Params &p, const xpr_geom_out &go)
    {
        float o[3];
        for (int64_t k = 0; k < p.first_iteration * S; ++k) jittered_origin(go, o);
    }
    // the reference skips the very first forward (the uniform volume's sums are preset); a
    // resumed volume is not uniform, so every sub-iteration of a resumed run projects
    static bool skips_forward(const Params &p, int64_t mit, int64_t sit)
    {
        return mit == 0 && sit == 0 && p.resume.empty();
    }
    // the sums' value before the run's first sub-iteration: FIXED(1) where that sub-iteration
    // skips its forward (reconstruction_n.hpp:60), else zero, as after any sub-iteration
    static uint32_t first_sums(const Params &p) { return skips_forward(p, p.first_iteration, 0) ? 1u << 22 : 0u; }

    void save_layers(const Params &p, const float *vol, int64_t y0, int64_t y1)
    {
        std::vector<float> layer((size_t)(W * W));
        for (int64_t l = y0; l < y1; ++l) {
            std::memcpy(layer.data(), vol + (size_t)(l - y0) * W * W, sizeof(float) * W * W);
            if (p.normalize)  // data_loader.hpp:133-141
                for (auto &v : layer) v = v * (nmax - nmin);
            tiff_write_f32(layer_path(p.output, l), layer.data(), (uint32_t)W, (uint32_t)W);
        }
    }
};

Engine::Engine(const Params &p, std::unique_ptr<ImageSource> images, bool write_files) : d_(new Impl), p_(p)
{
    Impl &d = *d_;
    d.src = std::move(images);
    d.write = write_files;
    if (p.method == Method::hartmann || p.method == Method::ipr)
        throw std::runtime_error(std::string("method '") + method_name(p.method) + "' is not provided by this backend");
    check(xpr_create(p.device, p.mem_cap, &d.ctx), "xpr_create");
    d.comp = std::make_unique<Stream>();
    d.up = std::make_unique<Stream>();
    d.down = std::make_unique<Stream>();
    if (p.seed_set) d.rng.seed(p.seed);
    else d.rng.seed(std::random_device()());
    d.arith = p.arith == "strict" ? XPR_ARITH_STRICT : XPR_ARITH_FAST;
    d.rdt = p.storage == "bf16" ? XPR_BF16 : (p.storage == "fp16" ? XPR_F16 : XPR_F32);
    d.idt = p.image_storage.empty() ? d.rdt
               : (p.image_storage == "bf16" ? XPR_BF16 : (p.image_storage == "fp16" ? XPR_F16 : XPR_F32));
    d.iesize = d.idt == XPR_F32 ? 4 : 2;
    d.rsize = d.rdt == XPR_F32 ? 4 : 2;
    // dataset.hpp:214-235
    d.P = d.src->count();
    d.Wd = d.src->width();
    d.Hd = d.src->height();
    d.S = p.sit;
    d.M = p.module_number;
    if (!p.angle_list.empty() && (int64_t)p.angle_list.size() != d.P)
        throw std::runtime_error("The size of the angle list is different from the number of projections");
    geom_params_from(p, d.P, d.Wd, d.Hd, &gp_, &d.mod_offset, &d.mod_rpy);
    d.pd_all.resize((size_t)(d.P * d.M));
    check(xpr_geometry(&gp_, p.geometry == "fp64" ? 1 : 0, d.pd_all.data(), &go_), "geometry");
    d.Pc = go_.concurrent;
    if (d.Pc < 1) throw std::runtime_error("fewer projections than sub-iterations");
    d.slots = (d.P + d.S - 1) / d.S;
    d.W = go_.vwidth;
    d.Hv = go_.vheight;
    d.WH = (uint64_t)d.Wd * d.Hd;
    d.N = (uint64_t)d.W * d.Hv * d.W;
    if (write_files) {
        fs::create_directories(p.output);
        if (!p.proj_output.empty()) fs::create_directories(p.proj_output);
    }
    std::cout << "Volume dimension : " << d.W << "x" << d.Hv << "x" << d.W << std::endl;
    std::cout << "Pixel size : " << p.px << ", Voxel size : " << go_.vx << std::endl;
}

Engine::~Engine() = default;

void Engine::reconstruct()
{
    Impl &d = *d_;
    const Params &p = p_;
    const double t0 = now();
    const uint64_t WH = d.WH, N = d.N;
    const int64_t W = d.W, Hv = d.Hv, S = d.S, Pc = d.Pc, M = d.M;
    const size_t PDB = sizeof(xpr_projdata);
    float origin[3];
    // the result goes to the caller's buffer when one is set, else to volume_
    float *vout = out_;
    if (!vout) {
        volume_.resize(N);
        vout = volume_.data();
    }

    if (p.method == Method::naive) {
        const uint64_t nvol = p.compat_pad ? xpr_ndrange(N) : N;
        const bool sep = d.rdt != XPR_F32;
        const uint64_t need = nvol * 4 + (uint64_t)(S * Pc) * WH * d.iesize + Pc * WH * 4 + (sep ? Pc * WH * d.rsize : 0) +
                              (uint64_t)(S * Pc * M) * PDB;
        std::cout << "Checking GPU memory requierments : " << need / (1024 * 1024) << "Mo" << std::endl;
        if (need > d.available()) throw std::runtime_error("Not enough GPU memory");
        DevBuf img(d.ctx, (uint64_t)(S * Pc) * WH * d.iesize), vol(d.ctx, nvol * 4), sum(d.ctx, Pc * WH * 4);
        DevBuf ratio = sep ? DevBuf(d.ctx, Pc * WH * d.rsize) : DevBuf();
        DevBuf pd(d.ctx, (uint64_t)(S * Pc * M) * PDB);
        std::cout << "Pre-processing images..." << std::flush;
        d.preprocess(p, [&](int64_t i, const void *dimg) {
            if (i / S >= Pc) return;  // the kernels use the first Pc angles of a sub-iteration
            const uint64_t slot = (uint64_t)((i % S) * Pc + i / S);
            check_cuda(cudaMemcpyAsync(img.at(slot * WH * d.iesize), dimg, WH * d.iesize, cudaMemcpyDeviceToDevice,
                                       d.comp->s), "copy");
        });
        std::cout << "Ok." << std::endl;
        const std::vector<xpr_projdata> spd = d.subset_projdata();
        check(xpr_upload(d.ctx, pd.p, spd.data(), spd.size() * PDB, d.comp->v()), "upload");
        check(xpr_fill_u32(d.ctx, vol.p, 0x3f800000u, nvol, d.comp->v()), "fill");          // :59
        check(xpr_fill_u32(d.ctx, sum.p, Impl::first_sums(p), Pc * WH, d.comp->v()), "fill");  // :60
        if (!p.resume.empty()) {
            std::vector<float> init(N);
            d.load_layers(p, init.data(), 0, Hv);
            check(xpr_upload(d.ctx, vol.p, init.data(), N * 4, d.comp->v()), "upload");
            d.comp->sync();
        }
        std::cout << "Executing reconstruction..." << std::flush;
        const double t1 = now();
        float weight = d.start_weight(p);
        d.skip_jitter(p, go_);
        for (int64_t mit = p.first_iteration; mit < p.it; ++mit) {
            for (int64_t sit = 0; sit < S; ++sit) {
                d.jittered_origin(go_, origin);
                xpr_launch L = d.launch(0, (int32_t)Hv, origin, go_.vx, (uint32_t)d.Hd, 0, (uint32_t)Pc,
                                        p.compat_pad ? 1 : 0);
                const bool first = Impl::skips_forward(p, mit, sit);
                check(xpr_subiteration(d.ctx, vol.as<float>(), sum.as<uint32_t>(),
                                       img.at((uint64_t)sit * Pc * WH * d.iesize), d.idt, sep ? ratio.p : sum.p,
                                       d.rdt, (const xpr_projdata *)pd.at((uint64_t)sit * Pc * M * PDB),
                                       (uint32_t)(Pc * M), &L, weight, first ? 1 : 0, nullptr, d.comp->v()),
                      "sub-iteration");
                stats_.subiterations++;
                stats_.pairs += (uint64_t)(first ? 1 : 2) * N * Pc;
            }
            weight *= p.weight_factor;
        }
        d.comp->sync();
        stats_.seconds_iterations = now() - t1;
        std::cout << "Ok" << std::endl;
        d.download_host(vout, vol.p, N * 4);
        if (d.write) {
            std::cout << "Saving result..." << std::flush;
            d.save_layers(p, vout, 0, Hv);
            std::cout << "Ok" << std::endl;
        }
        stats_.seconds_total = now() - t0;
        return;
    }

    if (p.method == Method::method_1a || p.method == Method::method_1b || p.method == Method::method_1c) {
        const bool lplh = p.method == Method::method_1c;
        const bool sync_mode = p.method == Method::method_1a;
        const int64_t slots = lplh ? d.slots : Pc;
        const bool sep = d.rdt != XPR_F32;
        PinBuf hvol(d.ctx, N * 4);
        PinBuf himg(d.ctx, (uint64_t)(S * slots) * WH * d.iesize);
        // device: one sub-iteration's images and sums, ProjData, lists, slab buffers
        DevBuf img(d.ctx, (uint64_t)slots * WH * d.iesize), sum(d.ctx, (uint64_t)slots * WH * 4);
        DevBuf ratio = sep ? DevBuf(d.ctx, (uint64_t)slots * WH * d.rsize) : DevBuf();
        DevBuf pd, lm, li;
        std::vector<uint16_t> hl_m, hl_i;
        if (lplh) {
            // every (angle, module) of the sub-iteration, image slot = position in the sub-iteration;
            // the per-layer culling of geometry.hpp:141-171 is conservative, so it drops no
            // in-bounds pair and the full list gives the same sums and updates
            pd = DevBuf(d.ctx, d.pd_all.size() * PDB);
            check(xpr_upload(d.ctx, pd.p, d.pd_all.data(), d.pd_all.size() * PDB, d.comp->v()), "upload");
            hl_m.resize((size_t)(S * slots * M));
            hl_i.resize(hl_m.size());
            for (int64_t s = 0; s < S; ++s)
                for (int64_t k = 0; k < slots; ++k)
                    for (int64_t m = 0; m < M; ++m) {
                        const size_t e = (size_t)((s * slots + k) * M + m);
                        const int64_t i = s + k * S;
                        hl_m[e] = (uint16_t)(i < d.P ? i * M + m : 0);
                        hl_i[e] = (uint16_t)k;
                    }
            lm = DevBuf(d.ctx, hl_m.size() * 2);
            li = DevBuf(d.ctx, hl_i.size() * 2);
            check(xpr_upload(d.ctx, lm.p, hl_m.data(), hl_m.size() * 2, d.comp->v()), "upload");
            check(xpr_upload(d.ctx, li.p, hl_i.data(), hl_i.size() * 2, d.comp->v()), "upload");
        } else {
            const std::vector<xpr_projdata> spd = d.subset_projdata();
            pd = DevBuf(d.ctx, spd.size() * PDB);
            check(xpr_upload(d.ctx, pd.p, spd.data(), spd.size() * PDB, d.comp->v()), "upload");
        }
        std::cout << "Pre-processing images..." << std::flush;
        d.preprocess(p, [&](int64_t i, const void *dimg) {
            if (i / S >= slots) return;
            check_cuda(cudaMemcpyAsync(himg.at((uint64_t)((i % S) * slots + i / S) * WH * d.iesize), dimg, WH * d.iesize,
                                       cudaMemcpyDeviceToHost, d.comp->s), "copy");
        });
        std::cout << "Ok." << std::endl;
        const uint64_t layer_bytes = (uint64_t)W * W * 4;
        const float init = lplh ? 1.0f / (float)std::sqrt((double)(W * W)) : 1.0f;  // reconstruction_lplh.hpp:194
        float *hv = hvol.as<float>();
#pragma omp parallel for schedule(static) num_threads(8)
        for (int64_t i = 0; i < (int64_t)N; ++i) hv[i] = init;
        if (!p.resume.empty()) d.load_layers(p, hv, 0, Hv);
        if (!lplh)  // reconstruction_lpla.hpp:243
            check(xpr_fill_u32(d.ctx, sum.p, Impl::first_sums(p), (uint64_t)slots * WH, d.comp->v()), "fill");
        double t1 = 0.0;
        if (sync_mode) {
            // method_1a (reconstruction_lpln.hpp:27-96): one slab buffer, every transfer
            // synchronous with the projector
            const uint64_t avail = d.available();
            const uint64_t budget = avail > (64ull << 20) ? avail - (64ull << 20) : layer_bytes;
            int64_t slab = std::max<int64_t>(1, std::min<int64_t>(Hv, (int64_t)(budget / layer_bytes)));
            if (p.slab > 0) slab = std::min<int64_t>(slab, p.slab);
            DevBuf sb(d.ctx, (uint64_t)slab * layer_bytes);
            std::cout << "Executing reconstruction..." << std::flush;
            t1 = now();
            float weight = d.start_weight(p);
            d.skip_jitter(p, go_);
            const int64_t nslab = (Hv + slab - 1) / slab;
            for (int64_t mit = p.first_iteration; mit < p.it; ++mit) {
                for (int64_t sit = 0; sit < S; ++sit) {
                    d.jittered_origin(go_, origin);
                    const bool first = Impl::skips_forward(p, mit, sit);
                    check(xpr_upload(d.ctx, img.p, himg.at((uint64_t)sit * slots * WH * d.iesize),
                                     (uint64_t)Pc * WH * d.iesize, d.comp->v()), "upload");
                    const void *pdp = pd.at((uint64_t)sit * Pc * M * PDB);
                    if (!first) {
                        for (int64_t j = 0; j < nslab; ++j) {
                            const int64_t y0 = j * slab, ny = std::min<int64_t>(Hv, (j + 1) * slab) - y0;
                            check(xpr_upload(d.ctx, sb.p, hvol.at((uint64_t)y0 * layer_bytes),
                                             (uint64_t)ny * layer_bytes, d.comp->v()), "upload");
                            xpr_launch L = d.launch((int32_t)y0, (int32_t)(y0 + ny), origin, go_.vx, (uint32_t)d.Hd,
                                                    0, (uint32_t)Pc, 0);
                            check(xpr_forward(d.ctx, sb.as<float>(), sum.as<uint32_t>(), (const xpr_projdata *)pdp,
                                              (uint32_t)(Pc * M), &L, d.comp->v()), "forward");
                            stats_.pairs += (uint64_t)ny * W * W * Pc;
                        }
                    }
                    check(xpr_error(d.ctx, img.p, d.idt, sum.as<uint32_t>(), sep ? ratio.p : sum.p, d.rdt,
                                    (uint64_t)Pc * WH, weight, XPR_ERROR_STD, 0, nullptr, d.comp->v()), "error");
                    for (int64_t j = 0; j < nslab; ++j) {
                        const int64_t y0 = j * slab, ny = std::min<int64_t>(Hv, (j + 1) * slab) - y0;
                        check(xpr_upload(d.ctx, sb.p, hvol.at((uint64_t)y0 * layer_bytes), (uint64_t)ny * layer_bytes,
                                         d.comp->v()), "upload");
                        xpr_launch L = d.launch((int32_t)y0, (int32_t)(y0 + ny), origin, go_.vx, (uint32_t)d.Hd, 0,
                                                (uint32_t)Pc, 0);
                        check(xpr_backward(d.ctx, sb.as<float>(), sep ? ratio.p : sum.p, d.rdt,
                                           (const xpr_projdata *)pdp, (uint32_t)(Pc * M), &L, d.comp->v()),
                              "backward");
                        stats_.pairs += (uint64_t)ny * W * W * Pc;
                        check(xpr_download(d.ctx, hvol.at((uint64_t)y0 * layer_bytes), sb.p,
                                           (uint64_t)ny * layer_bytes, d.comp->v()), "download");
                    }
                    check(xpr_fill_u32(d.ctx, sum.p, 0u, (uint64_t)slots * WH, d.comp->v()), "fill");
                    d.comp->sync();
                    stats_.subiterations++;
                }
                weight *= p.weight_factor;
            }
        } else {
            // method_1b / 1c (reconstruction_lpla.hpp:29-157, reconstruction_lplh.hpp:40-219) with
            // the volume's slabs kept in a device cache: as many slab buffers as the memory left
            // beside the images holds (all of them when the volume fits), forward passes in
            // ascending and backward passes in descending slab order so that each pass starts
            // on the slabs the previous one left resident, a slab written back to the host
            // only when its buffer is needed for another.  Uploads and write-backs run on
            // their own streams, ordered against the projector by events.
            const uint64_t avail = d.available();
            const uint64_t budget = avail > (64ull << 20) ? avail - (64ull << 20) : layer_bytes;
            int64_t slab = std::max<int64_t>(1, std::min<int64_t>(Hv, (int64_t)(budget / 8 / layer_bytes)));
            if (p.slab > 0) slab = std::min<int64_t>(slab, p.slab);
            const int64_t nslab = (Hv + slab - 1) / slab;
            int64_t nb = std::max<int64_t>(1, std::min<int64_t>(nslab, (int64_t)(budget / (slab * layer_bytes))));
            if (p.slab_cache > 0) nb = std::min<int64_t>(nb, p.slab_cache);
            struct SlabBuf {
                DevBuf mem;
                int64_t slab = -1;
                bool dirty = false, used_rec = false, saved_rec = false;
                uint64_t last = 0;
                Event ready, used, saved;
            };
            std::vector<std::unique_ptr<SlabBuf>> bufs;
            for (int64_t b = 0; b < nb; ++b) {
                bufs.emplace_back(std::make_unique<SlabBuf>());
                bufs.back()->mem = DevBuf(d.ctx, (uint64_t)slab * layer_bytes);
            }
            Event last_save;
            bool any_save = false;
            uint64_t clock = 0;
            auto extent = [&](int64_t j) {
                const int64_t y0 = j * slab;
                return std::make_pair(y0, std::min<int64_t>(Hv, y0 + slab) - y0);
            };
            auto write_back = [&](SlabBuf &b) {
                const auto [y0, ny] = extent(b.slab);
                if (b.used_rec) b.used.wait_in(*d.down);
                check(xpr_download(d.ctx, hvol.at((uint64_t)y0 * layer_bytes), b.mem.p, (uint64_t)ny * layer_bytes,
                                   d.down->v()), "download");
                b.saved.record(*d.down);
                b.saved_rec = true;
                last_save.record(*d.down);
                any_save = true;
                b.dirty = false;
            };
            auto acquire = [&](int64_t j) -> SlabBuf & {
                SlabBuf *v = nullptr;
                for (auto &b : bufs)
                    if (b->slab == j) v = b.get();
                if (!v) {  // load slab j into the least recently used buffer
                    for (auto &b : bufs)
                        if (!v || b->slab < 0 || (v->slab >= 0 && b->last < v->last)) v = b.get();
                    if (v->slab >= 0 && v->dirty) write_back(*v);
                    if (v->used_rec) v->used.wait_in(*d.up);
                    if (v->saved_rec) v->saved.wait_in(*d.up);
                    if (any_save) last_save.wait_in(*d.up);  // the host copy of slab j is current
                    const auto [y0, ny] = extent(j);
                    check(xpr_upload(d.ctx, v->mem.p, hvol.at((uint64_t)y0 * layer_bytes), (uint64_t)ny * layer_bytes,
                                     d.up->v()), "upload");
                    v->ready.record(*d.up);
                    v->ready.wait_in(*d.comp);
                    v->slab = j;
                    v->dirty = false;
                }
                v->last = ++clock;
                return *v;
            };
            std::cout << "Executing reconstruction..." << std::flush;
            t1 = now();
            float weight = d.start_weight(p);
            d.skip_jitter(p, go_);
            for (int64_t mit = p.first_iteration; mit < p.it; ++mit) {
                for (int64_t sit = 0; sit < S; ++sit) {
                    d.jittered_origin(go_, origin);
                    const bool first = Impl::skips_forward(p, mit, sit);
                    const int64_t nimg = lplh ? d.angles_in(sit) : Pc;
                    check(xpr_upload(d.ctx, img.p, himg.at((uint64_t)sit * slots * WH * d.iesize),
                                     (uint64_t)nimg * WH * d.iesize, d.comp->v()), "upload");
                    const void *pdp = lplh ? pd.p : pd.at((uint64_t)sit * Pc * M * PDB);
                    const uint32_t npd = lplh ? (uint32_t)d.pd_all.size() : (uint32_t)(Pc * M);
                    auto slab_launch = [&](int64_t j) {
                        const auto [y0, ny] = extent(j);
                        xpr_launch L = d.launch((int32_t)y0, (int32_t)(y0 + ny), origin, go_.vx, (uint32_t)d.Hd, 0,
                                                (uint32_t)(lplh ? slots : Pc), 0);
                        if (lplh) {
                            L.list_mvp = (const uint16_t *)lm.at((uint64_t)sit * slots * M * 2);
                            L.list_img = (const uint16_t *)li.at((uint64_t)sit * slots * M * 2);
                            L.n_list = (uint32_t)(nimg * M);
                        }
                        return L;
                    };
                    // ---- forward over the slabs, ascending (reconstruction_lpla.hpp:86-103)
                    if (!first) {
                        if (lplh) check(xpr_fill_u32(d.ctx, sum.p, 0u, (uint64_t)slots * WH, d.comp->v()), "fill");
                        for (int64_t j = 0; j < nslab; ++j) {
                            SlabBuf &b = acquire(j);
                            xpr_launch L = slab_launch(j);
                            check(xpr_forward(d.ctx, b.mem.as<float>(), sum.as<uint32_t>(), (const xpr_projdata *)pdp,
                                              npd, &L, d.comp->v()), "forward");
                            b.used.record(*d.comp);
                            b.used_rec = true;
                            stats_.pairs += (uint64_t)extent(j).second * W * W * nimg;
                        }
                    }
                    // ---- error
                    const int mode = lplh ? (first ? XPR_ERROR_FIRST_1C : XPR_ERROR_1C) : XPR_ERROR_STD;
                    check(xpr_error(d.ctx, img.p, d.idt, sum.as<uint32_t>(), sep ? ratio.p : sum.p, d.rdt,
                                    (uint64_t)nimg * WH, weight, mode, 0, nullptr, d.comp->v()), "error");
                    // ---- backward over the slabs, descending
                    for (int64_t j = nslab - 1; j >= 0; --j) {
                        SlabBuf &b = acquire(j);
                        xpr_launch L = slab_launch(j);
                        L.nan_skip = lplh ? 1 : 0;
                        check(xpr_backward(d.ctx, b.mem.as<float>(), sep ? ratio.p : sum.p, d.rdt,
                                           (const xpr_projdata *)pdp, npd, &L, d.comp->v()), "backward");
                        b.used.record(*d.comp);
                        b.used_rec = true;
                        b.dirty = true;
                        stats_.pairs += (uint64_t)extent(j).second * W * W * nimg;
                    }
                    if (!lplh) check(xpr_fill_u32(d.ctx, sum.p, 0u, (uint64_t)slots * WH, d.comp->v()), "fill");
                    stats_.subiterations++;
                }
                weight *= p.weight_factor;
            }
            for (auto &b : bufs)
                if (b->slab >= 0 && b->dirty) write_back(*b);
            d.comp->sync();
            d.up->sync();
            d.down->sync();
        }
        stats_.seconds_iterations = now() - t1;
        std::cout << "Ok" << std::endl;
        par_memcpy(vout, hvol.p, N * 4);
        if (d.write) d.save_layers(p, vout, 0, Hv);
        stats_.seconds_total = now() - t0;
        return;
    }

    if (p.method == Method::method_2) {
        // reconstruction_chunk.hpp:14: 98 % of the usable device memory; CUDA has no
        // per-allocation ceiling, so the planner's max-allocation bound is the same figure
        const uint64_t avail = (uint64_t)((double)d.available() * 0.98);
        std::vector<Chunk> chunks;
        if (!plan_chunks(gp_, go_, d.pd_all, avail, avail, p.overlap_fct, &chunks))
            throw std::runtime_error("Not enough GPU memory for the chunk division");
        std::cout << "Chunks : ";
        for (const auto &c : chunks) std::cout << " [" << c.vOffset << "-" << c.vOffset + c.vSize << "],";
        std::cout << std::endl;
        // layers no chunk reconstructs are NaN
        {
            std::vector<char> covered((size_t)Hv, 0);
            for (const auto &c : chunks)
                for (int64_t l = c.vOffset; l < c.vOffset + c.vSize && l < Hv; ++l)
                    if (l >= 0 && c.vSize > 0 && c.iSize > 0) covered[(size_t)l] = 1;
            for (int64_t l = 0; l < Hv; ++l)
                if (!covered[(size_t)l]) std::fill(vout + (uint64_t)l * W * W, vout + (uint64_t)(l + 1) * W * W, NAN);
        }
        const bool sep = d.rdt != XPR_F32;
        PinBuf himg(d.ctx, (uint64_t)(S * Pc) * WH * d.iesize);
        std::cout << "Pre-processing images..." << std::flush;
        d.preprocess(p, [&](int64_t i, const void *dimg) {
            if (i / S >= Pc) return;
            check_cuda(cudaMemcpyAsync(himg.at((uint64_t)((i % S) * Pc + i / S) * WH * d.iesize), dimg, WH * d.iesize,
                                       cudaMemcpyDeviceToHost, d.comp->s), "copy");
        });
        std::cout << "Ok." << std::endl;
        const std::vector<xpr_projdata> spd = d.subset_projdata();
        DevBuf pd(d.ctx, spd.size() * PDB);
        check(xpr_upload(d.ctx, pd.p, spd.data(), spd.size() * PDB, d.comp->v()), "upload");
        std::cout << "Processing chunks :" << std::endl;
        const double t1 = now();
        for (const Chunk &c : chunks) {
            if (c.vSize <= 0 || c.iSize <= 0) continue;
            std::cout << "[" << c.vOffset << "-" << c.vOffset + c.vSize << "]... " << std::flush;
            const int64_t y0 = c.vOffset - c.vPadTop, ny = c.vPadTop + c.vSize + c.vPadBot;
            const uint64_t rows = (uint64_t)c.iSize, cw = (uint64_t)d.Wd * rows;
            DevBuf slab(d.ctx, (uint64_t)ny * W * W * 4);
            DevBuf img(d.ctx, (uint64_t)Pc * cw * d.iesize), sum(d.ctx, (uint64_t)Pc * cw * 4);
            DevBuf ratio = sep ? DevBuf(d.ctx, (uint64_t)Pc * cw * d.rsize) : DevBuf();
            check(xpr_fill_u32(d.ctx, slab.p, 0x3f800000u, (uint64_t)ny * W * W, d.comp->v()), "fill");
            check(xpr_fill_u32(d.ctx, sum.p, Impl::first_sums(p), (uint64_t)Pc * cw, d.comp->v()), "fill");
            if (!p.resume.empty()) {
                // the chunk's layers with their padding from the stack (a continuous run's
                // padding layers are the chunk's own and are not saved, so a resumed chunk
                // starts its padding from the neighbouring chunks' saved layers)
                std::vector<float> init((size_t)ny * W * W);
                d.load_layers(p, init.data(), y0, y0 + ny);
                check(xpr_upload(d.ctx, slab.p, init.data(), init.size() * 4, d.comp->v()), "upload");
                d.comp->sync();
            }
            float weight = d.start_weight(p);
            d.skip_jitter(p, go_);
            for (int64_t mit = p.first_iteration; mit < p.it; ++mit) {
                for (int64_t sit = 0; sit < S; ++sit) {
                    // the chunk's detector-row window of this sub-iteration's images
                    for (int64_t k = 0; k < Pc; ++k)
                        check(xpr_upload(d.ctx, img.at((uint64_t)k * cw * d.iesize),
                                         himg.at(((uint64_t)(sit * Pc + k) * WH + (uint64_t)c.iOffset * d.Wd) * d.iesize),
                                         cw * d.iesize, d.comp->v()), "upload");
                    d.jittered_origin(go_, origin);
                    xpr_launch L = d.launch((int32_t)y0, (int32_t)(y0 + ny), origin, go_.vx, (uint32_t)rows,
                                            (int32_t)c.iOffset, (uint32_t)Pc, 0);
                    const bool first = Impl::skips_forward(p, mit, sit);
                    check(xpr_subiteration(d.ctx, slab.as<float>(), sum.as<uint32_t>(), img.p, d.idt,
                                           sep ? ratio.p : sum.p, d.rdt,
                                           (const xpr_projdata *)pd.at((uint64_t)sit * Pc * M * PDB), (uint32_t)(Pc * M),
                                           &L, weight, first ? 1 : 0, nullptr, d.comp->v()), "sub-iteration");
                    stats_.subiterations++;
                    stats_.pairs += (uint64_t)(first ? 1 : 2) * ny * W * W * Pc;
                }
                weight *= p.weight_factor;
            }
            d.download_host(vout + (uint64_t)c.vOffset * W * W, slab.at((uint64_t)c.vPadTop * W * W * 4),
                            (uint64_t)c.vSize * W * W * 4);
            if (d.write) d.save_layers(p, vout + (uint64_t)c.vOffset * W * W, c.vOffset, c.vOffset + c.vSize);
            std::cout << "Done." << std::endl;
        }
        stats_.seconds_iterations = now() - t1;
        stats_.seconds_total = now() - t0;
        return;
    }
    throw std::runtime_error("unsupported method");
}

void Engine::simulate()
{
    Impl &d = *d_;
    const Params &p = p_;
    const int64_t W = d.W, Hv = d.Hv, S = d.S, Pc = d.Pc, M = d.M;
    const uint64_t N = d.N, WH = d.WH;
    const int samples = 32;
    // the volume to re-project: the saved layers (reconstruction.hpp:114), / samples,
    // cylinder mask of radius W/2 - 1 (reconstruction.hpp:115-122)
    std::vector<float> vol(N);
    for (int64_t l = 0; l < Hv; ++l) {
        uint32_t w = 0, h = 0;
        std::vector<float> layer = tiff_read_f32(layer_path(p.output, l), &w, &h);
        if (w != (uint32_t)W || h != (uint32_t)W) throw std::runtime_error("layer size mismatch: " + layer_path(p.output, l));
        for (auto &v : layer) v /= (float)samples;
        for (int64_t j = 0; j < W; ++j)
            for (int64_t i = 0; i < W; ++i)
                if (std::sqrt(std::pow((float)i - (float)W * 0.5f, 2.0f) + std::pow((float)j - (float)W * 0.5f, 2.0f)) >=
                    (float)W * 0.5f - 1.0f)
                    layer[(size_t)(j * W + i)] = 0.0f;
        std::memcpy(vol.data() + (size_t)l * W * W, layer.data(), sizeof(float) * W * W);
    }
    const size_t PDB = sizeof(xpr_projdata);
    const std::vector<xpr_projdata> spd = d.subset_projdata();
    DevBuf pd(d.ctx, spd.size() * PDB), dvol(d.ctx, N * 4), sum(d.ctx, (uint64_t)Pc * WH * 4);
    check(xpr_upload(d.ctx, pd.p, spd.data(), spd.size() * PDB, d.comp->v()), "upload");
    check(xpr_upload(d.ctx, dvol.p, vol.data(), N * 4, d.comp->v()), "upload");
    std::vector<uint32_t> hs((size_t)(Pc * WH));
    std::vector<float> img(WH);
    float origin[3];
    for (int64_t sit = 0; sit < S; ++sit) {
        check(xpr_fill_u32(d.ctx, sum.p, 0u, (uint64_t)Pc * WH, d.comp->v()), "fill");
        for (int m = 0; m < samples; ++m) {
            // setOrigin(orig, {vx, vx, vx}) (reconstruction.hpp:106)
            d.jittered_origin(go_, origin);
            xpr_launch L = d.launch(0, (int32_t)Hv, origin, go_.vx, (uint32_t)d.Hd, 0, (uint32_t)Pc, 0);
            check(xpr_forward(d.ctx, dvol.as<float>(), sum.as<uint32_t>(),
                              (const xpr_projdata *)pd.at((uint64_t)sit * Pc * M * PDB), (uint32_t)(Pc * M), &L,
                              d.comp->v()), "forward");
        }
        check(xpr_download(d.ctx, hs.data(), sum.p, hs.size() * 4, d.comp->v()), "download");
        d.comp->sync();
        for (int64_t k = 0; k < Pc; ++k) {
            for (uint64_t q = 0; q < WH; ++q) img[q] = (float)hs[(size_t)(k * WH + q)] / 4194304.0f;  // FIXED_TO_FLOAT
            tiff_write_f32(proj_path(p.proj_output, sit + k * S), img.data(), (uint32_t)d.Wd, (uint32_t)d.Hd);
        }
    }
}

}  // namespace xpr
