// serve.cpp -- xpr_server: a request loop with continuous batching.
//
// Three host threads drive three CUDA streams:
//   io thread       admission (first come, first served, by device-memory budget),
//                   raw projections through a pinned ring to the device, -log /
//                   normalise into the storage type in subset-major order
//                   (dataset.hpp:133-140), volume set to 1.0
//   download thread the finished volume back to the caller through a second pinned
//                   ring, then the request's memory freed
//   compute thread  one tick = sub-iteration k_r of every active request r as one
//                   batched forward, error and backward launch (xpr_batch's kernels)
// A request joins at the first tick after its upload completes and leaves after its
// last sub-iteration, so requests that arrive while others run are served together
// with them.  Each request's arithmetic is that of the naive method alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "batch_plan.h"
#include "hostcopy.h"
#include "params.h"

namespace {

constexpr uint32_t kOneBits = 0x3f800000u;  // 1.0f
constexpr size_t kChunkBytes = 32u << 20;   // pinned upload / download rings: two chunks of this size

double now_s(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

struct Request {
    uint64_t ticket = 0;
    xpr::Params p;
    const float *raw = nullptr;
    bool raw_pinned = false, out_pinned = false;  // page-locked caller buffers: copied without staging
    int64_t P = 0;
    uint32_t W = 0, H = 0;
    float *out = nullptr;
    // derived at submit
    xpr_geom_params gp{};
    xpr_geom_out go{};
    std::vector<float> mod_offset, mod_rpy;
    std::vector<xpr_projdata> pd_sub;  // subset-major: (s * Pc + k) * M + module
    int64_t Pc = 0, S = 0, M = 1;
    uint64_t N = 0, npix = 0, bytes = 0, pairs = 0;
    // device
    void *arena = nullptr;
    float *raw_dev = nullptr;       // the raw images on the device, until the compute thread preprocesses them
    uint64_t raw_bytes = 0;
    int64_t raw_images = 0;         // images uploaded: all P when normalising (min / max over all), else S * Pc
    xpr::PlannedProblem pp;
    cudaEvent_t ready = nullptr, done_ev = nullptr;
    uint32_t step = 0;
    // state
    int state = XPR_REQ_QUEUED;
    int error = 0;
    double submit_s = 0, admit_s = 0, done_s = 0;
};

}  // namespace

struct xpr_server {
    xpr_ctx *ctx = nullptr;
    const xpr::DeviceInfo *di = nullptr;
    xpr_serve_opts opts{};
    size_t esize = 4;   // ratio element bytes
    size_t iesize = 4;  // image element bytes
    std::chrono::steady_clock::time_point t0;
    // state
    std::mutex mu;
    std::condition_variable cv_io, cv_compute, cv_done, cv_dl;
    bool stop = false;
    uint64_t next_ticket = 1;
    std::map<uint64_t, std::unique_ptr<Request>> reqs;
    std::deque<Request *> queue, ready, finishing;
    std::vector<Request *> active;
    uint64_t bytes_in_use = 0, peak_bytes = 0;
    xpr_serve_stats stats{};
    // io resources
    cudaStream_t io = nullptr, comp = nullptr, dl = nullptr;
    void *pinned[2] = {nullptr, nullptr};     // upload ring for callers' pageable images
    void *dl_pinned[2] = {nullptr, nullptr};  // download ring of dl_bytes per chunk
    size_t dl_bytes = 0;
    cudaEvent_t dl_ev[2] = {nullptr, nullptr};
    cudaEvent_t chunk_ev[2] = {nullptr, nullptr};
    size_t chunk_bytes = 0;
    float *minmax = nullptr;  // device {min, max} of the request being prepared (compute thread)
    // compute resources
    uint32_t *tickets = nullptr;
    char *items_host[2] = {nullptr, nullptr};
    char *items_dev[2] = {nullptr, nullptr};
    size_t items_cap = 0;
    cudaEvent_t tick_ev[2] = {nullptr, nullptr};
    unsigned grid_fwd = 0, grid_bwd = 0;
    int layers = 8;  // forward brick layers
    std::thread io_thread, compute_thread, dl_thread;
};

namespace {

int fail(int code, const char *msg) { return xpr::set_last_error(code, "%s", msg); }

using xpr::par_memcpy;

void check_cuda(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// --------------------------------------------------------------------------- io thread
bool ensure_chunks(xpr_server *s, size_t bytes)
{
    if (bytes <= s->chunk_bytes) return true;
    for (int b = 0; b < 2; ++b) {
        if (s->chunk_ev[b]) cudaEventSynchronize(s->chunk_ev[b]);
        if (s->pinned[b]) cudaFreeHost(s->pinned[b]);
        s->pinned[b] = nullptr;
    }
    s->chunk_bytes = 0;
    for (int b = 0; b < 2; ++b)
        if (cudaHostAlloc(&s->pinned[b], bytes, cudaHostAllocDefault) != cudaSuccess) return false;
    // the download ring keeps the size it was made with (the download thread owns it)
    for (int b = 0; b < 2 && !s->dl_pinned[b]; ++b) {
        if (cudaHostAlloc(&s->dl_pinned[b], bytes, cudaHostAllocDefault) != cudaSuccess) return false;
        s->dl_bytes = bytes;
    }
    s->chunk_bytes = bytes;
    return true;
}

// The request's raw images [0, raw_images) to its device buffer on the io stream: one copy
// from a page-locked caller buffer, else through the pinned ring (host copy, then a copy
// to the device, the two overlapped).  Only copies run here: the io stream carries no
// kernel, so the uploads never wait for the compute thread's persistent launches, which
// hold every SM while a tick runs.
void upload_raw(xpr_server *s, Request *r)
{
    const size_t total = (size_t)r->raw_images * r->W * r->H * sizeof(float);
    if (r->raw_pinned) {
        check_cuda(cudaMemcpyAsync(r->raw_dev, r->raw, total, cudaMemcpyHostToDevice, s->io), "upload");
        return;
    }
    int b = 0;
    for (size_t off = 0; off < total; off += s->chunk_bytes, b ^= 1) {
        const size_t n = std::min(s->chunk_bytes, total - off);
        check_cuda(cudaEventSynchronize(s->chunk_ev[b]), "staging");
        par_memcpy(s->pinned[b], (const char *)r->raw + off, n);
        check_cuda(cudaMemcpyAsync((char *)r->raw_dev + off, s->pinned[b], n, cudaMemcpyHostToDevice, s->io),
                   "upload");
        check_cuda(cudaEventRecord(s->chunk_ev[b], s->io), "staging");
    }
}

// The request's device memory (the arena and the raw-image buffer) from the stream-ordered
// pool; on failure neither is kept.  Finished requests free their memory in stream order
// (download and compute streams), so a failed allocation waits for those frees to run and
// tries once more.
cudaError_t alloc_request(xpr_server *s, Request *r)
{
    cudaError_t e = cudaSuccess;
    for (int attempt = 0; attempt < 2; ++attempt) {
        e = cudaMallocAsync(&r->arena, r->bytes, s->io);
        if (e == cudaSuccess) e = cudaMallocAsync((void **)&r->raw_dev, r->raw_bytes, s->io);
        if (e == cudaSuccess) return e;
        cudaGetLastError();  // an allocation failure is not sticky; clear it
        if (r->arena) cudaFreeAsync(r->arena, s->io);
        if (r->raw_dev) cudaFreeAsync(r->raw_dev, s->io);
        r->arena = nullptr;
        r->raw_dev = nullptr;
        if (e != cudaErrorMemoryAllocation) break;
        cudaStreamSynchronize(s->dl);
        cudaStreamSynchronize(s->comp);
        cudaStreamSynchronize(s->io);
    }
    return e;
}

void upload_request(xpr_server *s, Request *r)
{
    char *q = (char *)r->arena;
    auto take = [&](uint64_t bytes) {
        char *p = q;
        q += (bytes + 255) & ~255ull;
        return p;
    };
    float *vol = (float *)take(4 * r->N);
    char *images = take(s->iesize * r->npix * r->S);
    xpr_projdata *pd = (xpr_projdata *)take(sizeof(xpr_projdata) * r->pd_sub.size());
    uint32_t *sums = (uint32_t *)take(4 * r->npix);
    void *ratio = take(s->esize * r->npix);
    check_cuda(cudaMemcpyAsync(pd, r->pd_sub.data(), sizeof(xpr_projdata) * r->pd_sub.size(), cudaMemcpyHostToDevice,
                               s->io), "projdata upload");
    upload_raw(s, r);
    xpr_batch_problem bp{};
    bp.vol = vol;
    bp.images = images;
    bp.projdata = pd;
    bp.det_w = r->W;
    bp.det_h = r->H;
    bp.per_subset = (uint32_t)r->Pc;
    bp.modules = (uint32_t)r->M;
    bp.sit = (uint32_t)r->S;
    bp.it = (uint32_t)r->p.it;
    bp.vwidth = (uint32_t)r->go.vwidth;
    bp.vheight = (uint32_t)r->go.vheight;
    bp.voxel = r->go.vx;
    for (int c = 0; c < 3; ++c) bp.orig[c] = r->go.orig[c];
    bp.seed = r->p.seed;
    bp.weight = r->p.weight;
    bp.weight_factor = r->p.weight_factor;
    if (const char *m = xpr::plan_problem(bp, s->opts.arith, &r->pp)) throw std::runtime_error(m);
    r->pp.sums = sums;
    r->pp.ratio = ratio;
    check_cuda(cudaEventRecord(r->ready, s->io), "event");
}

// The finished volume back to the caller through the download ring (device -> pinned
// on the download stream, pinned -> caller by host threads, the two overlapped), then
// its memory freed.
void finish_request(xpr_server *s, Request *r)
{
    int err = r->error;  // set by the compute thread when a tick failed
    cudaError_t e = cudaEventSynchronize(r->done_ev);
    const size_t total = 4 * r->N;
    const char *src = (const char *)r->pp.p.vol;
    char *dst = (char *)r->out;
    size_t pending[2] = {0, 0}, pending_off[2] = {0, 0};
    int b = 0;
    if (r->out_pinned && e == cudaSuccess) {  // straight into the caller's page-locked buffer
        e = cudaMemcpyAsync(dst, src, total, cudaMemcpyDeviceToHost, s->dl);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->dl);
    }
    for (size_t off = 0; !r->out_pinned && e == cudaSuccess && off < total; off += s->dl_bytes, b ^= 1) {
        const size_t n = std::min(s->dl_bytes, total - off);
        if (pending[b]) {  // drain the chunk that used this buffer two copies ago
            e = cudaEventSynchronize(s->dl_ev[b]);
            if (e == cudaSuccess) par_memcpy(dst + pending_off[b], s->dl_pinned[b], pending[b]);
            pending[b] = 0;
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(s->dl_pinned[b], src + off, n, cudaMemcpyDeviceToHost, s->dl);
        if (e == cudaSuccess) e = cudaEventRecord(s->dl_ev[b], s->dl);
        pending[b] = n;
        pending_off[b] = off;
    }
    for (int k = 0; k < 2; ++k) {
        b ^= 1;
        if (e == cudaSuccess && pending[b]) {
            e = cudaEventSynchronize(s->dl_ev[b]);
            if (e == cudaSuccess) par_memcpy(dst + pending_off[b], s->dl_pinned[b], pending[b]);
        }
        pending[b] = 0;
    }
    if (e != cudaSuccess && !err) err = XPR_ERR_CUDA;
    if (r->arena) cudaFreeAsync(r->arena, s->dl);
    r->arena = nullptr;
    // a finished request keeps only what xpr_serve_poll reports
    std::vector<xpr_projdata>().swap(r->pd_sub);
    r->pp.origin = std::vector<float>();
    r->pp.weight = std::vector<float>();
    std::lock_guard<std::mutex> lk(s->mu);
    s->bytes_in_use -= r->bytes;
    r->done_s = now_s(s->t0);
    r->state = err ? XPR_REQ_FAILED : XPR_REQ_DONE;
    r->error = err;
    if (err) ++s->stats.failed;
    else ++s->stats.completed;
    s->cv_done.notify_all();
    s->cv_io.notify_all();  // memory freed: admission may proceed
}

void dl_loop(xpr_server *s)
{
    xpr::context_device(s->ctx);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        if (!s->finishing.empty()) {
            Request *r = s->finishing.front();
            s->finishing.pop_front();
            lk.unlock();
            finish_request(s, r);
            lk.lock();
            continue;
        }
        if (s->stop && s->queue.empty() && s->ready.empty() && s->active.empty()) break;
        s->cv_dl.wait(lk);
    }
}

void io_loop(xpr_server *s)
{
    xpr::context_device(s->ctx);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        if (!s->queue.empty()) {
            Request *r = s->queue.front();
            const uint64_t resident = s->active.size() + s->ready.size();
            const bool fits = s->bytes_in_use + r->bytes + r->raw_bytes <= s->opts.mem_budget;
            const bool slot = s->opts.max_active == 0 || resident < s->opts.max_active;
            if (fits && slot) {
                s->queue.pop_front();
                s->bytes_in_use += r->bytes + r->raw_bytes;
                s->peak_bytes = std::max(s->peak_bytes, s->bytes_in_use);
                r->admit_s = now_s(s->t0);
                const uint64_t others = s->bytes_in_use - (r->bytes + r->raw_bytes);
                lk.unlock();
                const cudaError_t ae = alloc_request(s, r);
                int err = 0;
                if (ae == cudaSuccess) {
                    try {
                        upload_request(s, r);
                    } catch (const std::exception &) {
                        err = XPR_ERR_CUDA;
                    }
                } else if (ae != cudaErrorMemoryAllocation) {
                    err = XPR_ERR_CUDA;
                }
                lk.lock();
                if (ae == cudaErrorMemoryAllocation) {
                    // the device holds less than the budget allows (memory of other users of
                    // the device, fragmentation): while other requests hold memory, the
                    // request waits at the head of the queue for one of them to release
                    // some; alone on the server it can never fit
                    s->bytes_in_use -= r->bytes + r->raw_bytes;
                    if (s->bytes_in_use > 0) {
                        s->queue.push_front(r);
                        if (s->bytes_in_use >= others) s->cv_io.wait(lk);  // else some was released meanwhile
                        continue;
                    }
                    err = XPR_ERR_OOM;
                    s->bytes_in_use += r->bytes + r->raw_bytes;  // released below with the failure
                }
                if (err) {
                    if (r->arena) cudaFreeAsync(r->arena, s->io);
                    if (r->raw_dev) cudaFreeAsync(r->raw_dev, s->io);
                    r->arena = nullptr;
                    r->raw_dev = nullptr;
                    s->bytes_in_use -= r->bytes + r->raw_bytes;
                    r->state = XPR_REQ_FAILED;
                    r->error = err;
                    r->done_s = now_s(s->t0);
                    ++s->stats.failed;
                    s->cv_done.notify_all();
                } else {
                    s->ready.push_back(r);
                    s->cv_compute.notify_all();
                }
                continue;
            }
        }
        if (s->stop && s->queue.empty()) break;
        s->cv_io.wait(lk);
    }
}

// ---------------------------------------------------------------------- compute thread
// A request joining the batch, on the compute stream ahead of its first tick: the volume
// set to 1.0 (reconstruction_n.hpp:59), then the -log / normalise preprocessing
// (data_loader.hpp:48-101; min / max over every image when normalising) of its raw images
// into the storage type in subset-major order, in one launch; the raw buffer is released.
cudaError_t prepare_on_device(xpr_server *s, Request *r)
{
    const uint64_t WH = (uint64_t)r->W * r->H;
    cudaError_t e = xpr::launch_fill_u32(r->pp.p.vol, kOneBits, r->N, *s->di, s->comp);
    if (e == cudaSuccess && r->p.normalize) {
        e = xpr::launch_fill_u32(s->minmax, 0x7f7fffffu, 1, *s->di, s->comp);  // FLT_MAX (data_loader.hpp:12-13)
        if (e == cudaSuccess) e = xpr::launch_fill_u32(s->minmax + 1, 0x00800000u, 1, *s->di, s->comp);  // FLT_MIN
        if (e == cudaSuccess) e = xpr::launch_minmax(r->raw_dev, (uint64_t)r->P * WH, s->minmax, *s->di, s->comp);
    }
    if (e == cudaSuccess)
        e = xpr::launch_preprocess_reorder(r->raw_dev, const_cast<void *>(r->pp.p.images), s->opts.image_storage, WH,
                                           (uint32_t)(r->S * r->Pc), (uint32_t)r->S, (uint32_t)r->Pc,
                                           r->p.normalize ? 1 : 0, s->minmax, r->p.mlog ? 1 : 0, *s->di, s->comp);
    const cudaError_t f = cudaFreeAsync(r->raw_dev, s->comp);
    r->raw_dev = nullptr;
    return e != cudaSuccess ? e : f;
}

void compute_loop(xpr_server *s)
{
    xpr::context_device(s->ctx);
    xpr::StepItems items;
    uint64_t tick = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // join the requests whose upload completed (preprocessed on this stream first)
        for (auto it = s->ready.begin(); it != s->ready.end();) {
            Request *r = *it;
            if (cudaEventQuery(r->ready) == cudaSuccess) {
                it = s->ready.erase(it);
                const cudaError_t e = prepare_on_device(s, r);
                s->bytes_in_use -= r->raw_bytes;
                s->cv_io.notify_all();  // the raw images' memory released: admission may proceed
                if (e != cudaSuccess) {
                    r->error = XPR_ERR_CUDA;
                    cudaEventRecord(r->done_ev, s->comp);
                    s->finishing.push_back(r);
                    s->cv_dl.notify_all();
                    continue;
                }
                r->state = XPR_REQ_ACTIVE;
                s->active.push_back(r);
            } else {
                ++it;
            }
        }
        if (s->active.empty()) {
            if (s->stop && s->queue.empty() && s->ready.empty()) break;
            s->cv_compute.wait_for(lk, std::chrono::microseconds(s->ready.empty() ? 20000 : 200));
            continue;
        }
        std::vector<Request *> act = s->active;
        lk.unlock();
        // one sub-iteration of every active request
        items.clear();
        uint64_t bricks = 0, max_e = 0, pairs = 0;
        for (Request *r : act) {
            const auto &p = r->pp.p;
            bricks += xpr::div_up(p.vwidth, xpr::forward_brick(0, s->layers)) *
                      xpr::div_up(p.vwidth, xpr::forward_brick(2, s->layers)) *
                      xpr::div_up(p.vheight, xpr::forward_brick(1, s->layers));
            max_e = std::max<uint64_t>(max_e, xpr::entries_of(p));
        }
        const uint64_t target = (uint64_t)s->grid_fwd * 3;  // three waves of the forward's resident CTAs
        const int splits = bricks >= target ? 1 : (int)std::max<uint64_t>(
                                                        1, std::min(xpr::div_up(target, bricks), xpr::div_up(max_e, 4)));
        bool ok = true;
        for (Request *r : act) {
            ok = ok && xpr::add_step_items(r->pp, r->step, splits, s->layers, 16, s->opts.image_storage, &items);
            pairs += r->N * (uint64_t)r->Pc;
        }
        const size_t fb = items.fwd.size() * sizeof(items.fwd[0]), eb = items.err.size() * sizeof(items.err[0]),
                     bb = items.bwd.size() * sizeof(items.bwd[0]);
        const size_t eo = (fb + 255) & ~(size_t)255, bo = eo + ((eb + 255) & ~(size_t)255), need = bo + bb;
        cudaError_t e = cudaSuccess;
        const int h = (int)(tick & 1);
        xpr::Range nvtx("xpr.serve_tick");
        if (ok && need > s->items_cap) {  // grow both buffers (rare): wait for the ticks in flight
            e = cudaStreamSynchronize(s->comp);
            for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
                cudaFreeHost(s->items_host[b]);
                cudaFree(s->items_dev[b]);
                s->items_host[b] = nullptr;
                s->items_dev[b] = nullptr;
                if ((e = cudaHostAlloc((void **)&s->items_host[b], 2 * need, cudaHostAllocDefault)) == cudaSuccess)
                    e = cudaMalloc((void **)&s->items_dev[b], 2 * need);
            }
            s->items_cap = e == cudaSuccess ? 2 * need : 0;
        }
        if (ok && e == cudaSuccess) {
            // the pinned buffer of this parity was last read by the copy of tick - 2
            e = cudaEventSynchronize(s->tick_ev[h]);
            char *hb = s->items_host[h], *db = s->items_dev[h];
            std::memcpy(hb, items.fwd.data(), fb);
            std::memcpy(hb + eo, items.err.data(), eb);
            std::memcpy(hb + bo, items.bwd.data(), bb);
            if (e == cudaSuccess) e = cudaMemcpyAsync(db, hb, need, cudaMemcpyHostToDevice, s->comp);
            if (e == cudaSuccess) e = cudaEventRecord(s->tick_ev[h], s->comp);
            if (e == cudaSuccess && !items.fwd.empty())
                e = xpr::launch_forward_batched((const xpr::BatchFwdItem *)db, (int)items.fwd.size(), items.fwd_units,
                                                s->tickets, s->opts.arith, s->layers, s->grid_fwd, s->comp);
            if (e == cudaSuccess)
                e = xpr::launch_error_batched((const xpr::BatchErrItem *)(db + eo), (int)items.err.size(),
                                              s->opts.image_storage, s->opts.storage, items.max_n, *s->di, s->comp);
            if (e == cudaSuccess)
                e = xpr::launch_backward_batched((const xpr::BatchBwdItem *)(db + bo), (int)items.bwd.size(),
                                                 items.bwd_units, s->tickets + 2, s->opts.arith, s->opts.storage, 16,
                                                 s->grid_bwd, s->comp);
        }
        ++tick;
        lk.lock();
        ++s->stats.ticks;
        s->stats.pairs += pairs;
        std::vector<Request *> left;
        for (Request *r : act) {
            r->step += 1;
            const bool failed = !ok || e != cudaSuccess;
            if (failed || r->step >= r->pp.steps()) {
                if (failed) {
                    r->error = ok ? XPR_ERR_CUDA : XPR_ERR_UNSUPPORTED;
                }
                cudaEventRecord(r->done_ev, s->comp);
                s->finishing.push_back(r);
            } else {
                left.push_back(r);
            }
        }
        s->active = left;  // only this thread changes s->active
        if (!s->finishing.empty()) s->cv_dl.notify_all();
    }
    s->cv_dl.notify_all();
}

// ------------------------------------------------------------------------ submission
bool prepare_request(xpr_server *s, Request *r, std::string *msg)
{
    try {
        r->p = xpr::load_params(*msg);
    } catch (const std::exception &e) {
        *msg = e.what();
        return false;
    }
    if (r->p.method == xpr::Method::hartmann || r->p.method == xpr::Method::ipr) {
        *msg = "the served method is the naive reconstruction";
        return false;
    }
    if (!r->p.seed_set) r->p.seed = std::random_device()();  // as the reference (random jitter)
    xpr::geom_params_from(r->p, r->P, r->W, r->H, &r->gp, &r->mod_offset, &r->mod_rpy);
    r->M = r->p.module_number;
    if (!r->p.angle_list.empty() && (int64_t)r->p.angle_list.size() != r->P) {
        *msg = "The size of the angle list is different from the number of projections";
        return false;
    }
    std::vector<xpr_projdata> all((size_t)(r->P * r->M));
    if (xpr_geometry(&r->gp, r->p.geometry == "fp64" ? 1 : 0, all.data(), &r->go) != XPR_OK) {
        *msg = "geometry";
        return false;
    }
    r->Pc = r->go.concurrent;
    r->S = r->p.sit;
    if (r->Pc < 1 || r->p.it < 1) {
        *msg = "fewer projections than sub-iterations, or it < 1";
        return false;
    }
    r->pd_sub.resize((size_t)(r->S * r->Pc * r->M));
    for (int64_t sb = 0; sb < r->S; ++sb)
        for (int64_t k = 0; k < r->Pc; ++k)
            for (int64_t m = 0; m < r->M; ++m)
                r->pd_sub[(size_t)((sb * r->Pc + k) * r->M + m)] = all[(size_t)((sb + k * r->S) * r->M + m)];
    r->N = (uint64_t)r->go.vwidth * r->go.vheight * r->go.vwidth;
    r->npix = (uint64_t)r->Pc * r->W * r->H;
    auto al = [](uint64_t b) { return (b + 255) & ~255ull; };
    r->bytes = al(4 * r->N) + al(s->iesize * r->npix * r->S) + al(sizeof(xpr_projdata) * r->pd_sub.size()) +
               al(4 * r->npix) + al(s->esize * r->npix);
    r->raw_images = r->p.normalize ? r->P : r->S * r->Pc;
    r->raw_bytes = al((uint64_t)r->raw_images * r->W * r->H * sizeof(float));
    r->pairs = r->N * (uint64_t)r->Pc * (uint64_t)r->S * (uint64_t)r->p.it;
    return true;
}

void release(xpr_server *s)
{
    for (int b = 0; b < 2; ++b) {
        if (s->pinned[b]) cudaFreeHost(s->pinned[b]);
        if (s->chunk_ev[b]) cudaEventDestroy(s->chunk_ev[b]);
        if (s->items_host[b]) cudaFreeHost(s->items_host[b]);
        if (s->items_dev[b]) cudaFree(s->items_dev[b]);
        if (s->tick_ev[b]) cudaEventDestroy(s->tick_ev[b]);
        if (s->dl_pinned[b]) cudaFreeHost(s->dl_pinned[b]);
        if (s->dl_ev[b]) cudaEventDestroy(s->dl_ev[b]);
    }
    for (auto &kv : s->reqs) {
        if (kv.second->ready) cudaEventDestroy(kv.second->ready);
        if (kv.second->done_ev) cudaEventDestroy(kv.second->done_ev);
    }
    if (s->tickets) cudaFree(s->tickets);
    if (s->minmax) cudaFree(s->minmax);
    if (s->io) cudaStreamDestroy(s->io);
    if (s->comp) cudaStreamDestroy(s->comp);
    if (s->dl) cudaStreamDestroy(s->dl);
    delete s;
}

void fill_info(const Request *r, xpr_request_info *info)
{
    info->state = r->state;
    info->error = r->error;
    info->submit_s = r->submit_s;
    info->admit_s = r->admit_s;
    info->done_s = r->done_s;
    info->pairs = r->pairs;
    info->device_bytes = r->bytes + r->raw_bytes;  // the peak: the raw images are held until the request joins
}

}  // namespace

extern "C" {

int xpr_serve_create(xpr_ctx *ctx, const xpr_serve_opts *opts, xpr_server **out)
{
    if (!out) return fail(XPR_ERR_INVALID, "xpr_serve_create: out is NULL");
    *out = nullptr;
    const xpr::DeviceInfo *di = xpr::context_device(ctx);
    if (!di) return XPR_ERR_INVALID;
    xpr_serve_opts o{};
    if (opts) o = *opts;
    if (o.arith != XPR_ARITH_STRICT && o.arith != XPR_ARITH_FAST) return fail(XPR_ERR_INVALID, "unknown arith");
    if (o.storage != XPR_F32 && o.storage != XPR_BF16 && o.storage != XPR_F16)
        return fail(XPR_ERR_INVALID, "unknown storage dtype");
    if (!o.image_storage_set) o.image_storage = o.storage;
    if (o.image_storage != XPR_F32 && o.image_storage != XPR_BF16 && o.image_storage != XPR_F16)
        return fail(XPR_ERR_INVALID, "unknown image storage dtype");
    if (xpr::prepare_device_kernels() != cudaSuccess) return fail(XPR_ERR_CUDA, "xpr_serve_create: kernels");
    xpr_server *s = new xpr_server();
    s->ctx = ctx;
    s->di = di;
    s->esize = o.storage == XPR_F32 ? 4 : 2;
    s->iesize = o.image_storage == XPR_F32 ? 4 : 2;
    s->t0 = std::chrono::steady_clock::now();
    if (o.mem_budget == 0) {
        uint64_t avail = 0;
        xpr_mem_available(ctx, &avail);
        o.mem_budget = (uint64_t)(0.9 * (double)avail);
    }
    s->opts = o;
    cudaError_t e = cudaStreamCreateWithFlags(&s->io, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->comp, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->dl, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        if ((e = cudaEventCreateWithFlags(&s->chunk_ev[b], cudaEventDisableTiming)) == cudaSuccess &&
            (e = cudaEventCreateWithFlags(&s->dl_ev[b], cudaEventDisableTiming)) == cudaSuccess)
            e = cudaEventCreateWithFlags(&s->tick_ev[b], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaMalloc((void **)&s->tickets, 256);
    if (e == cudaSuccess) e = cudaMemset(s->tickets, 0, 256);
    if (e == cudaSuccess) e = cudaMalloc((void **)&s->minmax, 2 * sizeof(float));
    if (e != cudaSuccess || !ensure_chunks(s, kChunkBytes)) {
        release(s);
        return fail(XPR_ERR_CUDA, "xpr_serve_create: streams / staging");
    }
    // 16-layer forward bricks in the STRICT contract (its per-column work spread over more voxels)
    s->layers = o.arith == XPR_ARITH_STRICT ? 16 : 8;
    s->grid_fwd = (unsigned)(di->sm_count * std::max(1, xpr::batched_ctas_per_sm(0, o.arith, o.storage, s->layers)));
    s->grid_bwd = (unsigned)(di->sm_count * std::max(1, xpr::batched_ctas_per_sm(1, o.arith, o.storage, 16)));
    s->io_thread = std::thread(io_loop, s);
    s->compute_thread = std::thread(compute_loop, s);
    s->dl_thread = std::thread(dl_loop, s);
    *out = s;
    return XPR_OK;
}

int xpr_serve_submit(xpr_server *s, const char *json, const float *raw, int64_t count, uint32_t width,
                     uint32_t height, float *vol_out, uint64_t vol_cap, uint64_t *ticket)
{
    if (!s || !raw || !vol_out || !ticket || count <= 0 || width == 0 || height == 0)
        return fail(XPR_ERR_INVALID, "xpr_serve_submit: bad arguments");
    auto r = std::make_unique<Request>();
    r->raw = raw;
    r->P = count;
    r->W = width;
    r->H = height;
    r->out = vol_out;
    std::string msg = json ? json : "{}";
    if (!prepare_request(s, r.get(), &msg)) return xpr::set_last_error(XPR_ERR_PARAM, "xpr_serve_submit: %s", msg.c_str());
    if (r->N > vol_cap)
        return xpr::set_last_error(XPR_ERR_INVALID, "xpr_serve_submit: vol_out holds %llu floats, %llu needed",
                                   (unsigned long long)vol_cap, (unsigned long long)r->N);
    if (r->bytes + r->raw_bytes > s->opts.mem_budget)
        return xpr::set_last_error(XPR_ERR_CAP, "xpr_serve_submit: the request needs %llu device bytes, the budget "
                                                "is %llu", (unsigned long long)(r->bytes + r->raw_bytes),
                                   (unsigned long long)s->opts.mem_budget);
    if (!xpr::context_device(s->ctx)) return XPR_ERR_INVALID;
    auto pinned = [](const void *p) {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeHost;
    };
    r->raw_pinned = pinned(raw) && pinned(raw + (size_t)count * width * height - 1);
    r->out_pinned = pinned(vol_out) && pinned(vol_out + r->N - 1);
    if (cudaEventCreateWithFlags(&r->ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->done_ev, cudaEventDisableTiming) != cudaSuccess)
        return fail(XPR_ERR_CUDA, "xpr_serve_submit: events");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail(XPR_ERR_INVALID, "xpr_serve_submit: the server is stopping");
    r->ticket = s->next_ticket++;
    r->submit_s = now_s(s->t0);
    *ticket = r->ticket;
    s->queue.push_back(r.get());
    s->reqs[r->ticket] = std::move(r);
    ++s->stats.submitted;
    s->cv_io.notify_all();
    return XPR_OK;
}

int xpr_serve_poll(xpr_server *s, uint64_t ticket, xpr_request_info *info)
{
    if (!s || !info) return fail(XPR_ERR_INVALID, "xpr_serve_poll: bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(XPR_ERR_INVALID, "xpr_serve_poll: unknown ticket");
    fill_info(it->second.get(), info);
    return XPR_OK;
}

int xpr_serve_wait(xpr_server *s, uint64_t ticket, double timeout_s, xpr_request_info *info)
{
    if (!s || !info) return fail(XPR_ERR_INVALID, "xpr_serve_wait: bad arguments");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(XPR_ERR_INVALID, "xpr_serve_wait: unknown ticket");
    Request *r = it->second.get();
    auto finished = [&] { return r->state == XPR_REQ_DONE || r->state == XPR_REQ_FAILED; };
    if (timeout_s < 0) s->cv_done.wait(lk, finished);
    else s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), finished);
    fill_info(r, info);
    return XPR_OK;
}

int xpr_serve_stats_get(xpr_server *s, xpr_serve_stats *stats)
{
    if (!s || !stats) return fail(XPR_ERR_INVALID, "xpr_serve_stats_get: bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    *stats = s->stats;
    stats->active = (uint32_t)s->active.size();
    stats->queued = (uint32_t)(s->queue.size() + s->ready.size());
    stats->bytes_in_use = s->bytes_in_use;
    stats->peak_bytes = s->peak_bytes;
    return XPR_OK;
}

int xpr_serve_destroy(xpr_server *s)
{
    if (!s) return XPR_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_io.notify_all();
        s->cv_compute.notify_all();
    }
    s->compute_thread.join();  // returns once nothing is queued, uploading or active
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->cv_io.notify_all();
        s->cv_dl.notify_all();
    }
    s->io_thread.join();
    s->dl_thread.join();
    xpr::context_device(s->ctx);
    cudaStreamSynchronize(s->io);
    cudaStreamSynchronize(s->comp);
    cudaStreamSynchronize(s->dl);
    release(s);
    return XPR_OK;
}

}  // extern "C"
