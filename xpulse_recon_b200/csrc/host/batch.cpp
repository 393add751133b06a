// batch.cpp -- xpr_batch: many independent naive reconstructions advanced in lock-step.
//
// Each problem is the sub-iteration loop of reconstruction_n.hpp:27-88 (volume 1.0,
// the first sub-iteration without forward, std::mt19937 origin jitter, weight *=
// weight_factor per main iteration).  The batch turns "sub-iteration k of every
// problem" into three persistent launches -- forward, error, backward -- whose CTAs
// claim work units (a brick x a projection run) from one list spanning all problems,
// so small problems share the GPU instead of each leaving most SMs idle, and a whole
// run is a fixed sequence of launches that a CUDA graph captures once.
//
// Results do not depend on the batch: the forward sums are integers (atomic order is
// irrelevant) and each voxel's backward sum runs over its projections in order inside
// one thread, whatever the brick shape or the split of projection runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "batch_plan.h"

namespace {

constexpr uint32_t kOneBits = 0x3f800000u;  // 1.0f

struct StepPlan {
    size_t fwd_off = 0, err_off = 0, bwd_off = 0;  // byte offsets in the work-list buffer
    int n_fwd = 0, n_err = 0, n_bwd = 0;
    uint32_t fwd_units = 0, bwd_units = 0;
    uint64_t max_n = 0;
};

// tuned schedules, per batch shape
using ShapeKey = std::tuple<int, int, int, std::vector<uint64_t>>;
std::mutex g_tune_mu;
std::map<ShapeKey, std::tuple<int, int, int, double>> g_tuned;  // splits, layers, column, step ms

}  // namespace

struct xpr_batch {
    xpr_ctx *ctx = nullptr;
    const xpr::DeviceInfo *di = nullptr;
    std::vector<xpr::PlannedProblem> probs;
    xpr_batch_opts opts{};
    uint32_t steps = 0;
    void *scratch = nullptr;               // sums and ratios of every problem
    uint32_t *tickets = nullptr;           // [0, 2): forward, [2, 4): backward
    void *lists = nullptr;                 // work lists of every step
    size_t lists_bytes = 0;
    xpr::BatchFillItem *fills = nullptr;   // [0, n): volumes <- 1.0, [n, 2n): sums <- 0, [2n, 3n): ratios <- 0
    uint64_t max_vol = 0, max_pix = 0, max_ratio_words = 0;
    std::vector<StepPlan> plan;
    int splits = 1, layers = 8, column = 16, ctas = 0;
    unsigned grid_fwd = 0, grid_bwd = 0;   // persistent CTAs of the forward / backward launches
    double tuned_ms = 0.0;
    cudaStream_t capture = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

int fail(int code, const char *msg) { return xpr::set_last_error(code, "%s", msg); }
int cuda_fail(cudaError_t e, const char *what)
{
    return xpr::set_last_error(XPR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// persistent CTAs for a launch kind (0 forward, 1 backward): the occupancy limit per SM
// (or the requested number below it) on every SM
unsigned grid_of(const xpr_batch *b, int kind)
{
    const int occ = xpr::batched_ctas_per_sm(kind, b->opts.arith, b->opts.storage, kind == 0 ? b->layers : b->column);
    const int per_sm = b->ctas > 0 ? std::min(b->ctas, std::max(occ, 1)) : std::max(occ, 1);
    return (unsigned)(b->di->sm_count * per_sm);
}

int build_lists(xpr_batch *b, int splits, int layers, int column, cudaStream_t s)
{
    std::vector<char> host;
    b->plan.assign(b->steps, StepPlan{});
    auto append = [&](const void *p, size_t bytes) {
        const size_t off = (host.size() + 15) & ~(size_t)15;
        host.resize(off + bytes);
        std::memcpy(host.data() + off, p, bytes);
        return off;
    };
    xpr::StepItems it;
    for (uint32_t k = 0; k < b->steps; ++k) {
        StepPlan &P = b->plan[k];
        it.clear();
        for (const auto &pp : b->probs)
            if (k < pp.steps() && !xpr::add_step_items(pp, k, splits, layers, column, b->opts.image_storage, &it))
                return fail(XPR_ERR_UNSUPPORTED, "batch step exceeds 2^31 work units");
        P.n_fwd = (int)it.fwd.size();
        P.n_err = (int)it.err.size();
        P.n_bwd = (int)it.bwd.size();
        P.fwd_units = it.fwd_units;
        P.bwd_units = it.bwd_units;
        P.max_n = it.max_n;
        if (!it.fwd.empty()) P.fwd_off = append(it.fwd.data(), it.fwd.size() * sizeof(it.fwd[0]));
        if (!it.err.empty()) P.err_off = append(it.err.data(), it.err.size() * sizeof(it.err[0]));
        if (!it.bwd.empty()) P.bwd_off = append(it.bwd.data(), it.bwd.size() * sizeof(it.bwd[0]));
    }
    if (host.size() > b->lists_bytes) {
        if (b->lists) xpr_free(b->ctx, b->lists);
        b->lists = nullptr;
        b->lists_bytes = 0;
        if (int rc = xpr_alloc(b->ctx, host.size(), &b->lists)) return rc;
        b->lists_bytes = host.size();
    }
    if (!host.empty()) {
        const cudaError_t e = cudaMemcpyAsync(b->lists, host.data(), host.size(), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_fail(e, "work-list upload");
        const cudaError_t e2 = cudaStreamSynchronize(s);  // `host` is pageable and local
        if (e2 != cudaSuccess) return cuda_fail(e2, "work-list upload");
    }
    b->splits = splits;
    b->layers = layers;
    b->column = column;
    b->grid_fwd = grid_of(b, 0);
    b->grid_bwd = grid_of(b, 1);
    // a new schedule invalidates a captured run
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    return XPR_OK;
}


cudaError_t enqueue_forward(xpr_batch *b, uint32_t k, cudaStream_t s)
{
    const StepPlan &P = b->plan[k];
    if (!P.n_fwd) return cudaSuccess;
    return xpr::launch_forward_batched((const xpr::BatchFwdItem *)((char *)b->lists + P.fwd_off), P.n_fwd,
                                       P.fwd_units, b->tickets, b->opts.arith, b->layers, b->grid_fwd, s);
}

cudaError_t enqueue_backward(xpr_batch *b, uint32_t k, cudaStream_t s)
{
    const StepPlan &P = b->plan[k];
    if (!P.n_bwd) return cudaSuccess;
    return xpr::launch_backward_batched((const xpr::BatchBwdItem *)((char *)b->lists + P.bwd_off), P.n_bwd,
                                        P.bwd_units, b->tickets + 2, b->opts.arith, b->opts.storage, b->column,
                                        b->grid_bwd, s);
}

cudaError_t enqueue_step(xpr_batch *b, uint32_t k, cudaStream_t s)
{
    const StepPlan &P = b->plan[k];
    cudaError_t e = enqueue_forward(b, k, s);
    if (e == cudaSuccess && P.n_err)
        e = xpr::launch_error_batched((const xpr::BatchErrItem *)((char *)b->lists + P.err_off), P.n_err,
                                      b->opts.image_storage, b->opts.storage, P.max_n, *b->di, s);
    if (e == cudaSuccess) e = enqueue_backward(b, k, s);
    return e;
}

cudaError_t enqueue_fill(xpr_batch *b, int which, cudaStream_t s)
{
    const int n = (int)b->probs.size();
    const uint64_t mx = which == 0 ? b->max_vol : (which == 1 ? b->max_pix : b->max_ratio_words);
    return xpr::launch_fill_batched(b->fills + (size_t)which * n, n, mx, *b->di, s);
}

cudaError_t enqueue_run(xpr_batch *b, cudaStream_t s)
{
    cudaError_t e = cudaSuccess;
    if (b->opts.init_volume) e = enqueue_fill(b, 0, s);
    for (uint32_t k = 0; k < b->steps && e == cudaSuccess; ++k) e = enqueue_step(b, k, s);
    return e;
}

// time `fn` (already warmed) on stream s, in ms
template <typename F>
float time_ms(cudaStream_t s, F &&fn)
{
    cudaEvent_t a, z;
    cudaEventCreate(&a);
    cudaEventCreate(&z);
    fn();  // warm-up
    cudaEventRecord(a, s);
    fn();
    cudaEventRecord(z, s);
    cudaEventSynchronize(z);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, z);
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    return ms;
}

// Candidate schedules, timed on the batch's own data: the forward of step 1 (sums are
// cleared after) for each forward brick (8 layers, and 16 in the STRICT contract) and
// projection-run split, the backward of step 0 against zero ratios for each column length.  exp(0 / count) is exactly 1, so a voxel is unchanged
// unless no projection of step 0 reaches it (count 0), and those voxels become NaN in
// step 0 of the run as well.
int autotune(xpr_batch *b, cudaStream_t s)
{
    uint32_t max_e = 0;
    std::vector<uint64_t> shape;
    for (const auto &pp : b->probs) {
        const xpr_batch_problem &p = pp.p;
        max_e = std::max(max_e, xpr::entries_of(p));
        shape.insert(shape.end(), {p.vwidth, p.vheight, p.det_w, p.det_h, p.per_subset, p.modules});
    }
    const ShapeKey key{b->opts.arith, b->opts.storage, b->opts.image_storage, shape};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            b->tuned_ms = std::get<3>(it->second);
            return build_lists(b, std::get<0>(it->second), std::get<1>(it->second), std::get<2>(it->second), s);
        }
    }
    int best_s = b->splits, best_l = b->layers, best_c = b->column;
    float best_f = 0.0f, best_b = 0.0f;
    if (b->steps > 1) {
        bool first = true;
        for (int ly : {8, 16}) {
            if (!xpr::forward_layers_ok(b->opts.arith, ly)) continue;
            for (int sp : {1, 2, 4, 8, 16}) {
                if (sp > 1 && (uint32_t)sp > xpr::div_up(max_e, 4)) break;
                if (int rc = build_lists(b, sp, ly, b->column, s)) return rc;
                const float ms = time_ms(s, [&] {
                    enqueue_forward(b, 1, s);
                    enqueue_fill(b, 1, s);
                });
                if (first || ms < best_f) {
                    best_f = ms;
                    best_s = sp;
                    best_l = ly;
                }
                first = false;
            }
        }
    }
    cudaError_t e = enqueue_fill(b, 2, s);
    if (e != cudaSuccess) return cuda_fail(e, "autotune");
    bool first = true;
    for (int cb : {16, 8}) {
        if (int rc = build_lists(b, best_s, best_l, cb, s)) return rc;
        const float ms = time_ms(s, [&] { enqueue_backward(b, 0, s); });
        if (first || ms < best_b) {
            best_b = ms;
            best_c = cb;
        }
        first = false;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "autotune");
    b->tuned_ms = (double)best_f + (double)best_b;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[key] = std::make_tuple(best_s, best_l, best_c, b->tuned_ms);
    }
    return build_lists(b, best_s, best_l, best_c, s);
}

void release(xpr_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->capture) cudaStreamDestroy(b->capture);
    if (b->lists) xpr_free(b->ctx, b->lists);
    if (b->scratch) xpr_free(b->ctx, b->scratch);
    delete b;
}

}  // namespace

extern "C" {

int xpr_batch_create(xpr_ctx *ctx, const xpr_batch_problem *problems, uint32_t n, const xpr_batch_opts *opts,
                     void *stream, xpr_batch **out)
{
    if (!out) return fail(XPR_ERR_INVALID, "xpr_batch_create: out is NULL");
    *out = nullptr;
    const xpr::DeviceInfo *di = xpr::context_device(ctx);
    if (!di) return XPR_ERR_INVALID;
    if (!problems || n == 0) return fail(XPR_ERR_INVALID, "xpr_batch_create: no problems");
    if (n > 65535) return fail(XPR_ERR_UNSUPPORTED, "xpr_batch_create: more than 65535 problems");
    xpr_batch_opts o{};
    if (opts) o = *opts;
    if (o.arith != XPR_ARITH_STRICT && o.arith != XPR_ARITH_FAST) return fail(XPR_ERR_INVALID, "unknown arith");
    if (o.storage != XPR_F32 && o.storage != XPR_BF16 && o.storage != XPR_F16)
        return fail(XPR_ERR_INVALID, "unknown storage dtype");
    if (!o.image_storage_set) o.image_storage = o.storage;
    if (o.image_storage != XPR_F32 && o.image_storage != XPR_BF16 && o.image_storage != XPR_F16)
        return fail(XPR_ERR_INVALID, "unknown image storage dtype");
    if (o.bwd_column != 0 && o.bwd_column != 8 && o.bwd_column != 16)
        return fail(XPR_ERR_INVALID, "bwd_column must be 0, 8 or 16");
    if (o.fwd_layers != 0 && !xpr::forward_layers_ok(o.arith, o.fwd_layers))
        return fail(XPR_ERR_INVALID, "fwd_layers must be 0 or 8 (FAST), 0, 8 or 16 (STRICT)");
    cudaError_t e = xpr::prepare_device_kernels();
    if (e != cudaSuccess) return cuda_fail(e, "xpr_batch_create");

    xpr_batch *b = new xpr_batch();
    b->ctx = ctx;
    b->di = di;
    b->opts = o;
    b->ctas = o.ctas_per_sm;
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint64_t scratch_bytes = 0;
    const int layers = o.fwd_layers ? o.fwd_layers : (o.arith == XPR_ARITH_STRICT ? 16 : 8);
    uint64_t total_bricks = 0;
    uint32_t max_e = 0;
    b->probs.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        const xpr_batch_problem &p = problems[i];
        if (const char *m = xpr::plan_problem(p, o.arith, &b->probs[i])) {
            release(b);
            return xpr::set_last_error(XPR_ERR_INVALID, "xpr_batch_create: problem %u: %s", i, m);
        }
        b->steps = std::max(b->steps, p.it * p.sit);
        const uint64_t npix = b->probs[i].npix();
        scratch_bytes += ((npix * 4 + 255) & ~255ull) + ((npix * xpr::dtype_size(o.storage) + 255) & ~255ull);
        b->max_vol = std::max<uint64_t>(b->max_vol, (uint64_t)p.vwidth * p.vheight * p.vwidth);
        b->max_pix = std::max(b->max_pix, npix);
        b->max_ratio_words = std::max<uint64_t>(b->max_ratio_words, xpr::div_up(npix * xpr::dtype_size(o.storage), 4));
        total_bricks += xpr::div_up(p.vwidth, xpr::forward_brick(0, layers)) *
                        xpr::div_up(p.vwidth, xpr::forward_brick(2, layers)) *
                        xpr::div_up(p.vheight, xpr::forward_brick(1, layers));
        max_e = std::max(max_e, xpr::entries_of(p));
    }
    scratch_bytes += 256 + 3 * sizeof(xpr::BatchFillItem) * n;
    if (int rc = xpr_alloc(ctx, scratch_bytes, &b->scratch)) {
        release(b);
        return rc;
    }
    char *q = (char *)b->scratch;
    b->tickets = (uint32_t *)q;
    q += 256;
    b->fills = (xpr::BatchFillItem *)q;
    q += ((3 * sizeof(xpr::BatchFillItem) * n + 255) & ~(size_t)255);
    std::vector<xpr::BatchFillItem> fills(3 * (size_t)n);
    for (uint32_t i = 0; i < n; ++i) {
        xpr::PlannedProblem &pp = b->probs[i];
        const xpr_batch_problem &p = pp.p;
        const uint64_t npix = pp.npix();
        pp.sums = (uint32_t *)q;
        q += (npix * 4 + 255) & ~255ull;
        pp.ratio = q;
        q += (npix * xpr::dtype_size(o.storage) + 255) & ~255ull;
        fills[i] = {(uint32_t *)p.vol, (uint64_t)p.vwidth * p.vheight * p.vwidth, kOneBits, 0};
        fills[n + i] = {pp.sums, npix, 0u, 0};
        fills[2 * n + i] = {(uint32_t *)pp.ratio, xpr::div_up(npix * xpr::dtype_size(o.storage), 4), 0u, 0};
    }
    if ((e = cudaMemsetAsync(b->tickets, 0, 256, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b->fills, fills.data(), fills.size() * sizeof(fills[0]), cudaMemcpyHostToDevice, s)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        release(b);
        return cuda_fail(e, "xpr_batch_create");
    }
    // default schedule: 16-layer forward bricks in the STRICT contract (its per-column work
    // spread over more voxels), 8 in FAST; split projection runs only when the batch has too
    // few bricks to fill the GPU (3 waves of the forward's resident CTAs)
    int splits = o.fwd_splits;
    if (splits <= 0) {
        const uint64_t target = (uint64_t)di->sm_count *
                                std::max(1, xpr::batched_ctas_per_sm(0, o.arith, o.storage, layers)) * 3;
        splits = total_bricks >= target
                     ? 1
                     : (int)std::min<uint64_t>(xpr::div_up(target, total_bricks), xpr::div_up(max_e, 4));
        splits = std::max(splits, 1);
    }
    const int column = o.bwd_column ? o.bwd_column : 16;
    if (int rc = build_lists(b, splits, layers, column, s)) {
        release(b);
        return rc;
    }
    if (o.autotune && o.fwd_splits <= 0 && o.fwd_layers == 0 && o.bwd_column == 0) {
        if (int rc = autotune(b, s)) {
            release(b);
            return rc;
        }
    }
    if ((e = cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking)) != cudaSuccess) {
        release(b);
        return cuda_fail(e, "xpr_batch_create");
    }
    *out = b;
    return XPR_OK;
}

uint32_t xpr_batch_steps(const xpr_batch *b) { return b ? b->steps : 0u; }

int xpr_batch_step(xpr_batch *b, uint32_t step, void *stream)
{
    if (!b) return fail(XPR_ERR_INVALID, "xpr_batch_step: NULL batch");
    if (step >= b->steps) return fail(XPR_ERR_INVALID, "xpr_batch_step: step out of range");
    if (!xpr::context_device(b->ctx)) return XPR_ERR_INVALID;
    xpr::Range nvtx("xpr.batch_step");
    const cudaError_t e = enqueue_step(b, step, reinterpret_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "xpr_batch_step");
}

int xpr_batch_run(xpr_batch *b, void *stream)
{
    if (!b) return fail(XPR_ERR_INVALID, "xpr_batch_run: NULL batch");
    if (!xpr::context_device(b->ctx)) return XPR_ERR_INVALID;
    xpr::Range nvtx("xpr.batch_run");
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!b->opts.use_graph) {
        const cudaError_t e = enqueue_run(b, s);
        return e == cudaSuccess ? XPR_OK : cuda_fail(e, "xpr_batch_run");
    }
    if (!b->exec) {
        cudaError_t e = cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_fail(e, "xpr_batch_run: capture");
        const cudaError_t ee = enqueue_run(b, b->capture);
        e = cudaStreamEndCapture(b->capture, &b->graph);
        if (ee != cudaSuccess) return cuda_fail(ee, "xpr_batch_run: capture");
        if (e != cudaSuccess) return cuda_fail(e, "xpr_batch_run: capture");
        e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            return cuda_fail(e, "xpr_batch_run: instantiate");
        }
    }
    const cudaError_t e = cudaGraphLaunch(b->exec, s);
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "xpr_batch_run: graph launch");
}

int xpr_batch_schedule(const xpr_batch *b, int32_t *fwd_splits, int32_t *fwd_layers, int32_t *bwd_column,
                       int32_t *ctas_per_sm, double *tuned_ms)
{
    if (!b) return fail(XPR_ERR_INVALID, "xpr_batch_schedule: NULL batch");
    if (fwd_splits) *fwd_splits = b->splits;
    if (fwd_layers) *fwd_layers = b->layers;
    if (bwd_column) *bwd_column = b->column;
    if (ctas_per_sm) *ctas_per_sm = (int32_t)(b->grid_fwd / (unsigned)b->di->sm_count);
    if (tuned_ms) *tuned_ms = b->tuned_ms;
    return XPR_OK;
}

int xpr_batch_destroy(xpr_batch *b)
{
    if (!b) return XPR_OK;
    xpr::context_device(b->ctx);  // its device current for the frees (which wait for its work)
    release(b);
    return XPR_OK;
}

}  // extern "C"
