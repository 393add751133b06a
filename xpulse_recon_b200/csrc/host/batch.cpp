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

#include "../xpr_internal.h"
#include "xpr.h"

namespace {

constexpr uint32_t kOneBits = 0x3f800000u;  // 1.0f

size_t dtype_size(int dt) { return dt == XPR_F32 ? 4 : 2; }

struct StepPlan {
    size_t fwd_off = 0, err_off = 0, bwd_off = 0;  // byte offsets in the work-list buffer
    int n_fwd = 0, n_err = 0, n_bwd = 0;
    uint32_t fwd_units = 0, bwd_units = 0;
    uint64_t max_n = 0;
};

// tuned schedules, per batch shape
using ShapeKey = std::tuple<int, int, std::vector<uint64_t>>;
std::mutex g_tune_mu;
std::map<ShapeKey, std::tuple<int, int, double>> g_tuned;

}  // namespace

struct xpr_batch {
    xpr_ctx *ctx = nullptr;
    const xpr::DeviceInfo *di = nullptr;
    std::vector<xpr_batch_problem> probs;
    xpr_batch_opts opts{};
    uint32_t steps = 0;
    // per problem: origins (3 per step) and weights (1 per step)
    std::vector<std::vector<float>> origin, weight;
    std::vector<xpr::LaunchArgs> base;     // launch args without origin / split
    std::vector<uint32_t *> sums;
    std::vector<void *> ratios;
    void *scratch = nullptr;               // sums and ratios of every problem
    uint32_t *tickets = nullptr;           // [0, 2): forward, [2, 4): backward
    void *lists = nullptr;                 // work lists of every step
    size_t lists_bytes = 0;
    xpr::BatchFillItem *fills = nullptr;   // [0, n): volumes <- 1.0, [n, 2n): sums <- 0, [2n, 3n): ratios <- 0
    uint64_t max_vol = 0, max_pix = 0, max_ratio_words = 0;
    std::vector<StepPlan> plan;
    int splits = 1, column = 16, ctas = 0;
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

uint64_t div_up(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

uint32_t entries_of(const xpr_batch_problem &p) { return p.per_subset * (p.modules ? p.modules : 1u); }

// persistent CTAs for a launch kind (0 forward, 1 backward): the occupancy limit per SM
// (or the requested number below it) on every SM
unsigned grid_of(const xpr_batch *b, int kind)
{
    const int occ = xpr::batched_ctas_per_sm(kind, b->opts.arith, b->opts.storage, b->column);
    const int per_sm = b->ctas > 0 ? std::min(b->ctas, std::max(occ, 1)) : std::max(occ, 1);
    return (unsigned)(b->di->sm_count * per_sm);
}

// per_split (entries per forward work unit, a multiple of the metadata group) for `splits`
uint32_t per_split_for(uint32_t entries, int splits)
{
    const uint32_t g = 4;
    return (uint32_t)div_up(div_up(entries, (uint64_t)std::max(1, splits)), g) * g;
}

int build_lists(xpr_batch *b, int splits, int column, cudaStream_t s)
{
    const int n = (int)b->probs.size();
    std::vector<char> host;
    b->plan.assign(b->steps, StepPlan{});
    const int fbx = xpr::forward_brick(0), fby = xpr::forward_brick(1), fbz = xpr::forward_brick(2);
    const int bbx = xpr::backward_brick(0, column), bby = xpr::backward_brick(1, column),
              bbz = xpr::backward_brick(2, column);
    auto append = [&](const void *p, size_t bytes) {
        const size_t off = (host.size() + 15) & ~(size_t)15;
        host.resize(off + bytes);
        std::memcpy(host.data() + off, p, bytes);
        return off;
    };
    for (uint32_t k = 0; k < b->steps; ++k) {
        StepPlan &P = b->plan[k];
        std::vector<xpr::BatchFwdItem> fw;
        std::vector<xpr::BatchErrItem> er;
        std::vector<xpr::BatchBwdItem> bw;
        for (int i = 0; i < n; ++i) {
            const xpr_batch_problem &p = b->probs[i];
            if (k >= p.it * p.sit) continue;
            const uint32_t s_idx = k % p.sit;
            const uint32_t E = entries_of(p);
            xpr::LaunchArgs a = b->base[i];
            for (int c = 0; c < 3; ++c) a.origin[c] = b->origin[i][3 * k + c];
            const xpr_projdata *pd = p.projdata + (size_t)s_idx * E;
            const uint64_t npix = (uint64_t)p.per_subset * p.det_w * p.det_h;
            if (k > 0) {
                xpr::BatchFwdItem f{};
                f.a = a;
                f.a.per_split = per_split_for(E, splits);
                f.vol = p.vol;
                f.sum = b->sums[i];
                f.pd = pd;
                f.bricks_x = (int)div_up(p.vwidth, fbx);
                f.bricks_z = (int)div_up(p.vwidth, fbz);
                f.splits = (uint32_t)div_up(E, f.a.per_split);
                f.unit_begin = P.fwd_units;
                const uint64_t units = (uint64_t)f.bricks_x * f.bricks_z * div_up(p.vheight, fby) * f.splits;
                if (P.fwd_units + units >= (1ull << 31)) return fail(XPR_ERR_UNSUPPORTED, "batch step too large");
                P.fwd_units += (uint32_t)units;
                fw.push_back(f);
            }
            xpr::BatchErrItem e{};
            e.images = (const char *)p.images + (size_t)s_idx * npix * dtype_size(b->opts.storage);
            e.sum = b->sums[i];
            e.ratio = b->ratios[i];
            e.residual = p.residual ? p.residual + k : nullptr;
            e.n = npix;
            e.weight = b->weight[i][k];
            e.first = k == 0;
            P.max_n = std::max(P.max_n, npix);
            er.push_back(e);
            xpr::BatchBwdItem w{};
            w.a = a;
            w.vol = p.vol;
            w.ratio = b->ratios[i];
            w.pd = pd;
            w.bricks_x = (int)div_up(p.vwidth, bbx);
            w.bricks_z = (int)div_up(p.vwidth, bbz);
            w.unit_begin = P.bwd_units;
            const uint64_t units = (uint64_t)w.bricks_x * w.bricks_z * div_up(p.vheight, bby);
            if (P.bwd_units + units >= (1ull << 31)) return fail(XPR_ERR_UNSUPPORTED, "batch step too large");
            P.bwd_units += (uint32_t)units;
            bw.push_back(w);
        }
        P.n_fwd = (int)fw.size();
        P.n_err = (int)er.size();
        P.n_bwd = (int)bw.size();
        if (!fw.empty()) P.fwd_off = append(fw.data(), fw.size() * sizeof(fw[0]));
        if (!er.empty()) P.err_off = append(er.data(), er.size() * sizeof(er[0]));
        if (!bw.empty()) P.bwd_off = append(bw.data(), bw.size() * sizeof(bw[0]));
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
                                       P.fwd_units, b->tickets, b->opts.arith, b->grid_fwd, s);
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
                                      b->opts.storage, b->opts.storage, P.max_n, *b->di, s);
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
// cleared after) for each projection-run split, the backward of step 0 against zero
// ratios for each column length.  exp(0 / count) is exactly 1, so a voxel is unchanged
// unless no projection of step 0 reaches it (count 0), and those voxels become NaN in
// step 0 of the run as well.
int autotune(xpr_batch *b, cudaStream_t s)
{
    uint32_t max_e = 0;
    std::vector<uint64_t> shape;
    for (const auto &p : b->probs) {
        max_e = std::max(max_e, entries_of(p));
        shape.insert(shape.end(), {p.vwidth, p.vheight, p.det_w, p.det_h, p.per_subset, p.modules});
    }
    const ShapeKey key{b->opts.arith, b->opts.storage, shape};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            b->tuned_ms = std::get<2>(it->second);
            return build_lists(b, std::get<0>(it->second), std::get<1>(it->second), s);
        }
    }
    int best_s = b->splits, best_c = b->column;
    float best_f = 0.0f, best_b = 0.0f;
    if (b->steps > 1) {
        bool first = true;
        for (int sp : {1, 2, 4, 8, 16}) {
            if (sp > 1 && (uint32_t)sp > div_up(max_e, 4)) break;
            if (int rc = build_lists(b, sp, b->column, s)) return rc;
            const float ms = time_ms(s, [&] {
                enqueue_forward(b, 1, s);
                enqueue_fill(b, 1, s);
            });
            if (first || ms < best_f) {
                best_f = ms;
                best_s = sp;
            }
            first = false;
        }
    }
    cudaError_t e = enqueue_fill(b, 2, s);
    if (e != cudaSuccess) return cuda_fail(e, "autotune");
    bool first = true;
    for (int cb : {16, 8}) {
        if (int rc = build_lists(b, best_s, cb, s)) return rc;
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
        g_tuned[key] = std::make_tuple(best_s, best_c, b->tuned_ms);
    }
    return build_lists(b, best_s, best_c, s);
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
    if (o.bwd_column != 0 && o.bwd_column != 8 && o.bwd_column != 16)
        return fail(XPR_ERR_INVALID, "bwd_column must be 0, 8 or 16");
    cudaError_t e = xpr::prepare_device_kernels();
    if (e != cudaSuccess) return cuda_fail(e, "xpr_batch_create");

    xpr_batch *b = new xpr_batch();
    b->ctx = ctx;
    b->di = di;
    b->opts = o;
    b->probs.assign(problems, problems + n);
    b->ctas = o.ctas_per_sm;
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint64_t scratch_bytes = 0;
    uint64_t total_bricks = 0;
    uint32_t max_e = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const xpr_batch_problem &p = b->probs[i];
        if (!p.vol || !p.images || !p.projdata) {
            release(b);
            return fail(XPR_ERR_INVALID, "xpr_batch_create: NULL buffer in a problem");
        }
        if (p.sit == 0 || p.it == 0 || p.per_subset == 0 || p.vwidth == 0 || p.vheight == 0) {
            release(b);
            return fail(XPR_ERR_INVALID, "xpr_batch_create: sit, it, per_subset and the grid must be positive");
        }
        xpr_launch L{};
        L.vmax[0] = (int32_t)p.vwidth;
        L.vmax[1] = (int32_t)p.vheight;
        L.vmax[2] = (int32_t)p.vwidth;
        for (int c = 0; c < 3; ++c) {
            L.origin[c] = p.orig[c];
            L.voxel[c] = p.voxel;
        }
        L.det_w = p.det_w;
        L.rows = p.det_h;
        L.n_angles = p.per_subset;
        L.modules = p.modules ? p.modules : 1u;
        L.arith = o.arith;
        xpr::LaunchArgs a;
        if (const char *m = xpr::make_launch_args(&L, entries_of(p), &a)) {
            release(b);
            return xpr::set_last_error(XPR_ERR_INVALID, "xpr_batch_create: problem %u: %s", i, m);
        }
        b->base.push_back(a);
        b->steps = std::max(b->steps, p.it * p.sit);
        // jitter: 3 draws per sub-iteration from std::mt19937(seed) (reconstruction.hpp:268-272)
        std::vector<float> jit((size_t)3 * p.it * p.sit), org(jit.size()), w((size_t)p.it * p.sit);
        xpr_jitter(p.seed, jit.size(), p.voxel, jit.data());
        float wt = p.weight;
        for (uint32_t k = 0; k < p.it * p.sit; ++k) {
            for (int c = 0; c < 3; ++c) org[3 * k + c] = p.orig[c] + jit[3 * k + c];
            w[k] = wt;
            if (k % p.sit == p.sit - 1) wt *= p.weight_factor;
        }
        b->origin.push_back(org);
        b->weight.push_back(w);
        const uint64_t npix = (uint64_t)p.per_subset * p.det_w * p.det_h;
        scratch_bytes += ((npix * 4 + 255) & ~255ull) + ((npix * dtype_size(o.storage) + 255) & ~255ull);
        b->max_vol = std::max<uint64_t>(b->max_vol, (uint64_t)p.vwidth * p.vheight * p.vwidth);
        b->max_pix = std::max(b->max_pix, npix);
        b->max_ratio_words = std::max<uint64_t>(b->max_ratio_words, div_up(npix * dtype_size(o.storage), 4));
        total_bricks += div_up(p.vwidth, 32) * div_up(p.vwidth, 32) * div_up(p.vheight, 8);
        max_e = std::max(max_e, entries_of(p));
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
        const xpr_batch_problem &p = b->probs[i];
        const uint64_t npix = (uint64_t)p.per_subset * p.det_w * p.det_h;
        b->sums.push_back((uint32_t *)q);
        q += (npix * 4 + 255) & ~255ull;
        b->ratios.push_back(q);
        q += (npix * dtype_size(o.storage) + 255) & ~255ull;
        fills[i] = {(uint32_t *)p.vol, (uint64_t)p.vwidth * p.vheight * p.vwidth, kOneBits, 0};
        fills[n + i] = {b->sums[i], npix, 0u, 0};
        fills[2 * n + i] = {(uint32_t *)b->ratios[i], div_up(npix * dtype_size(o.storage), 4), 0u, 0};
    }
    if ((e = cudaMemsetAsync(b->tickets, 0, 256, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b->fills, fills.data(), fills.size() * sizeof(fills[0]), cudaMemcpyHostToDevice, s)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        release(b);
        return cuda_fail(e, "xpr_batch_create");
    }
    // default schedule: split projection runs only when the batch has too few bricks to
    // fill the GPU (3 waves of the forward's 4 CTAs per SM)
    int splits = o.fwd_splits;
    if (splits <= 0) {
        const uint64_t target = (uint64_t)di->sm_count * 4 * 3;
        splits = total_bricks >= target ? 1 : (int)std::min<uint64_t>(div_up(target, total_bricks), div_up(max_e, 4));
        splits = std::max(splits, 1);
    }
    const int column = o.bwd_column ? o.bwd_column : 16;
    if (int rc = build_lists(b, splits, column, s)) {
        release(b);
        return rc;
    }
    if (o.autotune && o.fwd_splits <= 0 && o.bwd_column == 0) {
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
    const cudaError_t e = enqueue_step(b, step, reinterpret_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? XPR_OK : cuda_fail(e, "xpr_batch_step");
}

int xpr_batch_run(xpr_batch *b, void *stream)
{
    if (!b) return fail(XPR_ERR_INVALID, "xpr_batch_run: NULL batch");
    if (!xpr::context_device(b->ctx)) return XPR_ERR_INVALID;
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

int xpr_batch_schedule(const xpr_batch *b, int32_t *fwd_splits, int32_t *bwd_column, int32_t *ctas_per_sm,
                       double *tuned_ms)
{
    if (!b) return fail(XPR_ERR_INVALID, "xpr_batch_schedule: NULL batch");
    if (fwd_splits) *fwd_splits = b->splits;
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
