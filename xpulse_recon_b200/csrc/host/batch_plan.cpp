// batch_plan.cpp -- see batch_plan.h.
#include "batch_plan.h"

namespace xpr {

const char *plan_problem(const xpr_batch_problem &p, int arith, PlannedProblem *out)
{
    if (!p.vol || !p.images || !p.projdata) return "NULL buffer";
    if (p.sit == 0 || p.it == 0 || p.per_subset == 0 || p.vwidth == 0 || p.vheight == 0)
        return "sit, it, per_subset and the grid must be positive";
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
    L.arith = arith;
    if (const char *m = make_launch_args(&L, entries_of(p), &out->base)) return m;
    out->p = p;
    // the jitter: 3 draws per sub-iteration from std::mt19937(seed) (reconstruction.hpp:268-272);
    // the weight: *= weight_factor after each main iteration (reconstruction_n.hpp:84)
    const uint32_t n = p.it * p.sit;
    std::vector<float> jit((size_t)3 * n);
    xpr_jitter(p.seed, jit.size(), p.voxel, jit.data());
    out->origin.resize(jit.size());
    out->weight.resize(n);
    float wt = p.weight;
    for (uint32_t k = 0; k < n; ++k) {
        for (int c = 0; c < 3; ++c) out->origin[3 * k + c] = p.orig[c] + jit[3 * k + c];
        out->weight[k] = wt;
        if (k % p.sit == p.sit - 1) wt *= p.weight_factor;
    }
    return nullptr;
}

bool add_step_items(const PlannedProblem &pp, uint32_t k, int splits, int layers, int column, int image_dtype,
                    StepItems *out)
{
    const xpr_batch_problem &p = pp.p;
    const uint32_t s_idx = k % p.sit;
    const uint32_t E = entries_of(p);
    LaunchArgs a = pp.base;
    for (int c = 0; c < 3; ++c) a.origin[c] = pp.origin[3 * k + c];
    const xpr_projdata *pd = p.projdata + (size_t)s_idx * E;
    const uint64_t npix = pp.npix();
    if (k > 0) {  // the first sub-iteration has no forward (reconstruction_n.hpp:70)
        BatchFwdItem f{};
        f.a = a;
        f.a.per_split = per_split_for(E, splits);
        f.vol = p.vol;
        f.sum = pp.sums;
        f.pd = pd;
        f.bricks_x = (int)div_up(p.vwidth, forward_brick(0, layers));
        f.bricks_z = (int)div_up(p.vwidth, forward_brick(2, layers));
        f.splits = (uint32_t)div_up(E, f.a.per_split);
        f.unit_begin = out->fwd_units;
        const uint64_t units = (uint64_t)f.bricks_x * f.bricks_z * div_up(p.vheight, forward_brick(1, layers)) * f.splits;
        if (out->fwd_units + units >= (1ull << 31)) return false;
        out->fwd_units += (uint32_t)units;
        out->fwd.push_back(f);
    }
    BatchErrItem e{};
    e.images = (const char *)p.images + (size_t)s_idx * npix * dtype_size(image_dtype);
    e.sum = pp.sums;
    e.ratio = pp.ratio;
    e.residual = p.residual ? p.residual + k : nullptr;
    e.n = npix;
    e.weight = pp.weight[k];
    e.first = k == 0;
    out->max_n = out->max_n > npix ? out->max_n : npix;
    out->err.push_back(e);
    BatchBwdItem w{};
    w.a = a;
    w.vol = p.vol;
    w.ratio = pp.ratio;
    w.pd = pd;
    w.bricks_x = (int)div_up(p.vwidth, backward_brick(0, column));
    w.bricks_z = (int)div_up(p.vwidth, backward_brick(2, column));
    w.unit_begin = out->bwd_units;
    const uint64_t units = (uint64_t)w.bricks_x * w.bricks_z * div_up(p.vheight, backward_brick(1, column));
    if (out->bwd_units + units >= (1ull << 31)) return false;
    out->bwd_units += (uint32_t)units;
    out->bwd.push_back(w);
    return true;
}

}  // namespace xpr
