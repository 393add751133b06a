// batch_plan.h -- work lists of batched sub-iterations, shared by xpr_batch (a fixed set
// of problems run in lock-step) and xpr_server (requests joining and leaving a running
// batch).  A problem is the naive method of reconstruction_n.hpp:27-88; its
// sub-iteration k is one forward item (k > 0), one error item and one backward item.
#pragma once

#include <cstdint>
#include <vector>

#include "../xpr_internal.h"
#include "xpr.h"

namespace xpr {

inline uint64_t div_up(uint64_t a, uint64_t b) { return (a + b - 1) / b; }
inline size_t dtype_size(int dt) { return dt == XPR_F32 ? 4 : 2; }
inline uint32_t entries_of(const xpr_batch_problem &p) { return p.per_subset * (p.modules ? p.modules : 1u); }
// entries per forward work unit (a multiple of the metadata group of 4) for `splits` runs
inline uint32_t per_split_for(uint32_t entries, int splits)
{
    return (uint32_t)div_up(div_up(entries, (uint64_t)(splits > 1 ? splits : 1)), 4) * 4;
}

struct PlannedProblem {
    xpr_batch_problem p{};
    LaunchArgs base{};             // launch arguments without the jittered origin
    std::vector<float> origin;     // 3 per sub-iteration: grid origin + std::mt19937 jitter
    std::vector<float> weight;     // 1 per sub-iteration: weight * weight_factor^(main iteration)
    uint32_t *sums = nullptr;      // fixed-point scratch, per_subset * det_w * det_h words
    void *ratio = nullptr;         // ratio scratch in the storage type
    uint32_t steps() const { return p.it * p.sit; }
    uint64_t npix() const { return (uint64_t)p.per_subset * p.det_w * p.det_h; }
};

// Validates `p` and derives its launch arguments, origins and weights; returns an error
// message or nullptr.  sums / ratio are left for the caller to set.
const char *plan_problem(const xpr_batch_problem &p, int arith, PlannedProblem *out);

struct StepItems {
    std::vector<BatchFwdItem> fwd;
    std::vector<BatchErrItem> err;
    std::vector<BatchBwdItem> bwd;
    uint32_t fwd_units = 0, bwd_units = 0;
    uint64_t max_n = 0;
    void clear()
    {
        fwd.clear();
        err.clear();
        bwd.clear();
        fwd_units = bwd_units = 0;
        max_n = 0;
    }
};

// Appends sub-iteration k of `pp` (k < pp.steps()); false when the step would exceed 2^31
// work units.  splits: projection runs per forward brick; layers: the forward brick's
// layers (8, or 16 in the STRICT contract); column: backward column length.
bool add_step_items(const PlannedProblem &pp, uint32_t k, int splits, int layers, int column, int image_dtype,
                    StepItems *out);

}  // namespace xpr
