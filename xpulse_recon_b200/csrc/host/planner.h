// planner.h -- host-side planning for the out-of-core memory modes.
#pragma once

#include <cstdint>
#include <vector>

#include "../../../include/xpr.h"

namespace xpr {

// method_2 chunk (specialized_parameters.hpp:28-32)
struct Chunk {
    int64_t vOffset = 0, vSize = 0, iOffset = 0, iSize = 0, vPadTop = 0, vPadBot = 0;
};

// GeometryChunk::computeLayerYBounds + computeChunks (geometry_chunk.hpp:92-197).
// `all` holds the ProjData of every (angle, module).  Returns false when a single
// layer does not fit ("Not enough GPU memory for the chunk division").
bool plan_chunks(const xpr_geom_params &gp, const xpr_geom_out &go, const std::vector<xpr_projdata> &all,
                 uint64_t avail_bytes, uint64_t max_alloc_bytes, float overlap_fct, std::vector<Chunk> *chunks);

// Geometry::getMvpPerLayer for one (sub-iteration, layer) (geometry.hpp:141-171,
// 334-355): ProjData indexes and image slots that may touch the layer.  The index is
// angle*modules + module (per_module != 0) or the reference's angle index.
int cull_layer(const xpr_geom_params &gp, const xpr_geom_out &go, const std::vector<xpr_projdata> &all, int64_t sit,
               int64_t layer, bool per_module, uint16_t *mvp_idx, uint16_t *img_idx);

}  // namespace xpr
