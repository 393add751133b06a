// planner.cpp -- see planner.h.  Built with -ffp-contract=off: every float operation
// below is the single-precision operation of the reference's glm code, in order.
#include "planner.h"

#include <algorithm>
#include <cmath>

namespace xpr {

namespace {

// (point * mvp / w).y for point (x, y, z, 1) (geometry.hpp:135-139, geometry_chunk.hpp:58-62)
inline float project_y(const xpr_projdata &d, float x, float y, float z)
{
    const float *m = d.mvp;
    const float py = ((m[4] * x + m[5] * y) + m[6] * z) + m[7] * 1.0f;
    const float pw = ((m[12] * x + m[13] * y) + m[14] * z) + m[15] * 1.0f;
    return py / pw;
}

inline float smin(float a, float b) { return (b < a) ? b : a; }  // std::min
inline float smax(float a, float b) { return (a < b) ? b : a; }  // std::max

struct Planner {
    const xpr_geom_params &gp;
    const xpr_geom_out &go;
    std::vector<float> ymin, ymax;
    uint64_t avail, max_alloc;
    float overlap;

    void y_projection(int64_t off, int64_t h, float *a, float *b) const
    {
        *a = smin(ymin[off], ymin[off + h - 1]);
        *b = smax(ymax[off], ymax[off + h - 1]);
    }
    void update_image_viewport(Chunk &c) const
    {
        float a, b;
        y_projection(c.vOffset, c.vSize, &a, &b);
        c.iOffset = (int64_t)smax(std::floor(a) - 1.0f, 0.0f);
        c.iSize = (int64_t)smax(smin(std::ceil(b - (float)c.iOffset) + 2.0f, (float)(gp.dheight - c.iOffset)), 0.0f);
    }
    void update_volume_padding(Chunk &c) const
    {
        c.vPadTop = 0;
        c.vPadBot = 0;
        float a, b;
        while (c.vOffset - c.vPadTop > 0) {
            y_projection(c.vOffset - c.vPadTop, 1, &a, &b);
            if (!(b > (float)(c.iOffset - 1))) break;
            ++c.vPadTop;
        }
        while (c.vOffset + c.vSize + c.vPadBot < go.vheight - 1) {
            y_projection(c.vOffset + c.vSize + c.vPadBot, 1, &a, &b);
            if (!(a < (float)(c.iOffset + c.iSize + 1))) break;
            ++c.vPadBot;
        }
        c.vPadTop = (int64_t)std::ceil((float)c.vPadTop * overlap);
        c.vPadBot = (int64_t)std::ceil((float)c.vPadBot * overlap);
    }
    bool fit(const Chunk &c) const
    {
        const int64_t W = go.vwidth, layer = W * W, line = gp.dwidth, Pc = go.concurrent;
        const uint64_t total = (uint64_t)(((c.vSize + c.vPadTop + c.vPadBot) * layer + 2 * c.iSize * line * Pc) * 4);
        const uint64_t images = (uint64_t)(c.iSize * line * Pc * 4);
        const uint64_t padding = (uint64_t)(std::max(c.vPadBot, c.vPadTop) * layer * 4);
        return avail > total && max_alloc - 1 > images && max_alloc > padding;
    }
};

}  // namespace

bool plan_chunks(const xpr_geom_params &gp, const xpr_geom_out &go, const std::vector<xpr_projdata> &all,
                 uint64_t avail_bytes, uint64_t max_alloc_bytes, float overlap_fct, std::vector<Chunk> *chunks)
{
    const int64_t H = go.vheight;
    Planner pl{gp, go, std::vector<float>(H), std::vector<float>(H), avail_bytes, max_alloc_bytes,
               overlap_fct > 1.0f ? 1.0f : (overlap_fct < 0.01f ? 0.01f : overlap_fct)};
    const float ox = go.orig[0], oy = go.orig[1], oz = go.orig[2];
    const float bx[4] = {ox, -ox, ox, -ox}, bz[4] = {-oz, -oz, oz, oz};
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < H; ++l) {
        float mn = INFINITY, mx = -INFINITY;
        const float yt = oy + (float)(int)l * go.vx;
        const float yb = oy + (float)(int)(l + 1) * go.vx;
        for (const auto &d : all)
            for (int j = 0; j < 4; ++j) {
                const float a = project_y(d, bx[j], yt, bz[j]);
                const float b = project_y(d, bx[j], yb, bz[j]);
                if (a < mn) mn = a;
                if (b < mn) mn = b;
                if (mx < a) mx = a;
                if (mx < b) mx = b;
            }
        pl.ymin[l] = mn;
        pl.ymax[l] = mx;
    }
    // first / last complete layers: std::upper_bound over the (ascending) bounds
    int64_t first = 0, last = 0;
    while (first < H && !(0.0f < pl.ymin[first])) ++first;
    while (last < H && !((float)(H - 1) < pl.ymax[last])) ++last;
    chunks->clear();
    Chunk c0;
    c0.vOffset = first;
    chunks->push_back(c0);
    for (int64_t i = 0; i < last - first; ++i) {
        Chunk t = chunks->back();
        ++t.vSize;
        pl.update_image_viewport(t);
        pl.update_volume_padding(t);
        if (pl.fit(t)) {
            chunks->back() = t;
        } else {
            if (t.vSize <= 1) return false;
            Chunk n;
            n.vOffset = chunks->back().vOffset + chunks->back().vSize;
            chunks->push_back(n);
        }
    }
    return true;
}

int cull_layer(const xpr_geom_params &gp, const xpr_geom_out &go, const std::vector<xpr_projdata> &all, int64_t sit,
               int64_t layer, bool per_module, uint16_t *mvp_idx, uint16_t *img_idx)
{
    const int64_t P = gp.projections, S = gp.sit, M = gp.module_number;
    const float ox = go.orig[0], oy = go.orig[1], oz = go.orig[2];
    const float bx[8] = {ox, -ox, ox, -ox, ox, -ox, ox, -ox};
    const float by[8] = {oy - 1.0f, oy - 1.0f, oy - 1.0f, oy - 1.0f, oy + 1.0f, oy + 1.0f, oy + 1.0f, oy + 1.0f};
    const float bz[8] = {-oz, -oz, oz, oz, -oz, -oz, oz, oz};
    int n = 0;
    uint16_t slot = 0;
    for (int64_t i = sit; i < P; i += S) {
        for (int64_t mod = 0; mod < M; ++mod) {
            const int64_t k = per_module ? i * M + mod : i;
            const xpr_projdata &d = all[(size_t)k];
            int64_t mn = go.vheight * 2, mx = -go.vheight;
            for (int j = 0; j < 8; ++j) {
                const float y = by[j] + (float)(uint32_t)layer * go.vx;
                const int64_t line = (int64_t)project_y(d, bx[j], y, bz[j]);
                mn = std::min(mn, line);
                mx = std::max(mx, line);
            }
            const float fmn = (float)mn, fmx = (float)mx;
            if (!(fmn >= d.vp[3] && fmx >= d.vp[3]) && !(fmn < d.vp[2] && fmx < d.vp[2])) {
                mvp_idx[n] = (uint16_t)k;
                img_idx[n] = slot;
                ++n;
            }
        }
        ++slot;
    }
    return n;
}

}  // namespace xpr
