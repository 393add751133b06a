// run_api.cpp -- C ABI for whole runs and host utilities (include/xpr.h).
#include <cstring>
#include <iostream>
#include <string>

#include "../../../include/xpr.h"
#include "../xpr_internal.h"
#include "engine.h"
#include "params.h"
#include "planner.h"
#include "tiff.h"

namespace {

int copy_out(const std::string &s, char *buf, uint64_t cap, int64_t *len)
{
    if (len) *len = (int64_t)s.size();
    if (buf && cap) {
        const size_t n = std::min<size_t>(s.size(), (size_t)cap - 1);
        std::memcpy(buf, s.data(), n);
        buf[n] = 0;
        if (s.size() >= cap) return XPR_ERR_INVALID;
    }
    return XPR_OK;
}

}  // namespace

extern "C" {

int xpr_run(const char *json_or_path)
{
    xpr::Params p;
    try {
        p = xpr::load_params(json_or_path ? json_or_path : "");
    } catch (const std::exception &e) {
        std::cerr << e.what() << std::endl;
        return -2;  // RETURN_CODE_ERROR_PARAMETERS (main.cpp:23)
    }
    try {
        xpr::Engine eng(p, xpr::directory_images(p.input), true);
        if (!p.simulation) eng.reconstruct();           // main.cpp:123-126
        if (!p.proj_output.empty()) eng.simulate();     // main.cpp:129-131
    } catch (const std::exception &e) {
        std::cerr << "Error during the reconstruction : " << e.what() << std::endl;
        return -3;  // RETURN_CODE_ERROR_RECONSTRUCTION (main.cpp:24)
    }
    return 0;
}

int64_t xpr_template_json(char *buf, uint64_t cap)
{
    int64_t len = 0;
    copy_out(xpr::params_to_json(xpr::Params()), buf, cap, &len);
    return len;
}

int xpr_params_normalize(const char *json_or_path, char *buf, uint64_t cap, int64_t *len)
{
    try {
        return copy_out(xpr::params_to_json(xpr::load_params(json_or_path ? json_or_path : "")), buf, cap, len);
    } catch (const std::exception &e) {
        copy_out(e.what(), buf, cap, len);
        return XPR_ERR_PARAM;
    }
}

int xpr_reconstruct_host(const char *json, const float *images, int64_t count, uint32_t width, uint32_t height,
                         float *vol_out, uint64_t vol_cap, double *seconds)
{
    try {
        xpr::Params p = xpr::load_params(json ? json : "{}");
        xpr::Engine eng(p, xpr::memory_images(images, count, width, height), false);
        const uint64_t n = (uint64_t)eng.vwidth() * eng.vheight() * eng.vwidth();
        if (n > vol_cap)
            return xpr::set_last_error(XPR_ERR_INVALID, "xpr_reconstruct_host: vol_out holds %llu floats, %llu needed",
                                       (unsigned long long)vol_cap, (unsigned long long)n);
        eng.set_output(vol_out);  // straight into the caller's buffer
        eng.reconstruct();
        if (seconds) *seconds = eng.stats().seconds_iterations;
        return XPR_OK;
    } catch (const std::exception &e) {
        std::cerr << "xpr_reconstruct_host: " << e.what() << std::endl;
        return xpr::set_last_error(XPR_ERR_PARAM, "xpr_reconstruct_host: %s", e.what());
    }
}

int xpr_tiff_write(const char *path, const float *data, uint32_t width, uint32_t height)
{
    try {
        xpr::tiff_write_f32(path, data, width, height);
        return XPR_OK;
    } catch (const std::exception &e) {
        return xpr::set_last_error(XPR_ERR_IO, "xpr_tiff_write: %s", e.what());
    }
}

int xpr_tiff_read(const char *path, float *data, uint64_t cap, uint32_t *width, uint32_t *height)
{
    try {
        uint32_t w = 0, h = 0;
        std::vector<float> v = xpr::tiff_read_f32(path, &w, &h);
        if (width) *width = w;
        if (height) *height = h;
        if (data) {
            if (v.size() > cap)
                return xpr::set_last_error(XPR_ERR_INVALID, "xpr_tiff_read: the buffer holds %llu floats, %llu needed",
                                           (unsigned long long)cap, (unsigned long long)v.size());
            std::memcpy(data, v.data(), v.size() * sizeof(float));
        }
        return XPR_OK;
    } catch (const std::exception &e) {
        return xpr::set_last_error(XPR_ERR_IO, "xpr_tiff_read: %s", e.what());
    }
}

int xpr_plan_chunks(const xpr_geom_params *gp, const xpr_geom_out *go, const xpr_projdata *all, uint64_t avail,
                    uint64_t max_alloc, float overlap_fct, int64_t *chunks, int max_chunks, int *n_chunks)
{
    if (!gp || !go || !all || !chunks || !n_chunks) return XPR_ERR_INVALID;
    std::vector<xpr_projdata> v(all, all + gp->projections * gp->module_number);
    std::vector<xpr::Chunk> c;
    if (!xpr::plan_chunks(*gp, *go, v, avail, max_alloc, overlap_fct, &c)) {
        *n_chunks = -1;
        return XPR_OK;
    }
    *n_chunks = (int)c.size();
    for (size_t i = 0; i < c.size() && (int)i < max_chunks; ++i) {
        int64_t *o = chunks + 6 * i;
        o[0] = c[i].vOffset; o[1] = c[i].vSize; o[2] = c[i].iOffset; o[3] = c[i].iSize; o[4] = c[i].vPadTop; o[5] = c[i].vPadBot;
    }
    return (int)c.size() > max_chunks ? XPR_ERR_INVALID : XPR_OK;
}

int xpr_cull_layer(const xpr_geom_params *gp, const xpr_geom_out *go, const xpr_projdata *all, int64_t sit, int64_t layer,
                   int per_module, uint16_t *mvp_idx, uint16_t *img_idx, int *n)
{
    if (!gp || !go || !all || !mvp_idx || !img_idx || !n) return XPR_ERR_INVALID;
    std::vector<xpr_projdata> v(all, all + gp->projections * gp->module_number);
    *n = xpr::cull_layer(*gp, *go, v, sit, layer, per_module != 0, mvp_idx, img_idx);
    return XPR_OK;
}

}  // extern "C"
