// params.h -- the XPRecon parameter schema.
//
// Keys and defaults follow src/reconstruction/dataset/parameters/global_parameters.hpp:8-55
// and specialized_parameters.hpp:22-39; loading follows dataset/parameters.hpp:34-84
// (a path, or inline JSON when the argument starts with '{'; rx is converted from
// pixels to mm after loading).  Extensions of this backend (all optional):
//   recon.seed           origin-jitter seed (absent: std::random_device, as the reference)
//   recon.arith          "strict" | "fast"  projector arithmetic contract (strict: the
//                        reference kernels' IEEE single-precision results, bit for bit)
//   recon.storage        "fp32" | "bf16" | "fp16"  ratio storage, and the measured images'
//                        unless recon.image_storage is set
//   recon.image_storage  "fp32" | "bf16" | "fp16"  storage of the preprocessed measured images
//   recon.geometry       "fp32" | "fp64"  precision of the matrix construction (fp32: the
//                        reference's single-precision glm construction, the default)
//   recon.compat_pad     reproduce the reference's NDRange padding work-items (naive)
//   recon.mem_cap        device-memory cap, bytes or "64G" / "512M"
//   recon.device         CUDA device ordinal
//   recon.slab           layers per streamed y-slab in method_1a/1b/1c (0: as many as fit)
//   recon.slab_cache     slabs method_1b/1c keep on the device (0: as many as the memory holds)
//   recon.images_preproc alias of recon.normalize (the README's name for it)
//   recon.resume         directory of a previous result's layer_%05d.tif stack: the initial
//                        volume instead of the uniform one (every sub-iteration runs its
//                        forward; with recon.normalize the layers are divided by the images'
//                        max - min, the inverse of the scaling they were saved with)
//   recon.first_iteration  k: the run performs iterations k .. it - 1 of the schedule, with
//                        iteration k's weight (weight * weight_factor^k) and origin-jitter
//                        draws; with recon.resume on the result of iterations 0 .. k - 1 it
//                        continues that run bit for bit (naive, method_1a / 1b / 1c)
//   detector.modules[]   per-module {offset_x, offset_y, offset_z, roll, pitch, yaw}
//                        (the reference's commented-out global_parameters.hpp:38-44, 51)
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../../include/xpr.h"
#include "json.h"

namespace xpr {

enum class Method { naive, method_1a, method_1b, method_1c, method_2, hartmann, ipr };

struct ModuleParams {
    float offset_x = 0.0f, offset_y = 0.0f, offset_z = 0.0f;
    float roll = 0.0f, pitch = 0.0f, yaw = 0.0f;
};

struct Params {
    // recon (global_parameters.hpp:8-21)
    std::string input = "./";
    std::string output = "./recon/";
    std::string proj_output = "";
    Method method = Method::method_1b;
    int64_t it = 1, sit = 10;
    bool mlog = true;
    float weight = 1.0f, weight_factor = 0.9f;
    bool normalize = false;
    bool simulation = false;
    // geometry (:23-36)
    float so = 100.0f, sd = 1000.0f, angle = 360.0f;
    float heli_offset = 0.0f, heli_step = 1.0f;
    std::vector<float> angle_list;
    // detector (:46-54)
    float px = 0.1f, rx = 0.0f, sx = 0.0f, sy = 0.0f;  // rx in pixels as read; rx_mm() after loading
    int64_t module_number = 1;
    bool module_angle_offset_set = false;
    float module_angle_offset = 0.0f;
    float module_center_offset_z = 0.0f;
    std::vector<ModuleParams> modules;
    // method2 (specialized_parameters.hpp:34-39)
    float overlap_fct = 1.0f;
    // hartmann / ipr (kept for the schema and -template; the methods are not implemented here)
    std::string hm_devx = "./", hm_devy = "./";
    float hm_iterations = 0.0f, hm_iterations_fct = 1.0f;
    int64_t hm_iterations_step = 1;
    std::string hm_method = "gs";
    float ipr_iterations = 0.0f, ipr_iterations_fct = 1.0f;
    int64_t ipr_iterations_step = 1;
    float ipr_energy_kev = 1.0f;
    // extensions
    bool seed_set = false;
    uint32_t seed = 0;
    std::string arith = "strict";
    std::string storage = "fp32";
    std::string image_storage;  // empty: as storage
    std::string geometry = "fp32";
    bool compat_pad = false;
    std::string resume;  // empty: the uniform initial volume
    int64_t first_iteration = 0;
    uint64_t mem_cap = 0;
    int device = 0;
    int64_t slab = 0;
    int64_t slab_cache = 0;
};

const char *method_name(Method m);

// Parse a parameter file path or an inline JSON string (starting with '{'), apply
// initializeParameters (parameters.hpp:34-48).  Throws std::runtime_error.
Params load_params(const std::string &file_or_content);
Params params_from_json(const json::Value &root);
// The default parameter set serialised as JSON (XPRecon -template, main.cpp:75-79).
std::string params_to_json(const Params &p);
uint64_t parse_bytes(const std::string &s);

// The geometry parameters of `p` for `projections` images of width x height
// (dataset.hpp:214-235 derives dwidth / dheight / projections from the images).
// mod_offset / mod_rpy receive the per-module arrays gp points into.
void geom_params_from(const Params &p, int64_t projections, uint32_t width, uint32_t height,
                      xpr_geom_params *gp, std::vector<float> *mod_offset, std::vector<float> *mod_rpy);

}  // namespace xpr
