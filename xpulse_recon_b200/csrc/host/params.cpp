// params.cpp -- see params.h
#include "params.h"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace xpr {

namespace {

const char *kMethods[] = {"naive", "method_1a", "method_1b", "method_1c", "method_2", "hartmann", "ipr"};

double num(const json::Value &v, const char *key)
{
    if (v.type == json::Value::Number) return v.num;
    if (v.type == json::Value::Bool) return v.b ? 1.0 : 0.0;
    throw std::runtime_error(std::string("parameter '") + key + "' must be a number");
}
bool boolean(const json::Value &v, const char *key)
{
    if (v.type == json::Value::Bool) return v.b;
    if (v.type == json::Value::Number) return v.num != 0.0;
    throw std::runtime_error(std::string("parameter '") + key + "' must be a boolean");
}
std::string str(const json::Value &v, const char *key)
{
    if (v.type == json::Value::String) return v.str;
    throw std::runtime_error(std::string("parameter '") + key + "' must be a string");
}

template <class F>
void opt(const json::Value *obj, const char *key, F &&set)
{
    if (!obj) return;
    const json::Value *v = obj->get(key);
    if (v && v->type != json::Value::Null) set(*v);
}

std::string fnum(double v)
{
    char b[64];
    snprintf(b, sizeof b, "%.9g", v);
    return b;
}

}  // namespace

const char *method_name(Method m) { return kMethods[(int)m]; }

uint64_t parse_bytes(const std::string &s)
{
    if (s.empty()) return 0;
    char *end = nullptr;
    double v = std::strtod(s.c_str(), &end);
    double mul = 1.0;
    if (end && *end) {
        switch (*end) {
            case 'k': case 'K': mul = 1024.0; break;
            case 'm': case 'M': mul = 1024.0 * 1024.0; break;
            case 'g': case 'G': mul = 1024.0 * 1024.0 * 1024.0; break;
            case 't': case 'T': mul = 1024.0 * 1024.0 * 1024.0 * 1024.0; break;
            default: throw std::runtime_error("bad byte size '" + s + "'");
        }
    }
    if (!(v >= 0.0)) throw std::runtime_error("bad byte size '" + s + "'");
    return (uint64_t)(v * mul);
}

Params params_from_json(const json::Value &root)
{
    if (!root.is_object()) throw std::runtime_error("the parameters must be a JSON object");
    Params p;
    const json::Value *r = root.get("recon");
    opt(r, "input", [&](const json::Value &v) { p.input = str(v, "input"); });
    opt(r, "output", [&](const json::Value &v) { p.output = str(v, "output"); });
    opt(r, "proj_output", [&](const json::Value &v) { p.proj_output = str(v, "proj_output"); });
    opt(r, "method", [&](const json::Value &v) {
        const std::string m = str(v, "method");
        for (int i = 0; i < 7; ++i)
            if (m == kMethods[i]) { p.method = (Method)i; return; }
        throw std::runtime_error("unknown method '" + m + "' (naive|method_1a|method_1b|method_1c|method_2)");
    });
    opt(r, "it", [&](const json::Value &v) { p.it = (int64_t)num(v, "it"); });
    opt(r, "sit", [&](const json::Value &v) { p.sit = (int64_t)num(v, "sit"); });
    opt(r, "mlog", [&](const json::Value &v) { p.mlog = boolean(v, "mlog"); });
    opt(r, "weight", [&](const json::Value &v) { p.weight = (float)num(v, "weight"); });
    opt(r, "weight_factor", [&](const json::Value &v) { p.weight_factor = (float)num(v, "weight_factor"); });
    opt(r, "images_preproc", [&](const json::Value &v) { p.normalize = boolean(v, "images_preproc"); });
    opt(r, "normalize", [&](const json::Value &v) { p.normalize = boolean(v, "normalize"); });
    opt(r, "simulation", [&](const json::Value &v) { p.simulation = boolean(v, "simulation"); });
    opt(r, "seed", [&](const json::Value &v) {
        p.seed_set = true;
        p.seed = (uint32_t)(uint64_t)num(v, "seed");
    });
    opt(r, "arith", [&](const json::Value &v) {
        p.arith = str(v, "arith");
        if (p.arith != "fast" && p.arith != "strict") throw std::runtime_error("recon.arith must be fast|strict");
    });
    opt(r, "storage", [&](const json::Value &v) {
        p.storage = str(v, "storage");
        if (p.storage != "fp32" && p.storage != "bf16" && p.storage != "fp16")
            throw std::runtime_error("recon.storage must be fp32|bf16|fp16");
    });
    opt(r, "image_storage", [&](const json::Value &v) {
        p.image_storage = str(v, "image_storage");
        if (p.image_storage != "fp32" && p.image_storage != "bf16" && p.image_storage != "fp16")
            throw std::runtime_error("recon.image_storage must be fp32|bf16|fp16");
    });
    opt(r, "geometry", [&](const json::Value &v) {
        p.geometry = str(v, "geometry");
        if (p.geometry != "fp32" && p.geometry != "fp64") throw std::runtime_error("recon.geometry must be fp32|fp64");
    });
    opt(r, "compat_pad", [&](const json::Value &v) { p.compat_pad = boolean(v, "compat_pad"); });
    opt(r, "resume", [&](const json::Value &v) { p.resume = str(v, "resume"); });
    opt(r, "first_iteration", [&](const json::Value &v) {
        const double k = num(v, "first_iteration");
        if (k < 0.0 || k != (double)(int64_t)k) throw std::runtime_error("recon.first_iteration must be an integer >= 0");
        p.first_iteration = (int64_t)k;
    });
    opt(r, "mem_cap", [&](const json::Value &v) {
        p.mem_cap = v.type == json::Value::String ? parse_bytes(v.str) : (uint64_t)num(v, "mem_cap");
    });
    opt(r, "device", [&](const json::Value &v) { p.device = (int)num(v, "device"); });
    opt(r, "slab", [&](const json::Value &v) { p.slab = (int64_t)num(v, "slab"); });
    opt(r, "slab_cache", [&](const json::Value &v) { p.slab_cache = (int64_t)num(v, "slab_cache"); });

    const json::Value *g = root.get("geometry");
    opt(g, "so", [&](const json::Value &v) { p.so = (float)num(v, "so"); });
    opt(g, "sd", [&](const json::Value &v) { p.sd = (float)num(v, "sd"); });
    opt(g, "angle", [&](const json::Value &v) { p.angle = (float)num(v, "angle"); });
    opt(g, "heli_offset", [&](const json::Value &v) { p.heli_offset = (float)num(v, "heli_offset"); });
    opt(g, "heli_step", [&](const json::Value &v) { p.heli_step = (float)num(v, "heli_step"); });
    opt(g, "angle_list", [&](const json::Value &v) {
        if (v.type != json::Value::Array) throw std::runtime_error("geometry.angle_list must be an array");
        for (const auto &e : v.arr) p.angle_list.push_back((float)num(e, "angle_list"));
    });

    const json::Value *d = root.get("detector");
    opt(d, "px", [&](const json::Value &v) { p.px = (float)num(v, "px"); });
    opt(d, "rx", [&](const json::Value &v) { p.rx = (float)num(v, "rx"); });
    opt(d, "sx", [&](const json::Value &v) { p.sx = (float)num(v, "sx"); });
    opt(d, "sy", [&](const json::Value &v) { p.sy = (float)num(v, "sy"); });
    opt(d, "module_number", [&](const json::Value &v) { p.module_number = (int64_t)num(v, "module_number"); });
    opt(d, "module_angle_offset", [&](const json::Value &v) {
        p.module_angle_offset_set = true;
        p.module_angle_offset = (float)num(v, "module_angle_offset");
    });
    opt(d, "module_center_offset_z",
        [&](const json::Value &v) { p.module_center_offset_z = (float)num(v, "module_center_offset_z"); });
    opt(d, "modules", [&](const json::Value &v) {
        if (v.type != json::Value::Array) throw std::runtime_error("detector.modules must be an array");
        for (const auto &e : v.arr) {
            ModuleParams m;
            opt(&e, "offset_x", [&](const json::Value &x) { m.offset_x = (float)num(x, "offset_x"); });
            opt(&e, "offset_y", [&](const json::Value &x) { m.offset_y = (float)num(x, "offset_y"); });
            opt(&e, "offset_z", [&](const json::Value &x) { m.offset_z = (float)num(x, "offset_z"); });
            opt(&e, "roll", [&](const json::Value &x) { m.roll = (float)num(x, "roll"); });
            opt(&e, "pitch", [&](const json::Value &x) { m.pitch = (float)num(x, "pitch"); });
            opt(&e, "yaw", [&](const json::Value &x) { m.yaw = (float)num(x, "yaw"); });
            p.modules.push_back(m);
        }
    });

    const json::Value *m2 = root.get("method2");
    opt(m2, "overlap_fct", [&](const json::Value &v) { p.overlap_fct = (float)num(v, "overlap_fct"); });
    const json::Value *hm = root.get("hartmann");
    opt(hm, "devx", [&](const json::Value &v) { p.hm_devx = str(v, "devx"); });
    opt(hm, "devy", [&](const json::Value &v) { p.hm_devy = str(v, "devy"); });
    opt(hm, "iterations", [&](const json::Value &v) { p.hm_iterations = (float)num(v, "iterations"); });
    opt(hm, "iterations_fct", [&](const json::Value &v) { p.hm_iterations_fct = (float)num(v, "iterations_fct"); });
    opt(hm, "iterations_step", [&](const json::Value &v) { p.hm_iterations_step = (int64_t)num(v, "iterations_step"); });
    opt(hm, "method", [&](const json::Value &v) { p.hm_method = str(v, "method"); });
    const json::Value *ip = root.get("ipr");
    opt(ip, "iterations", [&](const json::Value &v) { p.ipr_iterations = (float)num(v, "iterations"); });
    opt(ip, "iterations_fct", [&](const json::Value &v) { p.ipr_iterations_fct = (float)num(v, "iterations_fct"); });
    opt(ip, "iterations_step", [&](const json::Value &v) { p.ipr_iterations_step = (int64_t)num(v, "iterations_step"); });
    opt(ip, "energy_kev", [&](const json::Value &v) { p.ipr_energy_kev = (float)num(v, "energy_kev"); });

    // initializeParameters (parameters.hpp:34-48); rx stays in pixels here and is
    // multiplied by px (in the geometry's precision) where the geometry is built
    if (p.overlap_fct > 1.0f) p.overlap_fct = 1.0f;
    if (p.overlap_fct < 0.01f) p.overlap_fct = 0.01f;
    if (p.heli_step < 1.0f) p.heli_step = 1.0f;
    if (p.it < 1 || p.sit < 1) throw std::runtime_error("recon.it and recon.sit must be >= 1");
    if (p.first_iteration >= p.it) throw std::runtime_error("recon.first_iteration must be below recon.it");
    if (p.module_number < 1) throw std::runtime_error("detector.module_number must be >= 1");
    if (!p.modules.empty() && (int64_t)p.modules.size() != p.module_number)
        throw std::runtime_error("detector.modules must list module_number entries");
    return p;
}

Params load_params(const std::string &file_or_content)
{
    std::string text;
    if (file_or_content.empty() || file_or_content[0] != '{') {
        std::ifstream f(file_or_content);
        std::stringstream ss;
        ss << f.rdbuf();
        text = ss.str();
        if (text.empty()) throw std::runtime_error("Can not read the parameters file");
    } else {
        text = file_or_content;
    }
    return params_from_json(json::parse(text));
}

std::string params_to_json(const Params &p)
{
    std::ostringstream o;
    auto b = [](bool v) { return v ? "true" : "false"; };
    o << "{\"recon\":{\"input\":" << json::quote(p.input) << ",\"output\":" << json::quote(p.output)
      << ",\"proj_output\":" << json::quote(p.proj_output) << ",\"method\":\"" << method_name(p.method)
      << "\",\"it\":" << p.it << ",\"sit\":" << p.sit << ",\"mlog\":" << b(p.mlog) << ",\"weight\":" << fnum(p.weight)
      << ",\"weight_factor\":" << fnum(p.weight_factor) << ",\"normalize\":" << b(p.normalize)
      << ",\"simulation\":" << b(p.simulation);
    if (p.seed_set) o << ",\"seed\":" << p.seed;
    o << ",\"arith\":\"" << p.arith << "\",\"storage\":\"" << p.storage << "\"";
    if (!p.image_storage.empty()) o << ",\"image_storage\":\"" << p.image_storage << "\"";
    if (!p.resume.empty()) o << ",\"resume\":" << json::quote(p.resume);
    if (p.first_iteration > 0) o << ",\"first_iteration\":" << p.first_iteration;
    o << ",\"geometry\":\"" << p.geometry
      << "\",\"compat_pad\":" << b(p.compat_pad) << ",\"mem_cap\":" << p.mem_cap << ",\"device\":" << p.device
      << ",\"slab\":" << p.slab << ",\"slab_cache\":" << p.slab_cache << "}";
    o << ",\"geometry\":{\"so\":" << fnum(p.so) << ",\"sd\":" << fnum(p.sd) << ",\"angle\":" << fnum(p.angle)
      << ",\"heli_offset\":" << fnum(p.heli_offset) << ",\"heli_step\":" << fnum(p.heli_step) << ",\"angle_list\":[";
    for (size_t i = 0; i < p.angle_list.size(); ++i) o << (i ? "," : "") << fnum(p.angle_list[i]);
    o << "]}";
    o << ",\"detector\":{\"px\":" << fnum(p.px) << ",\"rx\":" << fnum(p.rx) << ",\"sx\":" << fnum(p.sx)
      << ",\"sy\":" << fnum(p.sy) << ",\"module_number\":" << p.module_number << ",\"module_angle_offset\":";
    if (p.module_angle_offset_set) o << fnum(p.module_angle_offset);
    else o << "null";
    o << ",\"module_center_offset_z\":" << fnum(p.module_center_offset_z);
    if (!p.modules.empty()) {
        o << ",\"modules\":[";
        for (size_t i = 0; i < p.modules.size(); ++i) {
            const ModuleParams &m = p.modules[i];
            o << (i ? "," : "") << "{\"offset_x\":" << fnum(m.offset_x) << ",\"offset_y\":" << fnum(m.offset_y)
              << ",\"offset_z\":" << fnum(m.offset_z) << ",\"roll\":" << fnum(m.roll) << ",\"pitch\":" << fnum(m.pitch)
              << ",\"yaw\":" << fnum(m.yaw) << "}";
        }
        o << "]";
    }
    o << "}";
    o << ",\"method2\":{\"overlap_fct\":" << fnum(p.overlap_fct) << "}";
    o << ",\"hartmann\":{\"devx\":" << json::quote(p.hm_devx) << ",\"devy\":" << json::quote(p.hm_devy)
      << ",\"iterations\":" << fnum(p.hm_iterations) << ",\"iterations_fct\":" << fnum(p.hm_iterations_fct)
      << ",\"iterations_step\":" << p.hm_iterations_step << ",\"method\":" << json::quote(p.hm_method) << "}";
    o << ",\"ipr\":{\"iterations\":" << fnum(p.ipr_iterations) << ",\"iterations_fct\":" << fnum(p.ipr_iterations_fct)
      << ",\"iterations_step\":" << p.ipr_iterations_step << ",\"energy_kev\":" << fnum(p.ipr_energy_kev) << "}}";
    return o.str();
}

void geom_params_from(const Params &p, int64_t projections, uint32_t width, uint32_t height,
                      xpr_geom_params *gp, std::vector<float> *mod_offset, std::vector<float> *mod_rpy)
{
    *gp = xpr_geom_params{};
    gp->so = p.so;
    gp->sd = p.sd;
    gp->angle = p.angle;
    gp->heli_offset = p.heli_offset;
    gp->px = p.px;
    gp->rx_px = p.rx;
    gp->sx = p.sx;
    gp->sy = p.sy;
    gp->module_number = p.module_number;
    gp->module_angle_offset_set = p.module_angle_offset_set ? 1 : 0;
    gp->module_angle_offset = p.module_angle_offset;
    gp->module_center_offset_z = p.module_center_offset_z;
    gp->dwidth = width;
    gp->dheight = height;
    gp->projections = projections;
    gp->sit = p.sit;
    gp->angle_list = p.angle_list.empty() ? nullptr : p.angle_list.data();
    mod_offset->clear();
    mod_rpy->clear();
    if (!p.modules.empty()) {
        for (const auto &m : p.modules) {
            mod_offset->insert(mod_offset->end(), {m.offset_x, m.offset_y, m.offset_z});
            mod_rpy->insert(mod_rpy->end(), {m.roll, m.pitch, m.yaw});
        }
        gp->mod_offset = mod_offset->data();
        gp->mod_rpy = mod_rpy->data();
    }
}

}  // namespace xpr
