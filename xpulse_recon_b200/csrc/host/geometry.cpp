// geometry.cpp -- acquisition geometry -> ProjData (xpr_geometry) and the origin
// jitter sequence (xpr_jitter).
//
// Follows src/reconstruction/dataset/geometry.hpp:35-76 (source / detector
// placement), 182-234 (generalized perspective projection T*Mt*P*S), 244-265
// (detector corners), 267-292 (per-angle, per-module matrices), 298-328
// (ordering).  glm's conventions are kept: mat4(16 scalars) fills columns, a
// matrix product sums column vectors left to right, vec3 dot is
// (x*x' + y*y') + z*z', normalize(v) = v * (1/sqrt(dot(v,v))).  The template runs
// in float (the reference's single-precision construction, operation for
// operation) or in double (matrices built in FP64 and rounded once).
// Built with -ffp-contract=off so no multiply-add is fused.
#include <cmath>
#include <cstdint>
#include <random>

#include "../../../include/xpr.h"

namespace {

template <class T>
struct V3 {
    T x, y, z;
};
template <class T> V3<T> add(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> V3<T> sub(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> V3<T> mul(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> T dot(V3<T> a, V3<T> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class T> V3<T> cross(V3<T> a, V3<T> b)
{
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
template <class T> V3<T> normalize(V3<T> a) { return mul(a, T(1) / std::sqrt(dot(a, a))); }
template <class T> T radians(T d) { return d * T(0.01745329251994329576923690768489); }
template <class T> T degrees(T r) { return r * T(57.295779513082320876798154814105); }

// rotate(vec, origin, x, y, z) of geometry.hpp:88-95: about X, then Y, then Z (degrees)
template <class T>
V3<T> rotate_xyz(V3<T> vec, V3<T> o, T ax, T ay, T az)
{
    V3<T> v = sub(vec, o), t;
    T c = std::cos(radians(ax)), s = std::sin(radians(ax));
    t = v; t.y = v.y * c - v.z * s; t.z = v.y * s + v.z * c; v = t;
    c = std::cos(radians(ay)); s = std::sin(radians(ay));
    t = v; t.x = v.x * c + v.z * s; t.z = -v.x * s + v.z * c; v = t;
    c = std::cos(radians(az)); s = std::sin(radians(az));
    t = v; t.x = v.x * c - v.y * s; t.y = v.x * s + v.y * c; v = t;
    return add(v, o);
}

// rotation about a unit axis (Rodrigues) for the per-module roll/pitch/yaw extension
// (the reference's formula is commented out at geometry.hpp:260-262)
template <class T>
V3<T> rotate_axis(V3<T> v, T angle_rad, V3<T> k)
{
    T c = std::cos(angle_rad), s = std::sin(angle_rad);
    V3<T> kxv = cross(k, v);
    T kd = dot(k, v) * (T(1) - c);
    return add(add(mul(v, c), mul(kxv, s)), mul(k, kd));
}

template <class T>
struct M4 {
    T c[4][4];  // c[column][row]
};
template <class T> M4<T> from_scalars(const T r[16])
{
    M4<T> m;
    for (int i = 0; i < 16; ++i) m.c[i / 4][i % 4] = r[i];
    return m;
}
template <class T> M4<T> mmul(const M4<T> &A, const M4<T> &B)
{
    M4<T> R;
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 4; ++i)
            R.c[j][i] = ((A.c[0][i] * B.c[j][0] + A.c[1][i] * B.c[j][1]) + A.c[2][i] * B.c[j][2]) + A.c[3][i] * B.c[j][3];
    return R;
}

// computeGeneralizedProjection (geometry.hpp:182-234)
template <class T>
M4<T> generalized_projection(V3<T> pe, V3<T> pa, V3<T> pb, V3<T> pc, T vpl, T vpr, T vpb, T vpt, T sd)
{
    const V3<T> vr = normalize(sub(pb, pa));
    const V3<T> vu = normalize(sub(pc, pa));
    const V3<T> vn = normalize(cross(vu, vr));
    const V3<T> va = sub(pa, pe), vb = sub(pb, pe), vc = sub(pc, pe);
    const T d = -dot(va, vn);
    const T n = T(1), f = sd * T(2);
    const T l = dot(vr, va) * (n / d);
    const T r = dot(vr, vb) * (n / d);
    const T b = dot(vu, va) * (n / d);
    const T t = dot(vu, vc) * (n / d);
    const T z = T(0), one = T(1), h = T(0.5);
    const T P[16] = {(T(2) * n) / (r - l), z, (r + l) / (r - l), z,
                     z, (T(2) * n) / (t - b), (t + b) / (t - b), z,
                     z, z, -(f + n) / (f - n), -(T(2) * f * n) / (f - n),
                     z, z, -one, z};
    const T Mt[16] = {vr.x, vr.y, vr.z, z, vu.x, vu.y, vu.z, z, vn.x, vn.y, vn.z, z, z, z, z, one};
    const T Tm[16] = {one, z, z, -pe.x, z, one, z, -pe.y, z, z, one, -pe.z, z, z, z, one};
    const T S[16] = {(vpr - vpl) * h, z, z, (vpr + vpl) * h, z, (vpt - vpb) * h, z, (vpt + vpb) * h,
                     z, z, h, h, z, z, z, one};
    return mmul(mmul(mmul(from_scalars(Tm), from_scalars(Mt)), from_scalars(P)), from_scalars(S));
}

template <class T>
void build_matrices(const xpr_geom_params *gp, xpr_projdata *out)
{
    const int64_t P = gp->projections, M = gp->module_number;
    const uint64_t width = (uint64_t)gp->dwidth / (uint64_t)M;
    const uint64_t height = (uint64_t)gp->dheight;
    const T px = T(gp->px), sd = T(gp->sd), so = T(gp->so);
    const T rx = T(gp->rx_px) * px;  // parameters.hpp:39 (rx *= px)
    // geometry.hpp:59-67: source-space placement, then object space
    V3<T> source_pos = {T(0), T(0), T(0)};
    V3<T> source_at = add(source_pos, V3<T>{T(0), T(0), sd});
    V3<T> axis_proj = add(source_at, V3<T>{-T(gp->sx) + rx, -T(gp->sy), T(0)});
    V3<T> object_center = add(source_pos, mul(normalize(sub(axis_proj, source_pos)), so));
    source_pos = sub(source_pos, object_center);
    source_at = sub(source_at, object_center);
    object_center = {T(0), T(0), T(0)};
    const T heli_off = T(gp->heli_offset);
    for (int64_t i = 0; i < P; ++i) {
        const T heli = (heli_off / T(P)) * T(i) - heli_off * T(0.5);
        const T angle_deg = gp->angle_list ? T(gp->angle_list[i]) : T(i) * (T(gp->angle) / T(P));
        const V3<T> rsp = add(rotate_xyz(source_pos, object_center, T(0), angle_deg, T(0)), V3<T>{T(0), heli, T(0)});
        const V3<T> rsa = add(rotate_xyz(source_at, object_center, T(0), angle_deg, T(0)), V3<T>{T(0), heli, T(0)});
        for (int64_t mod = 0; mod < M; ++mod) {
            // detectorFromSource (geometry.hpp:244-265)
            const V3<T> vv = {T(0), T(1), T(0)};
            const V3<T> dir = sub(rsa, rsp);
            const V3<T> u = normalize(cross(vv, dir));
            const V3<T> nrm = normalize(dir);
            V3<T> detector = sub(sub(rsa, mul(u, T(gp->sx))), mul(vv, T(gp->sy)));
            if (gp->mod_offset) {
                const float *o = gp->mod_offset + 3 * mod;
                detector = add(detector, add(add(mul(u, T(o[0]) * px), mul(vv, T(o[1]) * px)), mul(nrm, T(o[2]) * px)));
            }
            V3<T> ul = sub(sub(detector, mul(u, T(0.5) * T(width) * px)), mul(vv, T(0.5) * T(height) * px));
            V3<T> ur = add(ul, mul(u, T(width) * px));
            V3<T> bl = add(ul, mul(vv, T(height) * px));
            if (gp->mod_rpy) {
                const float *a = gp->mod_rpy + 3 * mod;  // roll, pitch, yaw
                V3<T> *cs[3] = {&ul, &ur, &bl};
                for (int c = 0; c < 3; ++c) {
                    V3<T> w = sub(*cs[c], detector);
                    w = rotate_axis(w, radians(T(a[2])), u);
                    w = rotate_axis(w, radians(T(a[1])), vv);
                    w = rotate_axis(w, radians(T(a[0])), nrm);
                    *cs[c] = add(w, detector);
                }
            }
            // computeDetectorProjection (geometry.hpp:267-292)
            const V3<T> center = detector;
            const V3<T> mc = add(center, mul(normalize(sub(rsp, rsa)), sd - T(gp->module_center_offset_z)));
            const V3<T> dd = sub(center, mc);
            const T dist = std::sqrt(dot(dd, dd));
            const T mang = gp->module_angle_offset_set ? T(gp->module_angle_offset)
                                                       : degrees(T(2) * std::atan2(T(width) * T(0.5) * px, dist));
            const T mcur = mang * (T(mod) - std::floor(T(M) / T(2)));
            const V3<T> pa = rotate_xyz(ul, mc, T(0), mcur, T(0));
            const V3<T> pb = rotate_xyz(ur, mc, T(0), mcur, T(0));
            const V3<T> pc = rotate_xyz(bl, mc, T(0), mcur, T(0));
            const T vpl = T(width * (uint64_t)mod), vpr = T(width * (uint64_t)(mod + 1));
            const T vpb = T(0), vpt = T(gp->dheight);
            const M4<T> mvp = generalized_projection(rsp, pa, pb, pc, vpl, vpr, vpb, vpt, sd);
            xpr_projdata &o = out[i * M + mod];
            for (int c = 0; c < 4; ++c)
                for (int r = 0; r < 4; ++r) o.mvp[c * 4 + r] = (float)mvp.c[c][r];
            o.vp[0] = (float)vpl;
            o.vp[1] = (float)vpr;
            o.vp[2] = (float)vpb;
            o.vp[3] = (float)vpt;
        }
    }
}

}  // namespace

extern "C" int xpr_geometry(const xpr_geom_params *gp, int fp64, xpr_projdata *out, xpr_geom_out *go)
{
    if (!gp || !out || !go) return XPR_ERR_INVALID;
    if (gp->projections <= 0 || gp->sit <= 0 || gp->module_number <= 0 || gp->dwidth <= 0 || gp->dheight <= 0)
        return XPR_ERR_PARAM;
    if (!(gp->sd > 0.0f) || !(gp->so > 0.0f) || !(gp->px > 0.0f)) return XPR_ERR_PARAM;
    // geometry.hpp:49-68: voxel grid, single precision in both modes
    go->vx = gp->px * (gp->so / gp->sd);
    go->vwidth = gp->dwidth;
    go->vheight = gp->dheight + (int64_t)std::fabs(gp->heli_offset / go->vx);
    go->concurrent = (int64_t)std::floor((float)gp->projections / (float)gp->sit);
    // the object centre is the origin of object space (geometry.hpp:67-68)
    go->orig[0] = 0.0f + -0.5f * (float)go->vwidth * go->vx;
    go->orig[1] = 0.0f + -0.5f * (float)go->vheight * go->vx;
    go->orig[2] = 0.0f + -0.5f * (float)go->vwidth * go->vx;
    if (fp64) build_matrices<double>(gp, out);
    else build_matrices<float>(gp, out);
    return XPR_OK;
}

// reconstruction.hpp:268-272: std::uniform_real_distribution<float>(0, vx) drawn from
// std::mt19937, one value per axis per sub-iteration.
extern "C" int xpr_jitter(uint32_t seed, uint64_t n, float vx, float *out)
{
    if (!out && n) return XPR_ERR_INVALID;
    std::mt19937 gen(seed);
    for (uint64_t i = 0; i < n; ++i) out[i] = std::uniform_real_distribution<float>(0.0f, vx)(gen);
    return XPR_OK;
}
