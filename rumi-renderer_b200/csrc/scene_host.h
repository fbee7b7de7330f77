// Host-side conversions from the C-ABI scene description (include/rumi_b200.h) to the
// device records of scene.cuh.  Pure host code: used by rumi_scene_create and by the
// scene-parameter setters, and compiled with a host compiler alone by the host builds of
// the kernels that the CPU tests run under address and undefined-behaviour checks.
// Derived constants are computed the way the reference's constructors compute them, in
// float (double where the reference mixes in its double PI):
//   Rect              src/Shape/rect.cpp:12-38          Sphere  src/Shape/sphere.cpp:18-38
//   Glossy            src/Material/glossy.cpp:19-25     Subsurface src/Material/subsurface.cpp:21-40
//   AreaLight::Pdf    src/Light/arealight.cpp:114-117   (Rect::Pdf rect.cpp:154, Sphere::Pdf sphere.cpp:134)
//   HomogeneousVolume src/Volume/homogeneousvolume.cpp:24-44
//   Pinhole           src/Camera/pinhole.cpp:30-51
#pragma once
#include <cmath>
#include <cstring>
#include "../../include/rumi_b200.h"
#include "scene.cuh"

namespace rumi {

inline float f_len(const float *v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

inline DevMaterial make_material(const rumi_material &m) {
    DevMaterial d;
    memset(&d, 0, sizeof(d));
    d.type = m.type;
    d.kd = m.kd;
    d.ks = m.ks;
    d.e = m.exponent;
    d.rgb = make_float3(m.rgb[0], m.rgb[1], m.rgb[2]);
    d.eta_in = m.eta_in;
    d.eta_out = m.eta_out;
    d.rgb2 = make_float3(m.rgb2[0], m.rgb2[1], m.rgb2[2]);
    if (m.type == RUMI_MAT_GLOSSY) {
        d.kd_pdf = m.kd / (m.kd + m.ks);
        d.phong_norm = (float)((m.exponent + 1.0f) / (2.0f * 3.14159265358979323846));
    }
    if (m.type == RUMI_MAT_SUBSURFACE) {
        const float st[3] = {m.rgb[0] + m.rgb2[0], m.rgb[1] + m.rgb2[1], m.rgb[2] + m.rgb2[2]};
        d.sigma_t = make_float3(st[0], st[1], st[2]);
        const float density = m.density > 0.0f ? m.density : 1.0f;
        d.avg_sigma_t = (st[2] + st[1] + st[0]) / 3.0f * density;
        d.absorb = ((m.rgb2[2] / st[2]) + (m.rgb2[1] / st[1]) + (m.rgb2[0] / st[0])) / 3.0f;
    }
    if (m.type == RUMI_MAT_EMISSIVE) d.le = make_float3(m.rgb[0] * m.kd, m.rgb[1] * m.kd, m.rgb[2] * m.kd);
    return d;
}

// One light of a validated description; mats: the converted material table.
inline DevLight make_light(const rumi_scene_desc &d, const rumi_light &L, const DevMaterial *mats) {
    DevLight dl;
    memset(&dl, 0, sizeof(dl));
    dl.type = L.type;
    dl.shape_type = L.shape_type;
    dl.shape_index = L.shape_index;
    if (L.type == RUMI_LIGHT_AREA) {
        int mi;
        if (L.shape_type == RUMI_SHAPE_RECT) {
            const float *r = d.rects + 9 * (size_t)L.shape_index;
            const float len = f_len(r + 3), wid = f_len(r + 6);
            dl.inv_area = 1.0f / (len * wid);
            mi = d.rect_material[L.shape_index];
        } else {
            const float rad = d.spheres[4 * L.shape_index + 3];
            dl.inv_area = (float)(1.0f / (4.0f * 3.14159265358979323846 * rad * rad));
            mi = d.sphere_material[L.shape_index];
        }
        dl.le = mats[mi].le;
    } else if (L.type == RUMI_LIGHT_SPOT) {
        dl.position = make_float3(L.position[0], L.position[1], L.position[2]);
        dl.direction = make_float3(L.direction[0], L.direction[1], L.direction[2]);
        dl.cos_cone = (float)std::cos(L.cone_deg * 3.14159265358979323846 / 180.0);
        dl.intensity = make_float3(L.intensity[0], L.intensity[1], L.intensity[2]);
        dl.inv_area = 1.0f;
    }
    return dl;
}

// HomogeneousVolume's constructor (src/Volume/homogeneousvolume.cpp:24-44): the box, the
// coefficients and the derived mean extinction and absorption probability.
inline void fill_dev_volume(DevVolume &dv, const rumi_volume &v) {
    dv.present = v.present ? 1 : 0;
    dv.bmin = make_float3(v.pmin[0], v.pmin[1], v.pmin[2]);
    dv.bmax = make_float3(v.pmax[0], v.pmax[1], v.pmax[2]);
    dv.sigma_s = make_float3(v.sigma_s[0], v.sigma_s[1], v.sigma_s[2]);
    dv.sigma_a = make_float3(v.sigma_a[0], v.sigma_a[1], v.sigma_a[2]);
    dv.sigma_t = make_float3(v.sigma_a[0] + v.sigma_s[0], v.sigma_a[1] + v.sigma_s[1], v.sigma_a[2] + v.sigma_s[2]);
    dv.avg_sigma_t = (dv.sigma_t.z + dv.sigma_t.y + dv.sigma_t.x) * 0.33333333333f;
    const float3 r = make_float3(dv.sigma_a.x / dv.sigma_t.x, dv.sigma_a.y / dv.sigma_t.y, dv.sigma_a.z / dv.sigma_t.z);
    dv.absorb = (r.z + r.y + r.x) * 0.33333333333f;
    dv.g = v.g;
}

// Pinhole's constructor (src/Camera/pinhole.cpp:30-49) with _fov set, and DepthOfField.
// _dir, _up and _right are Mat4x4 * Vector3, which adds the matrix's translation column.
inline void fill_dev_camera(DevCamera &dc, const rumi_camera &c) {
    memset(&dc, 0, sizeof(dc));
    dc.p = make_float3(c.position[0], c.position[1], c.position[2]);
    for (int k = 0; k < 12; ++k) dc.m[k] = c.basis[k];
    const float fov = c.fov_deg > 0.0f ? c.fov_deg : 20.0f;
    dc.tanfov = (float)std::tan(3.14159265358979323846 / 180.f * fov * 0.5f);
    dc.plane_dist = 1.0f;
    dc.y_ratio = c.y_ratio;
    dc.film_area = (2.0f * dc.tanfov) * (2.0f * dc.tanfov * c.y_ratio);
    dc.dir = make_float3(c.basis[2] + c.basis[3], c.basis[6] + c.basis[7], c.basis[10] + c.basis[11]);
    dc.up = make_float3(c.basis[1] + c.basis[3], c.basis[5] + c.basis[7], c.basis[9] + c.basis[11]);
    dc.right = make_float3(c.basis[0] + c.basis[3], c.basis[4] + c.basis[7], c.basis[8] + c.basis[11]);
    dc.focal_distance = c.focal_distance;
    dc.lens_radius = c.lens_radius;
}

}  // namespace rumi
