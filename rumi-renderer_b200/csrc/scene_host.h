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
#include <vector>
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

// One texture of the description without its pixels (the caller points img / hdr at them).
inline DevTexture make_texture(const rumi_texture &t) {
    DevTexture dt;
    memset(&dt, 0, sizeof(dt));
    dt.type = t.type;
    dt.rep_u = t.repeat_u;
    dt.rep_v = t.repeat_v;
    dt.c1 = make_float3(t.color1[0], t.color1[1], t.color1[2]);
    dt.c2 = make_float3(t.color2[0], t.color2[1], t.color2[2]);
    dt.gamma = t.gamma;
    dt.iw = t.img_width;
    dt.ih = t.img_height;
    dt.bpp = t.type == RUMI_TEX_HDR ? 3 : t.bytes_per_pixel;
    return dt;
}

// Bytes of a texture's pixel array (0 for a checker).
inline size_t texture_pixel_bytes(const rumi_texture &t) {
    if (t.type == RUMI_TEX_CHECKER) return 0;
    return t.type == RUMI_TEX_HDR ? sizeof(float) * 3 * (size_t)t.img_width * t.img_height
                                  : (size_t)t.img_width * t.img_height * t.bytes_per_pixel;
}

// Whether the description binds any texture to a primitive.
inline bool has_textures(const rumi_scene_desc &d) {
    return d.n_textures > 0 && (d.tri_texture || d.rect_texture || d.sphere_texture);
}

// Per-primitive texture index in canonical order (-1 = none) and each sphere's frame rows
// (identity when the description has none).
inline void texture_tables(const rumi_scene_desc &d, std::vector<int> &prim_tex, std::vector<float4> &frame) {
    const int nT = d.n_triangles, nR = d.n_rects, nS = d.n_spheres;
    prim_tex.assign((size_t)nT + nR + nS, -1);
    for (int i = 0; d.tri_texture && i < nT; ++i) prim_tex[i] = d.tri_texture[i];
    for (int i = 0; d.rect_texture && i < nR; ++i) prim_tex[(size_t)nT + i] = d.rect_texture[i];
    for (int i = 0; d.sphere_texture && i < nS; ++i) prim_tex[(size_t)nT + nR + i] = d.sphere_texture[i];
    frame.resize((size_t)nS * 3);
    for (int i = 0; i < nS; ++i) {
        const float *f = d.sphere_frame ? d.sphere_frame + 9 * (size_t)i : nullptr;
        for (int r = 0; r < 3; ++r)
            frame[3 * i + r] = f ? make_float4(f[3 * r], f[3 * r + 1], f[3 * r + 2], 0.0f)
                                 : make_float4(r == 0, r == 1, r == 2, 0.0f);
    }
}

// Sphere::Intersect's image-based-light branch: an emissive sphere with a texture.
inline bool sphere_is_ibl(const rumi_scene_desc &d, const DevMaterial *mats, int i) {
    return mats[d.sphere_material[i]].type == RUMI_MAT_EMISSIVE && d.n_textures > 0 && d.sphere_texture &&
           d.sphere_texture[i] >= 0;
}

}  // namespace rumi
