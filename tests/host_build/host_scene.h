// A scene of the C-ABI description laid out as the device kernels read it, in host memory,
// for the host builds of the kernels (tests/host_build): the library's own host conversions
// (scene_host.h) plus, restated here, what the device build computes on the GPU -- the
// intersection records of the canonical primitives (prim_prepare_kernel in bvh_build.cu),
// the shading normals (pack_tri_shade_kernel in api.cu) and a BVH of one leaf holding every
// primitive in canonical order (every ray tests every primitive, which gives the closest hit
// of any valid tree).  Texture pixels are read where the description holds them.  Include
// after the kernel source.
#pragma once
#include <algorithm>
#include <vector>

namespace host_build {

using namespace rumi;

struct HostScene {
    std::vector<DevMaterial> mats;
    std::vector<DevLight> lights;
    std::vector<DevTexture> tex;
    std::vector<int> prim_tex;
    std::vector<float4> frame;
    bool has_ibl = false, has_subsurface = false;
    std::vector<float4> rects, spheres, tri_shade, tri_albedo, prims;
    std::vector<int> sphere_mat;
    BvhNode root;
    DevScene dev;
};

void grow(float lo[3], float hi[3], float x, float y, float z) {
    lo[0] = std::min(lo[0], x); lo[1] = std::min(lo[1], y); lo[2] = std::min(lo[2], z);
    hi[0] = std::max(hi[0], x); hi[1] = std::max(hi[1], y); hi[2] = std::max(hi[2], z);
}

// Returns 0, or -1 for a description this build does not cover.
int build_scene(const rumi_scene_desc &d, HostScene &H) {
    const int nT = d.n_triangles, nR = d.n_rects, nS = d.n_spheres, N = nT + nR + nS;
    H.mats.resize(d.n_materials);
    for (int i = 0; i < d.n_materials; ++i) {
        H.mats[i] = make_material(d.materials[i]);
        H.has_subsurface |= H.mats[i].type == RUMI_MAT_SUBSURFACE;
    }
    H.lights.resize(d.n_lights);
    for (int i = 0; i < d.n_lights; ++i) {
        H.has_ibl |= d.lights[i].type == RUMI_LIGHT_IBL;
        H.lights[i] = make_light(d, d.lights[i], H.mats.data());
    }
    if (has_textures(d)) {
        H.tex.resize(d.n_textures);
        for (int i = 0; i < d.n_textures; ++i) {
            const rumi_texture &t = d.textures[i];
            H.tex[i] = make_texture(t);
            if (t.type == RUMI_TEX_HDR)
                H.tex[i].hdr = static_cast<const float *>(t.pixels);
            else if (t.type != RUMI_TEX_CHECKER)
                H.tex[i].img = static_cast<const unsigned char *>(t.pixels);
        }
        texture_tables(d, H.prim_tex, H.frame);
    }
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    H.prims.resize(3 * (size_t)(N > 0 ? N : 1));
    H.tri_shade.resize(3 * (size_t)(nT > 0 ? nT : 1));
    for (int i = 0; i < nT; ++i) {
        const float *t = d.tri_vertices + 9 * (size_t)i;
        const float3 v0 = make_float3(t[0], t[1], t[2]), v1 = make_float3(t[3], t[4], t[5]),
                     v2 = make_float3(t[6], t[7], t[8]);
        for (int k = 0; k < 3; ++k) grow(lo, hi, t[3 * k], t[3 * k + 1], t[3 * k + 2]);
        const float3 e1 = rn_sub(v1, v0), e2 = rn_sub(v2, v0);
        H.prims[3 * i + 0] = make_float4(v0.x, v0.y, v0.z, __int_as_float(i));
        H.prims[3 * i + 1] = make_float4(e1.x, e1.y, e1.z, __int_as_float(PRIM_TRI));
        H.prims[3 * i + 2] = make_float4(e2.x, e2.y, e2.z, 0.0f);
        float3 n0, n1, n2;
        if (d.tri_normals) {
            const float *q = d.tri_normals + 9 * (size_t)i;
            n0 = make_float3(q[0], q[1], q[2]);
            n1 = make_float3(q[3], q[4], q[5]);
            n2 = make_float3(q[6], q[7], q[8]);
        } else {
            n0 = n1 = n2 = normalize_ref(rn_cross(e1, e2));
        }
        H.tri_shade[3 * i + 0] = make_float4(n0.x, n0.y, n0.z, __int_as_float(d.tri_material[i]));
        H.tri_shade[3 * i + 1] = make_float4(n1.x, n1.y, n1.z, 0.0f);
        H.tri_shade[3 * i + 2] = make_float4(n2.x, n2.y, n2.z, 0.0f);
    }
    if (nT > 0 && d.tri_albedo) {
        H.tri_albedo.resize(nT);
        for (int i = 0; i < nT; ++i)
            H.tri_albedo[i] = make_float4(d.tri_albedo[3 * i], d.tri_albedo[3 * i + 1], d.tri_albedo[3 * i + 2], 0.0f);
    }
    H.rects.resize(3 * (size_t)(nR > 0 ? nR : 1));
    for (int r = 0; r < nR; ++r) {
        const float *q = d.rects + 9 * (size_t)r;
        const int mi = d.rect_material[r];
        H.rects[3 * r + 0] = make_float4(q[0], q[1], q[2], __int_as_float(mi));
        H.rects[3 * r + 1] = make_float4(q[3], q[4], q[5], 0.0f);
        H.rects[3 * r + 2] = make_float4(q[6], q[7], q[8], 0.0f);
        const DevMaterial &m = H.mats[mi];
        const bool emissive = m.type == RUMI_MAT_EMISSIVE && (m.le.x != 0.0f || m.le.y != 0.0f || m.le.z != 0.0f);
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
                grow(lo, hi, q[0] + a * q[3] + b * q[6], q[1] + a * q[4] + b * q[7], q[2] + a * q[5] + b * q[8]);
        const int i = nT + r;
        H.prims[3 * i + 0] = make_float4(q[0], q[1], q[2], __int_as_float(i));
        H.prims[3 * i + 1] = make_float4(q[3], q[4], q[5], __int_as_float(PRIM_RECT | (emissive ? PRIM_FLAG_EMISSIVE : 0)));
        H.prims[3 * i + 2] = make_float4(q[6], q[7], q[8], 0.0f);
    }
    H.spheres.resize(nS > 0 ? nS : 1);
    H.sphere_mat.assign(d.sphere_material, d.sphere_material + nS);
    if (nS == 0) H.sphere_mat.push_back(0);
    for (int s = 0; s < nS; ++s) {
        const float *c = d.spheres + 4 * (size_t)s;
        H.spheres[s] = make_float4(c[0], c[1], c[2], c[3]);
        grow(lo, hi, c[0] - c[3], c[1] - c[3], c[2] - c[3]);
        grow(lo, hi, c[0] + c[3], c[1] + c[3], c[2] + c[3]);
        const int i = nT + nR + s;
        H.prims[3 * i + 0] = make_float4(c[0], c[1], c[2], __int_as_float(i));
        H.prims[3 * i + 1] = make_float4(c[3], 0.0f, 0.0f,
                                         __int_as_float(PRIM_SPHERE | (sphere_is_ibl(d, H.mats.data(), s) ? PRIM_FLAG_IBL : 0)));
        H.prims[3 * i + 2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    // the one leaf: its box padded by a little, so rays grazing the scene's bounds reach it
    memset(&H.root, 0, sizeof(H.root));
    if (N > 0) {
        float pad = 0.0f;
        for (int k = 0; k < 3; ++k) pad = std::max(pad, (hi[k] - lo[k]) * 1e-4f + 1e-4f);
        H.root.lo_x = lo[0] - pad; H.root.lo_y = lo[1] - pad; H.root.lo_z = lo[2] - pad;
        H.root.hi_x = hi[0] + pad; H.root.hi_y = hi[1] + pad; H.root.hi_z = hi[2] + pad;
        H.root.first = 0;
        H.root.count = N;
    } else {
        H.root.lo_x = H.root.lo_y = H.root.lo_z = 1.0f;
        H.root.hi_x = H.root.hi_y = H.root.hi_z = -1.0f;  // an empty box: every ray misses
    }
    DevScene &S = H.dev;
    memset(&S, 0, sizeof(S));
    S.nodes = &H.root;
    S.n_nodes = 1;
    S.leaf_prims = H.prims.data();
    S.tri_shade = H.tri_shade.data();
    S.tri_albedo = H.tri_albedo.empty() ? nullptr : H.tri_albedo.data();
    S.rects = H.rects.data();
    S.spheres = H.spheres.data();
    S.sphere_mat = H.sphere_mat.data();
    S.materials = H.mats.data();
    S.lights = H.lights.data();
    S.n_tris = nT;
    S.n_rects = nR;
    S.n_spheres = nS;
    S.n_prims = N;
    S.n_materials = d.n_materials;
    S.n_lights = d.n_lights;
    if (d.volume.present) fill_dev_volume(S.volume, d.volume);
    fill_dev_camera(S.camera, d.camera);
    S.width = d.width;
    S.height = d.height;
    if (!H.tex.empty()) {
        S.textures = H.tex.data();
        S.prim_tex = H.prim_tex.data();
        S.sphere_frame = H.frame.empty() ? nullptr : H.frame.data();
        S.n_textures = d.n_textures;
    }
    return 0;
}

}  // namespace host_build
