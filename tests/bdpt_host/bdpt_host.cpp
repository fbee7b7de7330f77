// Host build of the BDPT kernel (rumi-renderer_b200/csrc/bdpt.cu): the kernel body
// compiled by g++ as plain C++ and run one camera sample after another, so that the CPU
// tests can run it under AddressSanitizer and UndefinedBehaviorSanitizer with every
// automatic variable set to a non-zero pattern (an index read before it is written then
// leaves its range and is caught).  Test infrastructure, not part of the library.
//
// The scene goes through the library's own host conversions (scene_host.h); what the
// device build computes on the GPU is restated here on the host:
//   - the intersection records of the canonical primitives (prim_prepare_kernel in
//     bvh_build.cu) and the shading normals (pack_tri_shade_kernel in api.cu);
//   - a BVH of one leaf holding every primitive, in canonical order: the traversal then
//     tests all primitives for every ray, which gives the closest hit of any valid tree.
// Scenes with textures are not supported (the kernel's texture reads are not covered).
#include "cuda_host_shim.h"
#include "../../rumi-renderer_b200/csrc/bdpt.cu"

#include <algorithm>
#include <vector>

using namespace rumi;

namespace {

struct HostScene {
    std::vector<DevMaterial> mats;
    std::vector<DevLight> lights;
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
    if (d.n_textures > 0 && (d.tri_texture || d.rect_texture || d.sphere_texture)) return -1;
    const int nT = d.n_triangles, nR = d.n_rects, nS = d.n_spheres, N = nT + nR + nS;
    H.mats.resize(d.n_materials);
    for (int i = 0; i < d.n_materials; ++i) H.mats[i] = make_material(d.materials[i]);
    H.lights.resize(d.n_lights);
    for (int i = 0; i < d.n_lights; ++i) {
        if (d.lights[i].type == RUMI_LIGHT_IBL) return -1;
        H.lights[i] = make_light(d, d.lights[i], H.mats.data());
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
        H.prims[3 * i + 1] = make_float4(c[3], 0.0f, 0.0f, __int_as_float(PRIM_SPHERE));
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
    return 0;
}

}  // namespace

extern "C" {

// Renders camera samples [pix0 * spp, (pix0 + n_pix) * spp) of a BDPT frame, one after
// another, with the kernel's launch parameters set as bdpt_render sets them.
//   L_out      : n_pix * spp * 4 floats (each sample's value, as the kernel writes it)
//   light_film : width * height * 3 floats (B, G, R light-tracing splats), zeroed here
//   chk        : 4 ints, the kernel's index-check record (0 in chk[0]: no check fired)
// Returns 0, -1 for a description this build does not cover, -2 for bad arguments.
int rumi_host_bdpt(const rumi_scene_desc *d, int n_light, int n_eye, int spp, uint64_t seed, int pix0, int n_pix,
                   float *L_out, float *light_film, int *chk) {
    if (!d || !L_out || !light_film || !chk || spp < 1 || n_pix < 0 || pix0 < 0) return -2;
    if (n_light < 2 || n_eye < 2 || n_light > BD_MAXV || n_eye > BD_MAXV) return -2;
    if ((long long)pix0 + n_pix > (long long)d->width * d->height || d->n_lights <= 0) return -2;
    HostScene H;
    if (build_scene(*d, H) != 0) return -1;
    BdLaunch B;
    memset(&B, 0, sizeof(B));
    B.s = H.dev;
    B.nL = n_light;
    B.nE = n_eye;
    B.spp = spp;
    B.k0 = (uint32_t)seed;
    B.k1 = (uint32_t)(seed >> 32) ^ 0x5851F42Du;
    int g = 0;
    while ((g + 1) * (g + 1) <= spp) ++g;
    B.grid_d = g;
    B.square = g * g == spp;
    B.L = reinterpret_cast<float4 *>(L_out);
    B.light_film = light_film;
    memset(light_film, 0, sizeof(float) * 3 * (size_t)d->width * d->height);
    const DevCamera &c = B.s.camera;
    B.right = mk3(c.m[0] + c.m[3], c.m[4] + c.m[7], c.m[8] + c.m[11]);
    B.up = mk3(c.m[1] + c.m[3], c.m[5] + c.m[7], c.m[9] + c.m[11]);
    B.pix0 = pix0;
    B.n_paths = n_pix * spp;
    B.path0 = (long long)pix0 * spp;
    memset(g_bd_range, 0, sizeof(g_bd_range));
    blockDim = {(unsigned)BD_THREADS, 1, 1};
    gridDim = {(unsigned)((B.n_paths + BD_THREADS - 1) / BD_THREADS), 1, 1};
    for (int j = 0; j < B.n_paths; ++j) {
        blockIdx.x = (unsigned)(j / BD_THREADS);
        threadIdx.x = (unsigned)(j % BD_THREADS);
        if (n_light <= 8 && n_eye <= 8)
            bdpt_kernel<8>(B);
        else
            bdpt_kernel<BD_MAXV>(B);
    }
    memcpy(chk, g_bd_range, sizeof(g_bd_range));
    return 0;
}

}  // extern "C"
