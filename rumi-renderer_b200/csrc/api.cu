// C-ABI entry points (include/rumi_b200.h): scene upload + BVH build, render, ray
// queries, errors.  Derived constants are computed the way the reference's constructors
// compute them, in float (double where the reference mixes in its double PI):
//   Rect          src/Shape/rect.cpp:12-38          Sphere  src/Shape/sphere.cpp:18-38
//   Glossy        src/Material/glossy.cpp:19-25      Subsurface src/Material/subsurface.cpp:21-40
//   HomogeneousVolume src/Volume/homogeneousvolume.cpp:24-44
//   Pinhole       src/Camera/pinhole.cpp:30-51
#include <mutex>
#include "renderer.h"
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include <chrono>

static thread_local std::string g_last_error;

namespace rumi {

void set_error(const std::string &msg) { g_last_error = msg; }

rumi_status cuda_status(cudaError_t e, const char *what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? RUMI_ERR_OOM : RUMI_ERR_CUDA;
}

// Device allocations of scenes and render workspaces come from the device's default
// stream-ordered memory pool.  The pool keeps up to POOL_KEEP_BYTES of freed memory for
// reuse within this process, so creating a scene after destroying one does not go back
// to the CUDA driver.
static constexpr unsigned long long POOL_KEEP_BYTES = 16ull << 30;

void configure_pool(int device) {
    static bool done[64] = {};
    if (device < 0 || device >= 64 || done[device]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        unsigned long long keep = POOL_KEEP_BYTES;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    done[device] = true;
}

cudaError_t dalloc(void **p, size_t bytes, cudaStream_t s) {
    cudaError_t e = cudaMallocAsync(p, bytes > 0 ? bytes : 256, s);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
    }
    return e;
}

void dfree(void *p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

// One render workspace per device outlives the scene that used it: a scene destroyed
// hands its workspace here (its stream synchronised, so no work uses it any more) and the
// next scene on that device takes it if it is large enough.  A program that creates a
// scene per frame then allocates its ~0.7 GB of wave state once; through the pool alone a
// fresh 0.7 GB request after many scene-sized ones was measured to stall for up to ~0.7 s.
static std::mutex g_ws_mutex;
static void *g_ws_cache[64] = {};
static size_t g_ws_cache_bytes[64] = {};

static void workspace_release(rumi_scene *sc) {
    if (!sc->ws) return;
    void *drop = sc->ws;
    if (sc->device >= 0 && sc->device < 64) {
        std::lock_guard<std::mutex> lock(g_ws_mutex);
        if (g_ws_cache_bytes[sc->device] < sc->ws_bytes) {
            drop = g_ws_cache[sc->device];
            g_ws_cache[sc->device] = sc->ws;
            g_ws_cache_bytes[sc->device] = sc->ws_bytes;
        }
    }
    if (drop) dfree(drop, sc->stream);
    sc->ws = nullptr;
    sc->ws_bytes = 0;
}

rumi_status ensure_workspace(rumi_scene *sc, size_t bytes) {
    if (sc->ws_bytes >= bytes) return RUMI_OK;
    if (sc->ws) {
        dfree(sc->ws, sc->stream);
        sc->ws = nullptr;
        sc->ws_bytes = 0;
    }
    if (sc->device >= 0 && sc->device < 64) {
        std::lock_guard<std::mutex> lock(g_ws_mutex);
        if (g_ws_cache[sc->device] && g_ws_cache_bytes[sc->device] >= bytes) {
            sc->ws = g_ws_cache[sc->device];
            sc->ws_bytes = g_ws_cache_bytes[sc->device];
            g_ws_cache[sc->device] = nullptr;
            g_ws_cache_bytes[sc->device] = 0;
            return RUMI_OK;
        }
    }
    cudaError_t e = dalloc(&sc->ws, bytes, sc->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_status(e, "workspace allocation");
    }
    sc->ws_bytes = bytes;
    return RUMI_OK;
}

// The compressed eight-wide tree (trace_mode 5), collapsed from the binary tree the first
// time a call asks for it: a worst-case array first, then an exact copy.  Synchronous on
// the scene's stream; afterwards sc->dev carries it.
rumi_status ensure_bvh8(rumi_scene *sc) {
    if (sc->nodes8) return RUMI_OK;
    cudaStream_t s = sc->stream;
    const int N = sc->dev.n_prims;
    const int cap8 = bvh8_node_capacity(N);
    Bvh8Node *tmp8 = nullptr;
    void *scratch8 = nullptr;
    float4 *prims8 = nullptr;
    cudaError_t e = dalloc((void **)&tmp8, sizeof(Bvh8Node) * (size_t)cap8, s);
    if (e == cudaSuccess) e = dalloc((void **)&prims8, sizeof(float4) * 3 * (size_t)(N > 0 ? N : 1), s);
    if (e == cudaSuccess) e = dalloc(&scratch8, bvh8_scratch_bytes(N), s);
    int n8 = -1;
    if (e == cudaSuccess) n8 = bvh8_collapse(sc->nodes, sc->n_nodes, sc->leaf_prims, N, tmp8, cap8, prims8, scratch8, s);
    Bvh8Node *nodes8 = nullptr;
    if (e == cudaSuccess && n8 > 0) e = dalloc((void **)&nodes8, sizeof(Bvh8Node) * (size_t)n8, s);
    if (e == cudaSuccess && n8 > 0)
        e = cudaMemcpyAsync(nodes8, tmp8, sizeof(Bvh8Node) * (size_t)n8, cudaMemcpyDeviceToDevice, s);
    dfree(tmp8, s);
    dfree(scratch8, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    // stack entries hold node << 8: fewer than 2^24 nodes
    if (e != cudaSuccess || n8 <= 0 || n8 >= (1 << 24)) {
        dfree(nodes8, s);
        dfree(prims8, s);
        cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "eight-wide BVH");
        set_error("eight-wide BVH collapse failed");
        return RUMI_ERR_INTERNAL;
    }
    sc->nodes8 = nodes8;
    sc->prims8 = prims8;
    sc->n_nodes8 = n8;
    sc->dev.nodes8 = nodes8;
    sc->dev.prims8 = prims8;
    sc->dev.n_nodes8 = n8;
    return RUMI_OK;
}

}  // namespace rumi

using namespace rumi;

namespace {

template <typename T>
rumi_status upload(T **dst, const void *src, size_t bytes, cudaStream_t s) {
    *dst = nullptr;
    if (bytes == 0) return RUMI_OK;
    cudaError_t e = dalloc((void **)dst, bytes, s);
    if (e != cudaSuccess) return cuda_status(e, "device allocation");
    e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_status(e, "cudaMemcpyAsync");
    return RUMI_OK;
}

void free_scene(rumi_scene *sc) {
    if (!sc) return;
    cudaStream_t s = sc->stream;
    dfree(sc->nodes, s);
    dfree(sc->nodes4, s);
    dfree(sc->nodes8, s);
    dfree(sc->prims8, s);
    dfree(sc->leaf_prims, s);
    dfree(sc->tri_shade, s);
    dfree(sc->tri_albedo, s);
    dfree(sc->rects, s);
    dfree(sc->spheres, s);
    dfree(sc->sphere_mat, s);
    dfree(sc->materials, s);
    dfree(sc->lights, s);
    dfree(sc->textures, s);
    dfree(sc->prim_tex, s);
    dfree(sc->sphere_frame, s);
    dfree(sc->kept_L, s);
    for (void *p : sc->tex_pixels) dfree(p, s);
    if (sc->aux_stream) {
        cudaStreamSynchronize(sc->aux_stream);
        cudaStreamDestroy(sc->aux_stream);
    }
    if (sc->ev_fork) cudaEventDestroy(sc->ev_fork);
    if (sc->ev_join) cudaEventDestroy(sc->ev_join);
    if (s) cudaStreamSynchronize(s);  // nothing uses the workspace any more
    workspace_release(sc);
    if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    delete sc;
}

rumi_status validate(const rumi_scene_desc *d) {
    if (!d) return set_error("desc is NULL"), RUMI_ERR_INVALID_ARG;
    if (d->width <= 0 || d->height <= 0) return set_error("film size must be positive"), RUMI_ERR_INVALID_ARG;
    if (d->n_triangles < 0 || d->n_rects < 0 || d->n_spheres < 0 || d->n_materials < 0 || d->n_lights < 0)
        return set_error("negative count"), RUMI_ERR_INVALID_ARG;
    if ((long long)d->n_triangles + d->n_rects + d->n_spheres > 0x3fffffffLL)
        return set_error("too many primitives"), RUMI_ERR_INVALID_ARG;
    if (d->n_triangles > 0 && (!d->tri_vertices || !d->tri_material))
        return set_error("triangle arrays missing"), RUMI_ERR_INVALID_ARG;
    if (d->n_rects > 0 && (!d->rects || !d->rect_material)) return set_error("rect arrays missing"), RUMI_ERR_INVALID_ARG;
    if (d->n_spheres > 0 && (!d->spheres || !d->sphere_material))
        return set_error("sphere arrays missing"), RUMI_ERR_INVALID_ARG;
    if (d->n_materials > 0 && !d->materials) return set_error("materials missing"), RUMI_ERR_INVALID_ARG;
    if (d->n_lights > 0 && !d->lights) return set_error("lights missing"), RUMI_ERR_INVALID_ARG;
    auto check_mat = [&](const int32_t *m, int n) -> bool {
        for (int i = 0; i < n; ++i)
            if (m[i] < 0 || m[i] >= d->n_materials) return false;
        return true;
    };
    if (!check_mat(d->tri_material, d->n_triangles) || !check_mat(d->rect_material, d->n_rects) ||
        !check_mat(d->sphere_material, d->n_spheres))
        return set_error("material index out of range"), RUMI_ERR_INVALID_ARG;
    for (int i = 0; i < d->n_materials; ++i)
        if (d->materials[i].type < RUMI_MAT_MATTE || d->materials[i].type > RUMI_MAT_SUBSURFACE)
            return set_error("unknown material type"), RUMI_ERR_INVALID_ARG;
    for (int i = 0; i < d->n_lights; ++i) {
        const rumi_light &L = d->lights[i];
        if (L.type == RUMI_LIGHT_AREA) {
            if (L.shape_type == RUMI_SHAPE_RECT && (L.shape_index < 0 || L.shape_index >= d->n_rects))
                return set_error("light rect index out of range"), RUMI_ERR_INVALID_ARG;
            if (L.shape_type == RUMI_SHAPE_SPHERE && (L.shape_index < 0 || L.shape_index >= d->n_spheres))
                return set_error("light sphere index out of range"), RUMI_ERR_INVALID_ARG;
            if (L.shape_type != RUMI_SHAPE_RECT && L.shape_type != RUMI_SHAPE_SPHERE)
                return set_error("area lights must be rects or spheres"), RUMI_ERR_INVALID_ARG;
        } else if (L.type == RUMI_LIGHT_IBL) {
            if (L.shape_type != RUMI_SHAPE_SPHERE || L.shape_index < 0 || L.shape_index >= d->n_spheres)
                return set_error("an image-based light needs a sphere index"), RUMI_ERR_INVALID_ARG;
            // ImageBasedLight reads its radiance from the sphere's texture
            if (!d->sphere_texture || d->sphere_texture[L.shape_index] < 0)
                return set_error("the image-based light's sphere has no texture"), RUMI_ERR_INVALID_ARG;
        } else if (L.type != RUMI_LIGHT_SPOT) {
            return set_error("unknown light type"), RUMI_ERR_INVALID_ARG;
        }
    }
    if (d->volume.present) {
        // the free-flight sampler divides by the mean extinction and the absorption
        // probability by each channel's (rumi_scene_set_volume applies the same rule)
        for (int c = 0; c < 3; ++c)
            if (!(d->volume.sigma_s[c] >= 0.0f) || !(d->volume.sigma_a[c] >= 0.0f) ||
                !(d->volume.sigma_s[c] + d->volume.sigma_a[c] > 0.0f))
                return set_error("medium coefficients must be >= 0 with positive extinction"), RUMI_ERR_INVALID_ARG;
        if (!(d->volume.g > -1.0f && d->volume.g < 1.0f))
            return set_error("medium g must lie in (-1, 1)"), RUMI_ERR_INVALID_ARG;
    }
    if (d->n_textures < 0 || (d->n_textures > 0 && !d->textures))
        return set_error("textures missing"), RUMI_ERR_INVALID_ARG;
    for (int i = 0; i < d->n_textures; ++i) {
        const rumi_texture &t = d->textures[i];
        if (t.type == RUMI_TEX_CHECKER) continue;
        if (t.type != RUMI_TEX_IMAGE && t.type != RUMI_TEX_HDR)
            return set_error("unknown texture type"), RUMI_ERR_INVALID_ARG;
        if (t.img_width <= 0 || t.img_height <= 0 || !t.pixels ||
            (long long)t.img_width * t.img_height > (1LL << 28))
            return set_error("texture image missing or too large"), RUMI_ERR_INVALID_ARG;
        if (t.type == RUMI_TEX_IMAGE && (t.bytes_per_pixel < 3 || t.bytes_per_pixel > 4))
            return set_error("image textures need 3 or 4 bytes per pixel"), RUMI_ERR_INVALID_ARG;
    }
    auto check_tex = [&](const int32_t *a, int n) -> bool {
        if (!a) return true;
        for (int i = 0; i < n; ++i)
            if (a[i] < -1 || a[i] >= d->n_textures) return false;
        return true;
    };
    if (!check_tex(d->tri_texture, d->n_triangles) || !check_tex(d->rect_texture, d->n_rects) ||
        !check_tex(d->sphere_texture, d->n_spheres))
        return set_error("texture index out of range"), RUMI_ERR_INVALID_ARG;
    return RUMI_OK;
}

// Textures: DevTexture table, pixel arrays, per-primitive texture index and sphere frames.
// Nothing is allocated for a scene without textures.
static rumi_status upload_textures(rumi_scene *sc, const rumi_scene_desc *d, cudaStream_t s) {
    if (!has_textures(*d)) return RUMI_OK;
    std::vector<DevTexture> tex(d->n_textures);
    for (int i = 0; i < d->n_textures; ++i) {
        const rumi_texture &t = d->textures[i];
        tex[i] = make_texture(t);
        if (t.type == RUMI_TEX_CHECKER) continue;
        void *p = nullptr;
        rumi_status st = upload(&p, t.pixels, texture_pixel_bytes(t), s);
        if (p) sc->tex_pixels.push_back(p);
        if (st != RUMI_OK) return st;
        if (t.type == RUMI_TEX_HDR)
            tex[i].hdr = (const float *)p;
        else
            tex[i].img = (const unsigned char *)p;
    }
    std::vector<int> prim_tex;
    std::vector<float4> frame;
    texture_tables(*d, prim_tex, frame);
    const int nS = d->n_spheres;
    rumi_status st;
    if ((st = upload(&sc->textures, tex.data(), sizeof(DevTexture) * tex.size(), s)) != RUMI_OK) return st;
    if ((st = upload(&sc->prim_tex, prim_tex.data(), sizeof(int) * prim_tex.size(), s)) != RUMI_OK) return st;
    if (nS > 0 && (st = upload(&sc->sphere_frame, frame.data(), sizeof(float4) * frame.size(), s)) != RUMI_OK)
        return st;
    return RUMI_OK;
}

// tri_shade[3i..3i+2] = (n0, material), (n1, 0), (n2, 0); without normals the face
// normal Normalize(Cross(v1 - v0, v2 - v0)) as Model::LoadObjectFile computes it
// (src/Shape/model.cpp:320-323), with correctly rounded operations.
__global__ void pack_tri_shade_kernel(const float *verts, const float *nrm, const int *mat, int n, float4 *out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float3 n0, n1, n2;
        if (nrm) {
            const float *q = nrm + 9 * (size_t)i;
            n0 = make_float3(q[0], q[1], q[2]);
            n1 = make_float3(q[3], q[4], q[5]);
            n2 = make_float3(q[6], q[7], q[8]);
        } else {
            const float *v = verts + 9 * (size_t)i;
            const float3 v0 = make_float3(v[0], v[1], v[2]);
            const float3 e1 = rn_sub(make_float3(v[3], v[4], v[5]), v0), e2 = rn_sub(make_float3(v[6], v[7], v[8]), v0);
            n0 = n1 = n2 = normalize_ref(rn_cross(e1, e2));
        }
        out[3 * (size_t)i + 0] = make_float4(n0.x, n0.y, n0.z, __int_as_float(mat[i]));
        out[3 * (size_t)i + 1] = make_float4(n1.x, n1.y, n1.z, 0.0f);
        out[3 * (size_t)i + 2] = make_float4(n2.x, n2.y, n2.z, 0.0f);
    }
}

__global__ void pack_albedo_kernel(const float *a, int n, float4 *out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = make_float4(a[3 * (size_t)i], a[3 * (size_t)i + 1], a[3 * (size_t)i + 2], 0.0f);
}

}  // namespace

namespace rumi {

void pack_albedo(const float *a_dev, int n, float4 *out, cudaStream_t s) {
    const int grid = n < 256 * 1184 ? (n + 255) / 256 : 1184;
    if (n > 0) pack_albedo_kernel<<<grid, 256, 0, s>>>(a_dev, n, out);
}

}  // namespace rumi

extern "C" {

const char *rumi_last_error_string(void) { return g_last_error.c_str(); }

const char *rumi_version(void) { return "rumi_b200 0.1 (sm_100a)"; }

rumi_status rumi_scene_create(const rumi_scene_desc *d, rumi_scene **out) {
    if (!out) return set_error("out is NULL"), RUMI_ERR_INVALID_ARG;
    *out = nullptr;
    rumi_status st = validate(d);
    if (st != RUMI_OK) return st;
    rumi_scene *sc = new rumi_scene();
    cudaGetDevice(&sc->device);
    cudaDeviceGetAttribute(&sc->num_sms, cudaDevAttrMultiProcessorCount, sc->device);
    cudaError_t e = cudaStreamCreateWithFlags(&sc->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete sc;
        return cuda_status(e, "cudaStreamCreate");
    }
    cudaStream_t s = sc->stream;
    const int nT = d->n_triangles, nR = d->n_rects, nS = d->n_spheres;
    const int N = nT + nR + nS;
    configure_pool(sc->device);
    std::vector<float4> rects((size_t)nR * 3);
    std::vector<int> rect_emissive((size_t)nR + nS);  // prim flags: rects, then spheres
    std::vector<DevMaterial> mats(d->n_materials);
    for (int i = 0; i < d->n_materials; ++i) {
        mats[i] = make_material(d->materials[i]);
        if (mats[i].type == RUMI_MAT_SUBSURFACE) sc->has_subsurface = true;
    }
    for (int i = 0; i < nR; ++i) {
        const float *r = d->rects + 9 * (size_t)i;
        int mi = d->rect_material[i];
        float mif;
        memcpy(&mif, &mi, 4);
        rects[3 * i + 0] = make_float4(r[0], r[1], r[2], mif);
        rects[3 * i + 1] = make_float4(r[3], r[4], r[5], 0.0f);
        rects[3 * i + 2] = make_float4(r[6], r[7], r[8], 0.0f);
        const DevMaterial &m = mats[mi];
        // Rect::Intersect's one-sided test keys on Le() != Color() (rect.cpp:80-81)
        rect_emissive[i] = m.type == RUMI_MAT_EMISSIVE && (m.le.x != 0.0f || m.le.y != 0.0f || m.le.z != 0.0f);
    }
    std::vector<float4> spheres(nS);
    for (int i = 0; i < nS; ++i) {
        spheres[i] = make_float4(d->spheres[4 * i], d->spheres[4 * i + 1], d->spheres[4 * i + 2], d->spheres[4 * i + 3]);
        rect_emissive[(size_t)nR + i] = sphere_is_ibl(*d, mats.data(), i);
    }
    std::vector<DevLight> lights(d->n_lights);
    for (int i = 0; i < d->n_lights; ++i) {
        lights[i] = make_light(*d, d->lights[i], mats.data());
        if (d->lights[i].type == RUMI_LIGHT_IBL) sc->has_ibl = true;
    }
    DevScene &ds = sc->dev;
    memset(&ds, 0, sizeof(ds));
    ds.width = d->width;
    ds.height = d->height;
    ds.n_tris = nT;
    ds.n_rects = nR;
    ds.n_spheres = nS;
    ds.n_prims = N;
    ds.n_materials = d->n_materials;
    ds.n_lights = d->n_lights;
    // volume
    if (d->volume.present) fill_dev_volume(ds.volume, d->volume);
    // camera
    fill_dev_camera(ds.camera, d->camera);
    // ---- uploads
    float *d_tri_v = nullptr, *d_tri_n = nullptr, *d_alb = nullptr;
    int *d_rect_em = nullptr, *d_tri_m = nullptr;
    void *scratch = nullptr;
    auto fail = [&](rumi_status code) {
        dfree(d_tri_v, s);
        dfree(d_tri_n, s);
        dfree(d_tri_m, s);
        dfree(d_alb, s);
        dfree(d_rect_em, s);
        dfree(scratch, s);
        free_scene(sc);
        return code;
    };
    const int pack_grid = nT > 0 ? (nT + 255) / 256 < sc->num_sms * 8 ? (nT + 255) / 256 : sc->num_sms * 8 : 1;
    if ((st = upload(&d_tri_v, d->tri_vertices, sizeof(float) * 9 * (size_t)nT, s)) != RUMI_OK) return fail(st);
    if (nT > 0) {
        if (d->tri_normals &&
            (st = upload(&d_tri_n, d->tri_normals, sizeof(float) * 9 * (size_t)nT, s)) != RUMI_OK)
            return fail(st);
        if ((st = upload(&d_tri_m, d->tri_material, sizeof(int) * (size_t)nT, s)) != RUMI_OK) return fail(st);
        e = dalloc((void **)&sc->tri_shade, sizeof(float4) * 3 * (size_t)nT, s);
        if (e != cudaSuccess) return fail(cuda_status(e, "device allocation"));
        pack_tri_shade_kernel<<<pack_grid, 256, 0, s>>>(d_tri_v, d_tri_n, d_tri_m, nT, sc->tri_shade);
        if (d->tri_albedo) {
            if ((st = upload(&d_alb, d->tri_albedo, sizeof(float) * 3 * (size_t)nT, s)) != RUMI_OK) return fail(st);
            e = dalloc((void **)&sc->tri_albedo, sizeof(float4) * (size_t)nT, s);
            if (e != cudaSuccess) return fail(cuda_status(e, "device allocation"));
            pack_albedo_kernel<<<pack_grid, 256, 0, s>>>(d_alb, nT, sc->tri_albedo);
        }
    }
    if ((st = upload(&sc->rects, rects.data(), sizeof(float4) * rects.size(), s)) != RUMI_OK) return fail(st);
    if ((st = upload(&d_rect_em, rect_emissive.data(), sizeof(int) * rect_emissive.size(), s)) != RUMI_OK)
        return fail(st);
    if ((st = upload(&sc->spheres, spheres.data(), sizeof(float4) * spheres.size(), s)) != RUMI_OK) return fail(st);
    if ((st = upload(&sc->sphere_mat, d->sphere_material, sizeof(int) * (size_t)nS, s)) != RUMI_OK) return fail(st);
    if ((st = upload(&sc->materials, mats.data(), sizeof(DevMaterial) * mats.size(), s)) != RUMI_OK) return fail(st);
    if ((st = upload(&sc->lights, lights.data(), sizeof(DevLight) * lights.size(), s)) != RUMI_OK) return fail(st);
    if ((st = upload_textures(sc, d, s)) != RUMI_OK) return fail(st);
    // ---- BVH
    sc->n_nodes = bvh_node_capacity(N);
    e = dalloc((void **)&sc->nodes, sizeof(BvhNode) * (size_t)sc->n_nodes, s);
    if (e != cudaSuccess) return fail(cuda_status(e, "device allocation (nodes)"));
    e = dalloc((void **)&sc->leaf_prims, sizeof(float4) * 3 * (size_t)(N > 0 ? N : 1), s);
    if (e != cudaSuccess) return fail(cuda_status(e, "device allocation (primitives)"));
    e = dalloc(&scratch, bvh_scratch_bytes(N), s);
    if (e != cudaSuccess) return fail(cuda_status(e, "device allocation (BVH scratch)"));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    int rc = bvh_build(d_tri_v, nT, sc->rects, d_rect_em, nR, sc->spheres, nS, sc->nodes, sc->leaf_prims, scratch, s,
                       &sc->info);
    if (rc != 0) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rc > 0) return fail(cuda_status((cudaError_t)rc, "bvh_build"));
        set_error("bvh_build: internal limit reached");
        return fail(RUMI_ERR_INTERNAL);
    }
    if (RUMI_BVH_WIDE) {
        // four-wide tree: collapse into a worst-case array, then keep an exact copy
        const int cap4 = bvh4_node_capacity(N);
        Bvh4Node *tmp4 = nullptr;
        void *scratch4 = nullptr;
        e = dalloc((void **)&tmp4, sizeof(Bvh4Node) * (size_t)cap4, s);
        if (e == cudaSuccess) e = dalloc(&scratch4, bvh4_scratch_bytes(N), s);
        int n4 = -1;
        if (e == cudaSuccess) n4 = bvh4_collapse(sc->nodes, sc->n_nodes, tmp4, cap4, scratch4, s);
        if (e == cudaSuccess && n4 > 0) e = dalloc((void **)&sc->nodes4, sizeof(Bvh4Node) * (size_t)n4, s);
        if (e == cudaSuccess && n4 > 0)
            e = cudaMemcpyAsync(sc->nodes4, tmp4, sizeof(Bvh4Node) * (size_t)n4, cudaMemcpyDeviceToDevice, s);
        dfree(tmp4, s);
        dfree(scratch4, s);
        if (e != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return fail(cuda_status(e, "four-wide BVH"));
        }
        if (n4 <= 0) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            set_error("four-wide BVH collapse failed");
            return fail(RUMI_ERR_INTERNAL);
        }
        sc->n_nodes4 = n4;
    }
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    sc->build_ms = ms;
    dfree(d_tri_v, s);
    dfree(d_tri_n, s);
    dfree(d_tri_m, s);
    dfree(d_alb, s);
    dfree(d_rect_em, s);
    dfree(scratch, s);
    d_tri_v = d_tri_n = d_alb = nullptr;
    d_rect_em = d_tri_m = nullptr;
    scratch = nullptr;
    ds.nodes = sc->nodes;
    ds.nodes4 = sc->nodes4;
    ds.n_nodes4 = sc->n_nodes4;
    ds.nodes8 = sc->nodes8;
    ds.prims8 = sc->prims8;
    ds.n_nodes8 = sc->n_nodes8;
    ds.leaf_prims = sc->leaf_prims;
    ds.tri_shade = sc->tri_shade;
    ds.tri_albedo = sc->tri_albedo;
    ds.rects = sc->rects;
    ds.spheres = sc->spheres;
    ds.sphere_mat = sc->sphere_mat;
    ds.materials = sc->materials;
    ds.lights = sc->lights;
    ds.n_nodes = sc->n_nodes;
    ds.textures = sc->textures;
    ds.prim_tex = sc->prim_tex;
    ds.sphere_frame = sc->sphere_frame;
    ds.n_textures = sc->textures ? d->n_textures : 0;
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(cuda_status(e, "scene upload"));
    if (uses_bvh8(0)) {  // the default walk is the eight-wide one: its tree is needed at once
        const rumi_status st8 = ensure_bvh8(sc);
        if (st8 != RUMI_OK) return fail(st8);
    }
    *out = sc;
    return RUMI_OK;
}

rumi_status rumi_scene_destroy(rumi_scene *scene) {
    free_scene(scene);
    return RUMI_OK;
}

rumi_status rumi_scene_bvh_info(const rumi_scene *sc, rumi_bvh_info *info) {
    if (!sc || !info) return set_error("NULL argument"), RUMI_ERR_INVALID_ARG;
    info->large_levels = sc->info.large_levels;
    info->small_tasks = sc->info.small_tasks;
    info->n_nodes = sc->n_nodes;
    info->build_ms = sc->build_ms;
    return RUMI_OK;
}

rumi_status rumi_render(rumi_scene *sc, const rumi_render_params *p, float *film, int32_t film_on_device,
                        rumi_render_stats *stats) {
    if (!sc || !p || !film) return set_error("NULL argument"), RUMI_ERR_INVALID_ARG;
    if (p->spp <= 0) return set_error("spp must be positive"), RUMI_ERR_INVALID_ARG;
    cudaStream_t s = p->stream ? (cudaStream_t)p->stream : sc->stream;
    const size_t film_bytes = sizeof(float) * 3 * (size_t)sc->dev.width * sc->dev.height;
    float *film_dev = film;
    float *tmp = nullptr;
    if (!film_on_device) {
        cudaError_t e = dalloc((void **)&tmp, film_bytes, s);
        if (e != cudaSuccess) return cuda_status(e, "device allocation (film)");
        film_dev = tmp;
    }
    rumi_status st;
    if (p->integrator == RUMI_PATH_TRACER || p->integrator == RUMI_RAY_TRACER) {
        // a path has at least one vertex; the ray tracer's depth limit may be 0 (camera rays only)
        if (p->max_depth < (p->integrator == RUMI_PATH_TRACER ? 1 : 0)) {
            dfree(tmp, s);
            return set_error("max_depth out of range"), RUMI_ERR_INVALID_ARG;
        }
        st = pt_render(sc, p, film_dev, stats, s);
    } else if (p->integrator == RUMI_BDPT) {
        st = bdpt_render(sc, p, film_dev, stats, s);
    } else {
        dfree(tmp, s);
        return set_error("unknown integrator"), RUMI_ERR_INVALID_ARG;
    }
    if (st == RUMI_OK && !film_on_device) {
        cudaError_t e = cudaMemcpyAsync(film, film_dev, film_bytes, cudaMemcpyDeviceToHost, s);
        dfree(tmp, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_status(e, "film copy");
    } else {
        dfree(tmp, s);
    }
    return st;
}

rumi_status rumi_trace_rays(rumi_scene *sc, int64_t n, const float *rays, int32_t anyhit, float *t, int32_t *prim,
                            int32_t on_device, int64_t *node_visits, int64_t *prim_tests, void *stream) {
    if (!sc || n < 0 || (n > 0 && (!rays || !t || !prim))) return set_error("bad argument"), RUMI_ERR_INVALID_ARG;
    cudaStream_t s = stream ? (cudaStream_t)stream : sc->stream;
    if (on_device) return trace_rays(sc, n, rays, anyhit, t, prim, node_visits, prim_tests, s);
    float *dr = nullptr, *dt = nullptr;
    int32_t *dp = nullptr;
    rumi_status st = RUMI_OK;
    cudaError_t e = dalloc((void **)&dr, sizeof(float) * 8 * (size_t)(n > 0 ? n : 1), s);
    if (e == cudaSuccess) e = dalloc((void **)&dt, sizeof(float) * (size_t)(n > 0 ? n : 1), s);
    if (e == cudaSuccess) e = dalloc((void **)&dp, sizeof(int32_t) * (size_t)(n > 0 ? n : 1), s);
    if (e != cudaSuccess) st = cuda_status(e, "device allocation (rays)");
    if (st == RUMI_OK) {
        cudaMemcpyAsync(dr, rays, sizeof(float) * 8 * (size_t)n, cudaMemcpyHostToDevice, s);
        st = trace_rays(sc, n, dr, anyhit, dt, dp, node_visits, prim_tests, s);
    }
    if (st == RUMI_OK) {
        cudaMemcpyAsync(t, dt, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(prim, dp, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_status(e, "trace copy");
    }
    dfree(dr, s);
    dfree(dt, s);
    dfree(dp, s);
    cudaStreamSynchronize(s);
    return st;
}

}  // extern "C"
