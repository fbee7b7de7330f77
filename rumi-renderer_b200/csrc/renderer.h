// Host-side owner of a scene's device allocations and the render entry points.
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include "../../include/rumi_b200.h"
#include "scene.cuh"
#include "bvh_build.h"
#include "scene_host.h"

// Paths in flight per wave when the caller passes wave_paths = 0: 2^25 (5.9 GB of path
// tracer wave state at 176 bytes per path; a frame with fewer paths takes one wave of
// its own size).  Every bounce of a wave is one persistent launch per kernel, and a
// launch's tail (SMs idle while its last rays finish) is a smaller share of a longer
// launch: the 1024x1024, 64 spp, depth-10 frame of the 1M-triangle workload renders in
// 161 ms at 2^25 paths per wave against 184 ms at 2^22.
static constexpr long long RUMI_DEFAULT_WAVE_PATHS = 1LL << 25;

struct rumi_scene {
    DevScene dev;
    // owned device allocations
    BvhNode *nodes = nullptr;
    Bvh4Node *nodes4 = nullptr;
    int n_nodes4 = 0;
    Bvh8Node *nodes8 = nullptr;
    float4 *prims8 = nullptr;
    int n_nodes8 = 0;
    float4 *leaf_prims = nullptr;
    float4 *tri_shade = nullptr;
    float4 *tri_albedo = nullptr;
    float4 *rects = nullptr;
    float4 *spheres = nullptr;
    int *sphere_mat = nullptr;
    DevMaterial *materials = nullptr;
    DevLight *lights = nullptr;
    DevTexture *textures = nullptr;
    int *prim_tex = nullptr;
    float4 *sphere_frame = nullptr;
    std::vector<void *> tex_pixels;  // one device array per image texture
    bool has_ibl = false;
    bool has_subsurface = false;  // a Subsurface material (its random walk runs in shading)
    // the any-hit launch of a bounce runs beside the next bounce's closest-hit launch
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // per-path radiance kept by rumi_forward (RUMI_FLAG_KEEP_RADIANCE) for rumi_backward
    float4 *kept_L = nullptr;
    long long kept_cap = 0;
    bool kept_valid = false;
    uint64_t kept_seed = 0;
    int kept_spp = 0, kept_depth = 0;
    int n_nodes = 0;
    rumi::BvhBuildInfo info{};
    double build_ms = 0.0;
    cudaStream_t stream = nullptr;
    int device = 0;
    int num_sms = 148;
    // render workspace, grown on demand
    void *ws = nullptr;
    size_t ws_bytes = 0;
};

// A scene without a medium, textures, image-based lights or subsurface materials: its
// forward shading runs the instantiation with those branches compiled out.
inline bool shade_lean(const rumi_scene *sc) {
    return !sc->dev.volume.present && !sc->dev.prim_tex && !sc->has_ibl && !sc->has_subsurface;
}

namespace rumi {

struct BatchWave {
    long long pix0, pix1, path0, path1;  // global pixel / path ranges of one wave
};

// One frame of a multi-scene batch (device tables; `waves` on the host).
struct BatchFrame {
    bool lean = false;  // every scene qualifies for the lean shading instantiation (shade_lean)
    const DevScene *scenes;
    const long long *scene_path0, *scene_pix0;
    const uint32_t *scene_key;
    const int *scene_spp;
    int n_scenes;
    int max_depth;
    long long wave_paths;
    int blocks_per_sm;
    std::vector<BatchWave> waves;
};

size_t pt_adjoint_workspace_bytes(long long paths);
rumi_status pt_backward(rumi_scene *sc, const rumi_render_params *p, const float *dfilm_dev, float *g_albedo,
                        float *g_medium, rumi_render_stats *stats, cudaStream_t stream);
size_t pt_batch_workspace_bytes(long long wave_paths);
// aux, ev_fork, ev_join: the batch's second stream and its events for the two-stream
// schedule (aux == nullptr: every launch in order on `stream`)
rumi_status pt_enqueue_batch(const BatchFrame &F, void *ws, float *films, cudaStream_t stream, int num_sms,
                             cudaStream_t aux = nullptr, cudaEvent_t ev_fork = nullptr, cudaEvent_t ev_join = nullptr);
unsigned long long *pt_batch_stats_ptr(void *ws, long long wave_paths);

void set_error(const std::string &msg);
void pack_albedo(const float *a_dev, int n, float4 *out, cudaStream_t s);
rumi_status cuda_status(cudaError_t e, const char *what);

rumi_status pt_render(rumi_scene *sc, const rumi_render_params *p, float *film_dev, rumi_render_stats *stats,
                      cudaStream_t stream, float4 *keep_L = nullptr);
size_t pt_workspace_bytes(long long paths);
rumi_status bdpt_render(rumi_scene *sc, const rumi_render_params *p, float *film_dev, rumi_render_stats *stats,
                        cudaStream_t stream);
// overlap: run each bounce's any-hit launch on the scene's auxiliary stream beside the
// next bounce's closest-hit launch (false: one stream, in order)
// keep_L: when set, every wave's per-path radiance is copied there at global path index
// pixel * spp + sample
rumi_status pt_render_in(rumi_scene *sc, const rumi_render_params *p, float *film_dev, rumi_render_stats *stats,
                         cudaStream_t stream, void *ws, long long pix_per_wave, bool overlap = false,
                         float4 *keep_L = nullptr);
rumi_status trace_rays(rumi_scene *sc, int64_t n, const float *rays_dev, int anyhit, float *t_dev, int32_t *prim_dev,
                       int64_t *node_visits, int64_t *prim_tests, cudaStream_t stream);
rumi_status trace_rays_scheme(rumi_scene *sc, int64_t n, const float *rays_dev, int anyhit, int trace_mode,
                              float *t_dev, int32_t *prim_dev, cudaStream_t stream);
rumi_status ensure_workspace(rumi_scene *sc, size_t bytes);
// builds the eight-wide tree on first use (trace_mode 5); a no-op once built
rumi_status ensure_bvh8(rumi_scene *sc);
// true when trace_mode selects the eight-wide walk
bool uses_bvh8(int trace_mode);
cudaError_t dalloc(void **p, size_t bytes, cudaStream_t s);
void dfree(void *p, cudaStream_t s);
void configure_pool(int device);

}  // namespace rumi
