// Host build of the path tracer's kernels (rumi-renderer_b200/csrc/pt.cu): generation,
// closest-hit and any-hit traversal (each queue walked ray by ray), and shading, compiled by
// g++ as plain C++ and run in the launch order of the library's serial schedule, so the CPU
// tests can run them under AddressSanitizer and UndefinedBehaviorSanitizer and compare the
// shading kernel's two instantiations (general and lean) on the same scenes.  On the host
// nothing contracts multiply-adds, so the two must agree bit for bit wherever the lean one
// applies.  Test infrastructure, not part of the library.
//
// One emulated thread is one block of one thread: the shading kernel's block-wide
// direction grouping then degenerates to the ray itself (a path's result does not depend on
// its queue position), and each warp operation sees one lane.
#include "cuda_host_shim.h"
#include "../../rumi-renderer_b200/csrc/pt.cu"

using namespace rumi;

#include <cstdlib>

#include "host_scene.h"

using namespace host_build;

namespace {

template <typename F>
void each_thread(long long n, F f) {
    blockDim = {1, 1, 1};
    threadIdx.x = 0;
    for (long long j = 0; j < n; ++j) {
        blockIdx.x = (unsigned)j;
        f();
    }
}

template <typename F>
void one_thread(F f) {
    blockDim = {1, 1, 1};
    threadIdx.x = 0;
    blockIdx.x = 0;
    f();
}

}  // namespace

extern "C" {

// Renders one frame (one wave of every pixel's samples) with the path tracer or the
// Whitted ray tracer.  lean: -1 picks the shading instantiation as the library does, 0 the
// general one, 1 the lean one (only for scenes it applies to).
//   film  : width * height * 3 floats (B, G, R sums over the pixel's samples)
//   stats : the wave's counters (S_NUM unsigned 64-bit values), may be NULL
// Returns 0, -1 for a description this build does not cover, -2 for bad arguments.
int rumi_host_pt(const rumi_scene_desc *d, int integrator, int max_depth, int spp, uint64_t seed, int lean,
                 float *film, unsigned long long *stats) {
    if (!d || !film || spp < 1 || max_depth < 1) return -2;
    HostScene H;
    if (build_scene(*d, H) != 0) return -1;
    // shade_lean's rule (renderer.h)
    const bool can_lean = !H.dev.volume.present && !H.dev.prim_tex && !H.has_ibl && !H.has_subsurface;
    if (lean == 1 && !can_lean) return -2;
    const bool use_lean = lean < 0 ? can_lean : lean == 1;
    const long long n_pix = (long long)d->width * d->height;
    const size_t Wp = (size_t)(n_pix * spp);
    const size_t bytes = pt_workspace_bytes((long long)Wp);
    void *ws = std::aligned_alloc(256, (bytes + 255) & ~(size_t)255);
    if (!ws) return -2;
    memset(ws, 0, bytes);
    PtLaunch L;
    carve_wave(L, ws, Wp);
    L.s = H.dev;
    L.spp = spp;
    const bool whitted = integrator == RUMI_RAY_TRACER;
    const int bounces = whitted ? max_depth + 1 : max_depth;
    L.max_depth = bounces;
    L.k0 = (uint32_t)seed;
    L.k1 = (uint32_t)(seed >> 32) ^ 0x5851F42Du;
    int g = 0;
    while ((g + 1) * (g + 1) <= spp) ++g;
    L.grid_d = g;
    L.square = g * g == spp;
    std::vector<float> dev_film((size_t)n_pix * 3, 0.0f);
    L.film = dev_film.data();
    L.refill_min = 8;
    L.pix0 = 0;
    L.n_pix = (int)n_pix;
    L.n_paths = (int)Wp;
    L.path0 = 0;
    each_thread(L.n_paths, [&] { pt_generate(L); });
    for (int b = 0; b < bounces; ++b) {
        one_thread([&] { pt_reset(L, b); });
        one_thread([&] { pt_extend<3, false, 16>(L, b); });
        if (whitted)
            each_thread(L.n_paths, [&] { pt_shade_whitted(L, b); });
        else if (use_lean)
            each_thread(L.n_paths, [&] { pt_shade<false, true>(L, b); });
        else
            each_thread(L.n_paths, [&] { pt_shade<false>(L, b); });
        one_thread([&] { pt_shadow<3, false, 16>(L); });
    }
    one_thread([&] { pt_finish(L); });
    // pt_resolve's sums, in its order (a warp per pixel adds the samples in index order)
    for (long long q = 0; q < n_pix; ++q) {
        float ax = 0.0f, ay = 0.0f, az = 0.0f;
        for (int s = 0; s < spp; ++s) {
            const float4 l = L.L[(size_t)q * spp + s];
            if (l.x != l.x || l.y != l.y || l.z != l.z) continue;
            ax += l.x; ay += l.y; az += l.z;
        }
        film[3 * q + 0] = az;
        film[3 * q + 1] = ay;
        film[3 * q + 2] = ax;
    }
    if (stats) memcpy(stats, L.stats, sizeof(unsigned long long) * S_NUM);
    std::free(ws);
    return 0;
}

}  // extern "C"
