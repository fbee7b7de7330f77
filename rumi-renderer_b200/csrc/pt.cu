// Wavefront path tracer with next-event estimation.
//
// The reference's PathTracer::Trace(w, h, ...) (src/Integrator/pathtracer.cpp:117-354)
// walks forward recording a vertex chain, then accumulates backwards
//     L_k = A_k * (direct_k + vol_k * fr_k * L_{k+1} * cos_k / Average(pdf_wi_k * pdf_path_k))
// (A_k: medium factor of the arriving segment).  Expanding the recursion gives the
// forward estimator used here: L = sum_k beta_k * direct_k with
//     beta_{k+1} = beta_k * vol_k * fr_k * cos_k / Average(pdf_wi_k * pdf_path_k),
// which lets every bounce run as independent kernels over queues of rays:
//
//   generate  camera rays (Pinhole::CastViewRay, the reference's pixel sampler)
//   extend    closest hit of every queued ray            (persistent, work-fetching)
//   shade     medium free flight, emission, BSDF sample, NEE; compacts the next
//             bounce's rays and this bounce's shadow rays with warp-aggregated atomics
//   shadow    any-hit test of the shadow rays; adds their contribution
//   resolve   per-pixel sum of the samples in sample order (NaN samples dropped and
//             counted, src/Scene/scene.cpp:229-241)
//
// Random numbers: Philox4x32-10 keyed by the seed, counter (path, bounce, group); a
// path's stream does not depend on the wave size or launch order.
#include "renderer.h"
#include "traverse.cuh"
#include "shading.cuh"
#include "camera.cuh"
#include <vector>
#include <type_traits>

namespace rumi {

static constexpr int TRACE_THREADS = 128;
// Minimum resident traversal blocks per SM: 8 caps the extend / shadow kernels at 64
// registers (32 warps per SM instead of 28 at their natural 72); measured 5% faster per
// frame on the 1M-triangle workload.  10 and 12 spill and are slower.  The any-hit kernel
// alone (55 registers at 8) measured 83.2 / 84.9 / 122.0 ms per frame at 9 / 10 / 12
// blocks against 83.6 at 8.
#ifndef RUMI_TRACE_MIN_BLOCKS
#define RUMI_TRACE_MIN_BLOCKS 8
#endif
#ifndef RUMI_EXTEND_MIN_BLOCKS
#define RUMI_EXTEND_MIN_BLOCKS RUMI_TRACE_MIN_BLOCKS
#endif
#ifndef RUMI_SHADOW_MIN_BLOCKS
#define RUMI_SHADOW_MIN_BLOCKS RUMI_TRACE_MIN_BLOCKS
#endif
// The default walk (scheme 3, the speculative while-while walk over the binary tree) at 9
// blocks: 56 registers with a 38-byte spill (closest-hit) and 55 without one (any-hit);
// per 1024x1024x64 frame 83.3 / 44.5 ms of closest-hit / any-hit against 83.8 / 45.7 at 8.
#ifndef RUMI_WW_MIN_BLOCKS
#define RUMI_WW_MIN_BLOCKS 9
#endif
static constexpr int trace_min_blocks(int mode, bool extend) {
    return mode == 3 ? RUMI_WW_MIN_BLOCKS : (extend ? RUMI_EXTEND_MIN_BLOCKS : RUMI_SHADOW_MIN_BLOCKS);
}
// 1: each bounce's any-hit launch runs on an auxiliary stream beside the next bounce's
// closest-hit launch (pt_render_in); 0: one stream, launches in order.
#ifndef RUMI_PT_OVERLAP
#define RUMI_PT_OVERLAP 1
#endif
static constexpr int STACK_SMEM = 32;
// Threads per block of the shading kernels; a block groups its next rays by direction, so
// the block size is also the grouping's width (128: shading 0.5 ms faster per frame,
// closest-hit 0.5 ms slower).
#ifndef RUMI_SHADE_THREADS
#define RUMI_SHADE_THREADS 256
#endif
static constexpr int SHADE_THREADS = RUMI_SHADE_THREADS;

enum { PFL_LE = 1, PFL_IN = 2 };
// A queued ray's o.w holds its path slot (bits 0-29) and its flags: bit 31 = in_object
// (read by the traversal), bit 30 = le.  Its throughput travels in the queue too
// (beta_q, same position), so shading reads and writes path state in queue order.
RUMI_D float pack_slot(int slot, unsigned fl) {
    return __int_as_float(slot | ((fl & PFL_IN) ? (int)0x80000000 : 0) | ((fl & PFL_LE) ? 0x40000000 : 0));
}
RUMI_D int slot_of(float w) { return __float_as_int(w) & 0x3fffffff; }
RUMI_D unsigned flags_of(float w) {
    const unsigned b = __float_as_uint(w);
    return ((b >> 31) ? PFL_IN : 0u) | (((b >> 30) & 1u) ? PFL_LE : 0u);
}
// counters
enum { C_RAY0 = 0, C_RAY1 = 1, C_SHADOW = 2, C_FETCH_EXT = 3, C_FETCH_SH = 4, C_NUM = 8 };
// 64-bit device statistics
enum { S_RAYS_EXT = 0, S_RAYS_SH = 1, S_NAN = 2, S_NODES = 3, S_PRIMS = 4, S_NUM = 8 };

struct PtLaunch {
    DevScene s;
    int spp, max_depth;
    uint32_t k0, k1;
    int grid_d, square;
    long long path0;
    int n_paths, pix0, n_pix;
    float4 *ray_o[2], *ray_d[2], *hit;
    float4 *sh_o, *sh_d, *sh_c;
    float4 *beta_q[2], *L;  // beta_q: throughput (+ one word) in queue order, per ray buffer
    int *cnt;
    unsigned long long *stats;
    float *film;
    int refill_min;
    // multi-scene batches (scenes == nullptr: the single scene s)
    const DevScene *scenes;
    const long long *scene_path0;  // n_scenes + 1 prefix: first global path of each scene
    const long long *scene_pix0;   // n_scenes + 1 prefix: first global pixel of each scene
    const uint32_t *scene_key;     // Philox key per scene (2 words)
    const int *scene_spp;
    int n_scenes;
    int *slot_scene;               // scene of each wave slot
    // path-replay adjoint (dls == nullptr: plain rendering)
    const float4 *Lt;              // per slot: the path's radiance from the first pass
    float4 *dls;                   // per slot: dLoss / d(path radiance), RGB (0 for NaN paths)
    const float *dfilm;            // dLoss / dfilm, H*W*3 in B,G,R order
    float2 *sh_s;                  // per shadow ray: (d log / d sigma coefficient, d log / d g)
    float *g_albedo;               // n_tris * 3 RGB, or nullptr
    float *g_medium;               // 7: sigma_s rgb, sigma_a rgb, g
};

// Parameter order of the medium gradient.
enum { GM_SIGMA_S = 0, GM_SIGMA_A = 3, GM_G = 6, GM_NUM = 7 };

// d/dg log p_HG(cos; g): the score of a direction drawn from (or weighted by) the
// Henyey-Greenstein phase function.
RUMI_D float hg_dlog_dg(float c, float g) {
    const float denom = 1.0f + g * g - 2.0f * g * c;
    return -2.0f * g / (1.0f - g * g) - 3.0f * (g - c) / denom;
}

// Sums `v` over the lanes of the warp that share `key` (>= 0) and adds the sums to
// base[3 * key + 0..2] with one atomic per group.  Called by all 32 lanes.
RUMI_D void warp_add3_by_key(float *base, int key, float3 v) {
    const unsigned act = __ballot_sync(0xffffffffu, key >= 0);
    if (key < 0) return;
    const unsigned grp = __match_any_sync(act, key);
    float3 acc = mk3(0.0f, 0.0f, 0.0f);
    unsigned m = grp;
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        acc.x += __shfl_sync(grp, v.x, src);
        acc.y += __shfl_sync(grp, v.y, src);
        acc.z += __shfl_sync(grp, v.z, src);
    }
    if ((int)(threadIdx.x & 31) == __ffs(grp) - 1) {
        atomicAdd(base + 3 * key + 0, acc.x);
        atomicAdd(base + 3 * key + 1, acc.y);
        atomicAdd(base + 3 * key + 2, acc.z);
    }
}

RUMI_D float warp_sum(float x) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Largest k with prefix[k] <= g (prefix has n + 1 ascending entries).
RUMI_D int find_scene(const long long *prefix, int n, long long g) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (prefix[mid] <= g)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

RUMI_D int isqrt_floor(int n) {
    int d = 0;
    while ((d + 1) * (d + 1) <= n) ++d;
    return d;
}

__global__ void pt_generate(PtLaunch P) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j == 0) P.cnt[C_RAY0] = P.n_paths;
    if (j >= P.n_paths) return;
    // one call site of the sampler and camera for both forms, so a batched scene's rays
    // are bit-identical to the single-scene ones
    const DevScene *S = &P.s;
    long long pixel, path = P.path0 + j;
    int s, spp = P.spp, gd = P.grid_d;
    bool square = P.square != 0;
    uint32_t k0 = P.k0, k1 = P.k1;
    if (P.scenes) {
        const long long g = P.path0 + j;
        const int k = find_scene(P.scene_path0, P.n_scenes, g);
        S = &P.scenes[k];
        spp = P.scene_spp[k];
        const long long local = g - P.scene_path0[k];
        path = local;
        pixel = local / spp;
        s = (int)(local % spp);
        gd = isqrt_floor(spp);
        square = gd * gd == spp;
        k0 = P.scene_key[2 * k];
        k1 = P.scene_key[2 * k + 1];
        P.slot_scene[j] = k;
    } else {
        pixel = (long long)P.pix0 + j / P.spp;
        s = j % P.spp;
    }
    const int W = S->width;
    const int w = (int)(pixel % W), h = (int)(pixel / W);
    const float2 smp = pixel_sample(s, spp, gd, square, pixel, k0, k1);
    float3 o, d;
    const float2 lu = S->camera.focal_distance > 0.0f ? lens_uniforms((uint64_t)path, k0, k1) : make_float2(0.f, 0.f);
    camera_ray(S->camera, W, S->height, w, h, smp.x, smp.y, lu.x, lu.y, o, d);
    P.ray_o[0][j] = make_float4(o.x, o.y, o.z, pack_slot(j, PFL_LE));
    P.ray_d[0][j] = make_float4(d.x, d.y, d.z, FLT_MAX);
    P.beta_q[0][j] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    P.L[j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (P.dls) {
        // the film drops NaN samples (pt_resolve), so they receive no gradient
        const long long px = (long long)P.pix0 + j / P.spp;
        const float4 lt = P.Lt[j];
        const bool nan = lt.x != lt.x || lt.y != lt.y || lt.z != lt.z;
        P.dls[j] = nan ? make_float4(0.0f, 0.0f, 0.0f, 0.0f)
                       : make_float4(P.dfilm[3 * px + 2], P.dfilm[3 * px + 1], P.dfilm[3 * px + 0], 0.0f);
    }
}

__global__ void pt_reset(PtLaunch P, int bounce) {
    const int cur = bounce & 1, nxt = cur ^ 1;
    P.stats[S_RAYS_EXT] += (unsigned long long)P.cnt[cur];
    if (bounce > 0) P.stats[S_RAYS_SH] += (unsigned long long)P.cnt[C_SHADOW];
    P.cnt[nxt] = 0;
    P.cnt[C_SHADOW] = 0;
    P.cnt[C_FETCH_EXT] = 0;
    P.cnt[C_FETCH_SH] = 0;
}

__global__ void pt_finish(PtLaunch P) { P.stats[S_RAYS_SH] += (unsigned long long)P.cnt[C_SHADOW]; }

// pt_reset in two halves for the overlapped schedule: before a closest-hit launch (its
// queue into the statistics, its work counter cleared), and before shading, once the
// previous bounce's shadow rays are traced (their count into the statistics, the queues
// shading pushes into cleared).
__global__ void pt_reset_extend(PtLaunch P, int bounce) {
    P.stats[S_RAYS_EXT] += (unsigned long long)P.cnt[bounce & 1];
    P.cnt[C_FETCH_EXT] = 0;
}
__global__ void pt_reset_shade(PtLaunch P, int bounce) {
    // (at bounce 0 the count is the previous wave's last bounce, which pt_finish added)
    if (bounce > 0) P.stats[S_RAYS_SH] += (unsigned long long)P.cnt[C_SHADOW];
    P.cnt[C_SHADOW] = 0;
    P.cnt[C_FETCH_SH] = 0;
    P.cnt[(bounce & 1) ^ 1] = 0;
}

// Persistent traversal kernels: every block takes rays from the bounce's queue until it
// is empty (traverse_queue in traverse.cuh; MODE selects the scheme, see there).
// SMEM: traversal stack entries per thread kept in shared memory (deeper entries spill to
// local memory); a smaller stack leaves more of the SM's unified L1/shared storage to L1.
template <int MODE, bool STATS, int SMEM = STACK_SMEM>
__global__ void __launch_bounds__(TRACE_THREADS, trace_min_blocks(MODE, true)) pt_extend(PtLaunch P, int bounce) {
    __shared__ int stack[SMEM * TRACE_THREADS];
    const int cur = bounce & 1;
    TraceStats st{0, 0};
    auto fetch = [&](int i, float3 &o, float3 &d, float &tmax, bool &in_obj) {
        const float4 o4 = P.ray_o[cur][i];
        const float4 d4 = P.ray_d[cur][i];
        o = f4xyz(o4);
        d = f4xyz(d4);
        tmax = d4.w;
        in_obj = (__float_as_uint(o4.w) >> 31) != 0;
    };
    auto finish = [&](int i, const HitRec &h) {
        const int code = h.t > 0.0f ? (h.id | (h.back ? (int)0x80000000 : 0)) : -1;
        P.hit[i] = make_float4(h.t, __int_as_float(code), h.u, h.v);
    };
    traverse_queue<MODE, false, SMEM, STATS>(P.s, P.cnt[cur], &P.cnt[C_FETCH_EXT], P.refill_min,
                                             stack + threadIdx.x, TRACE_THREADS, fetch, finish, st);
    if (STATS) {
        atomicAdd(&P.stats[S_NODES], (unsigned long long)st.nodes);
        atomicAdd(&P.stats[S_PRIMS], (unsigned long long)st.prims);
    }
}

template <int MODE, bool ADJ = false, int SMEM = STACK_SMEM>
__global__ void __launch_bounds__(TRACE_THREADS, trace_min_blocks(MODE, false)) pt_shadow(PtLaunch P) {
    __shared__ int stack[SMEM * TRACE_THREADS];
    TraceStats st{0, 0};
    float acc_sigma = 0.0f, acc_g = 0.0f;  // adjoint: score-weighted contributions
    auto fetch = [&](int i, float3 &o, float3 &d, float &tmax, bool &in_obj) {
        const float4 o4 = P.sh_o[i];
        const float4 d4 = P.sh_d[i];
        o = f4xyz(o4);
        d = f4xyz(d4);
        tmax = d4.w;
        in_obj = false;
    };
    auto finish = [&](int i, const HitRec &h) {
        if (h.t == 0.0f) {
            const int slot = __float_as_int(P.sh_o[i].w);
            const float4 c = P.sh_c[i];
            float4 l = P.L[slot];
            l.x += c.x; l.y += c.y; l.z += c.z;
            P.L[slot] = l;
            if (ADJ) {
                // this NEE term alone carries the shadow ray's transmittance decision
                // and (in a medium) the phase function's value at the light direction
                const float4 dl = P.dls[slot];
                const float dterm = dl.x * c.x + dl.y * c.y + dl.z * c.z;
                const float2 sc = P.sh_s[i];
                acc_sigma += sc.x * dterm;
                acc_g += sc.y * dterm;
            }
        }
    };
    traverse_queue<MODE, true, SMEM, false>(P.s, P.cnt[C_SHADOW], &P.cnt[C_FETCH_SH], P.refill_min,
                                            stack + threadIdx.x, TRACE_THREADS, fetch, finish, st);
    if (ADJ) {
        __syncwarp();
        acc_sigma = warp_sum(acc_sigma);
        acc_g = warp_sum(acc_g);
        if ((threadIdx.x & 31) == 0 && (acc_sigma != 0.0f || acc_g != 0.0f)) {
            for (int k = 0; k < 6; ++k) atomicAdd(&P.g_medium[k], acc_sigma);
            atomicAdd(&P.g_medium[GM_G], acc_g);
        }
    }
}

// Multi-scene batches: the default traversal scheme (speculative while-while, the walk
// rumi_render uses) with each ray's own scene, so a batched scene resolves exact-distance
// ties exactly as its single-scene render does.
template <bool ANYHIT>
__global__ void __launch_bounds__(TRACE_THREADS, RUMI_TRACE_MIN_BLOCKS) pt_trace_multi(PtLaunch P, int bounce) {
    __shared__ int stack[STACK_SMEM * TRACE_THREADS];
    const int cur = bounce & 1;
    const int n = ANYHIT ? P.cnt[C_SHADOW] : P.cnt[cur];
    int *counter = ANYHIT ? &P.cnt[C_FETCH_SH] : &P.cnt[C_FETCH_EXT];
    TraceStats st{0, 0};
    auto scene_of = [&](int i) -> const DevScene * {
        if (i < 0) return &P.scenes[0];
        const float4 o4 = ANYHIT ? P.sh_o[i] : P.ray_o[cur][i];
        return &P.scenes[P.slot_scene[ANYHIT ? __float_as_int(o4.w) : slot_of(o4.w)]];
    };
    auto fetch = [&](int i, float3 &o, float3 &d, float &tmax, bool &in_obj) {
        const float4 o4 = ANYHIT ? P.sh_o[i] : P.ray_o[cur][i];
        const float4 d4 = ANYHIT ? P.sh_d[i] : P.ray_d[cur][i];
        o = f4xyz(o4);
        d = f4xyz(d4);
        tmax = d4.w;
        in_obj = !ANYHIT && (__float_as_uint(o4.w) >> 31) != 0;
    };
    auto finish = [&](int i, const HitRec &h) {
        if (ANYHIT) {
            if (h.t == 0.0f) {
                const int slot = __float_as_int(P.sh_o[i].w);
                const float4 c = P.sh_c[i];
                float4 l = P.L[slot];
                l.x += c.x; l.y += c.y; l.z += c.z;
                P.L[slot] = l;
            }
        } else {
            const int code = h.t > 0.0f ? (h.id | (h.back ? (int)0x80000000 : 0)) : -1;
            P.hit[i] = make_float4(h.t, __int_as_float(code), h.u, h.v);
        }
    };
    traverse_queue_walk<ANYHIT, STACK_SMEM, false>(scene_of, n, counter, P.refill_min, stack + threadIdx.x,
                                                   TRACE_THREADS, fetch, finish, st);
}

// Next-event estimation toward one light sample from p.  Returns false when the light
// faces away or lies outside a spot cone (Scene::VisibilityTest's facing test,
// src/Scene/scene.cpp:99-123).  wi / dist: the shadow ray; G: AreaLight::G.
RUMI_D bool nee_setup(const LightSample &ls, float3 p, float3 &wi, float &dist, float &G) {
    if (ls.is_ibl) {  // ImageBasedLight: Wi is the sampled direction, G = 1
        wi = ls.wi;
        const float3 dv = rn_sub(ls.P, p);
        dist = __fsqrt_rn(rn_dot(dv, dv));
        G = 1.0f;
        return rn_dot(wi, ls.nL) < 0.0f;
    }
    const float3 dv = ls.P - p;
    wi = normalize_ref(dv);
    dist = sqrtf(dot3(p - ls.P, p - ls.P));
    if (ls.is_delta) {
        if (dot3(-wi, ls.spot_dir) < ls.cos_cone) return false;
        G = 1.0f / (dist * dist);
        return true;
    }
    if (dot3(wi, ls.nL) >= 0.0f) return false;
    G = fmaxf(-dot3(wi, ls.nL), 0.0f) / (dist * dist);
    return true;
}

// ADJ: the replay pass of the path-replay adjoint (pt_backward).  Every path is traced a
// second time on the same random numbers; at each of its events the part of the path's
// radiance that the event influences -- Lt (the first pass's total) minus the terms
// already accumulated -- is weighted with dLoss/dradiance and with the event's score:
//   triangle albedo at a Lambertian vertex: d log / d rho = 1 / rho (per channel)
//   medium segment passed through:         log P = -avg(sigma_t) * s_max
//   medium scatter at distance s:          log p = log avg(sigma_t) - avg(sigma_t) s
//                                                  + log(1 - avg(sigma_a / sigma_t)),
//                                          weight sigma_s / sigma_t (per channel)
//   phase direction (applied at the next vertex) and NEE phase value: d log HG / d g
//   binary shadow transmittance (applied by the shadow kernel to that NEE term alone).
// Forward shading is bound by the latency of its scattered per-path loads: three blocks
// of 256 threads per SM (80 registers, a 120-byte spill to L1) ran the 1024x1024x64
// BVH-bound frame's shading in 31.0 ms against 37.7 ms at two blocks (118 registers);
// four blocks (64 registers) gave the same as three.  The adjoint replay keeps its
// registers.
#ifndef RUMI_SHADE_MIN_BLOCKS
#define RUMI_SHADE_MIN_BLOCKS 3
#endif
// LEAN: the instantiation for scenes without a medium, textures, image-based lights or
// subsurface materials (the host picks it only for those): the same code with the branches
// those features take compiled out, so the kernel holds fewer registers and instructions.
// Everything it executes is what the general instantiation executes for such a scene.
// The lean instantiation fits four blocks (64 registers, a 52-byte spill): 21.8 ms of
// shading per frame against 25.6 ms at three blocks (72 registers, no spill) and 27.9 ms for
// the general instantiation.
#ifndef RUMI_SHADE_LEAN_MIN_BLOCKS
#define RUMI_SHADE_LEAN_MIN_BLOCKS 4
#endif
template <bool ADJ, bool LEAN = false>
__global__ void __launch_bounds__(SHADE_THREADS, ADJ ? 1 : (LEAN ? RUMI_SHADE_LEAN_MIN_BLOCKS : RUMI_SHADE_MIN_BLOCKS))
    pt_shade(PtLaunch P, int bounce) {
    const int cur = bounce & 1, nxt = cur ^ 1;
    const int n = P.cnt[cur];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;

    bool want_next = false, want_sh = false;
    float3 nx_o = mk3(0, 0, 0), nx_d = mk3(0, 0, 0);
    unsigned nx_flags = 0;
    float3 sh_o = mk3(0, 0, 0), sh_d = mk3(0, 0, 0), sh_c = mk3(0, 0, 0);
    float sh_tmax = 0.0f;
    int slot = 0;
    float3 beta = mk3(0, 0, 0);
    float pend_g = 0.0f;                     // adjoint: score of the phase direction sampled here
    float2 sh_score = make_float2(0.0f, 0.0f);
    float gm[GM_NUM];
    int alb_key = -1;
    float3 alb_grad = mk3(0.0f, 0.0f, 0.0f);
    if (ADJ) {
#pragma unroll
        for (int k = 0; k < GM_NUM; ++k) gm[k] = 0.0f;
    }

    if (active) {
        const float4 o4 = P.ray_o[cur][i];
        const float4 d4 = P.ray_d[cur][i];
        const float4 hv = P.hit[i];
        slot = slot_of(o4.w);
        const DevScene *Sp = &P.s;
        uint32_t k0 = P.k0, k1 = P.k1;
        uint64_t path = (uint64_t)(P.path0 + slot);
        if (P.scenes) {
            const int sk = P.slot_scene[slot];
            Sp = &P.scenes[sk];
            k0 = P.scene_key[2 * sk];
            k1 = P.scene_key[2 * sk + 1];
            path = (uint64_t)(P.path0 + slot - P.scene_path0[sk]);
        }
        const DevScene &S = *Sp;
        const float3 o = f4xyz(o4), d = f4xyz(d4);
        const float t = hv.x;
        const bool hit = t > 0.0f;
        const int code = __float_as_int(hv.y);
        const unsigned fl = flags_of(o4.w);
        const bool le = (fl & PFL_LE) != 0, inobj = (fl & PFL_IN) != 0;
        const float4 beta4 = P.beta_q[cur][i];
        beta = f4xyz(beta4);
        // adjoint: radiance of the terms from this vertex on, and its loss weights
        float3 Lo = mk3(0.0f, 0.0f, 0.0f), dl = mk3(0.0f, 0.0f, 0.0f);
        float D = 0.0f;
        if (ADJ) {
            const float4 lt = P.Lt[slot], la = P.L[slot], d4 = P.dls[slot];
            Lo = mk3(lt.x - la.x, lt.y - la.y, lt.z - la.z);
            dl = f4xyz(d4);
            D = dot3(dl, Lo);
            gm[GM_G] += beta4.w * D;  // the direction sampled at the previous (medium) vertex
        }
        const Uniform4 U0 = path_uniforms(path, bounce, 0, k0, k1);
        const Uniform4 U1 = path_uniforms(path, bounce, 1, k0, k1);
        const bool last = bounce + 1 >= P.max_depth;
        float3 addL = mk3(0, 0, 0);
        bool done = false;

        // ---------------------------------------------- homogeneous medium
        const DevVolume &V = S.volume;
        if (!LEAN && V.present && !inobj) {
            float tn, tf;
            const float thit = hit ? t : 0.0f;
            if (volume_intersect(V, o, d, thit, tn, tf)) {
                const float smax = volume_max_distance(thit, tn, tf);
                const DistSample ds = distance_sample(V.sigma_t, V.avg_sigma_t, V.absorb, smax, U1.u[2], U1.u[3]);
                if (ADJ) {
                    const float third = 0.33333333333f;
                    if (ds.outcome == 0) {
                        const float c = -smax * third * D;
#pragma unroll
                        for (int k = 0; k < 6; ++k) gm[k] += c;
                    } else if (ds.outcome == 1) {
                        const float base = (third / V.avg_sigma_t - ds.s * third) * D;
                        const float inv1a = 1.0f / (1.0f - V.absorb);
                        const float ss[3] = {V.sigma_s.x, V.sigma_s.y, V.sigma_s.z};
                        const float sa[3] = {V.sigma_a.x, V.sigma_a.y, V.sigma_a.z};
                        const float st[3] = {V.sigma_t.x, V.sigma_t.y, V.sigma_t.z};
                        const float q[3] = {dl.x * Lo.x, dl.y * Lo.y, dl.z * Lo.z};
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const float t2 = 3.0f * st[c] * st[c];
                            const float ws = ss[c] > 0.0f ? 1.0f / ss[c] - 1.0f / st[c] : 0.0f;
                            gm[GM_SIGMA_S + c] += base + sa[c] / t2 * inv1a * D + ws * q[c];
                            gm[GM_SIGMA_A + c] += base - ss[c] / t2 * inv1a * D - q[c] / st[c];
                        }
                    }
                }
                if (ds.outcome == 2) {
                    done = true;  // absorbed (pathtracer.cpp:164-167)
                } else if (ds.outcome == 1) {
                    const float3 p = o + d * (tn < 0.0f ? ds.s : tn + ds.s);
                    const float3 vol = ds.tau / ds.pdf;
                    // HomogeneousVolume::DirectLighting (homogeneousvolume.cpp:231-250)
                    if (S.n_lights > 0) {
                        // the vertex keeps the normal of the surface hit beyond the scatter
                        // point (pathtracer.cpp:154-170 moves only _p); an image-based light
                        // samples about it
                        float3 nb = mk3(0.0f, 1.0f, 0.0f);
                        if (hit && S.lights[pick_light(S, U0.u[3])].type == LIGHT_IBL) {
                            const int hid = code & 0x7fffffff;
                            nb = surface_normal(S, hid, code < 0, hv.z, hv.w, o, rn_madd(o, d, t),
                                                S.materials[prim_material(S, hid)]);
                        }
                        const LightSample ls = sample_light(S, U0.u[3], U1.u[0], U1.u[1], p, nb);
                        float3 wi;
                        float dist, G;
                        if (nee_setup(ls, p, wi, dist, G)) {
                            const Uniform4 U2 = path_uniforms(path, bounce, 2, k0, k1);
                            float smax_sh = 0.0f;
                            const float tr = volume_shadow_tr(V, p, wi, dist, U2.u[2], &smax_sh);
                            if (tr > 0.0f) {
                                if (ADJ) sh_score = make_float2(-smax_sh * 0.33333333333f, hg_dlog_dg(dot3(d, wi), V.g));
                                const float fp = V.g == 0.0f ? 1.0f / (4.0f * RUMI_PI_F) : hg_eval(dot3(d, wi), V.g);
                                const float3 direct = ls.Li * tr * V.sigma_s * fp * G * (1.0f / ls.pdf);
                                want_sh = true;
                                sh_o = p;
                                sh_d = wi;
                                sh_tmax = dist;
                                sh_c = beta * vol * direct;
                            }
                        }
                    }
                    // phase sampling; Fp / pdf = sigma_s (isotropic: the reference's
                    // Fp = sigma_s / 4 pi over Average(pdf_wi) = 1 / 4 pi)
                    float pdf_phase;
                    const float3 w = V.g == 0.0f ? isotropic_dir(d, U0.u[1], U0.u[2])
                                                 : hg_sample(d, V.g, U0.u[1], U0.u[2], pdf_phase);
                    float3 fp_over_pdf;
                    if (V.g == 0.0f) {
                        const float fp = 1.0f / (4.0f * RUMI_PI_F);
                        const float pdf = avg3(mk3(fp, fp, fp));
                        fp_over_pdf = V.sigma_s * fp * (1.0f / pdf);
                    } else {
                        fp_over_pdf = V.sigma_s;
                    }
                    beta = beta * vol * fp_over_pdf;
                    if (ADJ) pend_g = hg_dlog_dg(dot3(d, w), V.g);
                    nx_o = p;
                    nx_d = w;
                    nx_flags = 0;  // le = false, in_object = false
                    want_next = !last;
                    done = true;
                }
            }
        }

        // ---------------------------------------------------- surface
        if (!done && hit) {
            const int id = code & 0x7fffffff;
            const bool back = code < 0;
            const int mi = prim_material(S, id);
            const DevMaterial m = S.materials[mi];
            float3 p = rn_madd(o, d, t);
            float3 nrm;
            float3 albedo = m.rgb;
            if (id < S.n_tris) {
                const float4 n0 = __ldg(&S.tri_shade[3 * id]), n1 = __ldg(&S.tri_shade[3 * id + 1]),
                             n2 = __ldg(&S.tri_shade[3 * id + 2]);
                const float u = hv.z, v = hv.w;
                nrm = bary_ref(f4xyz(n0), f4xyz(n1), f4xyz(n2), u, v);  // triangle.cpp:111 (Q3)
                if (back && material_opaque(m)) nrm = -nrm;
                if (S.tri_albedo) albedo = f4xyz(__ldg(&S.tri_albedo[id]));
                if (ADJ && P.g_albedo && S.tri_albedo && m.type == MAT_MATTE) {
                    // every term from this vertex on carries the factor albedo (per channel)
                    alb_key = id;
                    alb_grad = mk3(albedo.x > 0.0f ? dl.x * Lo.x / albedo.x : 0.0f,
                                   albedo.y > 0.0f ? dl.y * Lo.y / albedo.y : 0.0f,
                                   albedo.z > 0.0f ? dl.z * Lo.z / albedo.z : 0.0f);
                }
            } else if (id < S.n_tris + S.n_rects) {
                const int r = id - S.n_tris;
                nrm = normalize_ref(cross3(f4xyz(S.rects[3 * r + 1]), f4xyz(S.rects[3 * r + 2])));
            } else {
                const float4 c = S.spheres[id - S.n_tris - S.n_rects];
                const float3 cc = f4xyz(c);
                if (m.type == MAT_EMISSIVE) {
                    const float3 oc = o - cc;
                    nrm = sqrtf(dot3(oc, oc)) > c.w ? normalize_ref(p - cc) : normalize_ref(cc - p);
                } else {
                    nrm = normalize_ref(p - cc);
                }
            }
            if (m.type == MAT_EMISSIVE) {
                // Emissive::DirectLighting (emissive.cpp:61-74) times the texture
                // (pathtracer.cpp:343-344); the path ends here.
                if (le && !inobj && -dot3(d, nrm) > 0.0f) addL = LEAN ? beta * m.le : beta * m.le * tex_pattern(S, id, p);
            } else {
                const float3 wo = -d;
                BsdfSample b;
                float3 vol_ratio = mk3(1, 1, 1), volw = mk3(1, 1, 1);
                bool walk_scatter = false, absorbed = false;
                if (!LEAN && m.type == MAT_SUBSURFACE && inobj) {
                    // Subsurface::PhaseSampling (subsurface.cpp:121-142): random walk step
                    const Uniform4 U2 = path_uniforms(path, bounce, 2, k0, k1);
                    const DistSample ws = distance_sample(m.sigma_t, m.avg_sigma_t, m.absorb, t, U2.u[0], U2.u[1]);
                    if (ws.outcome == 1) {
                        walk_scatter = true;
                        p = o + d * ws.s;
                        b.w = isotropic_dir(-wo, U0.u[1], U0.u[2]);
                        b.le = true;
                        b.go_in = true;
                        b.xi = 1.0f;
                        b.pdf_path = 1.0f;
                        b.cost = 1.0f;
                        b.pdfw = 1.0f / (4.0f * RUMI_PI_F);
                        volw = ws.tau / ws.pdf * (m.rgb * (1.0f / (4.0f * RUMI_PI_F)));
                    } else if (ws.outcome == 2) {
                        absorbed = true;
                    } else {
                        vol_ratio = ws.tau / ws.pdf;
                        b = material_sample(m, wo, nrm, U0.u[0], U0.u[1], U0.u[2]);
                    }
                } else {
                    b = material_sample(m, wo, nrm, U0.u[0], U0.u[1], U0.u[2]);
                }
                // Texture::Pattern scales everything this vertex returns, its light
                // sample and what comes after it (pathtracer.cpp:343-344)
                if (!LEAN && S.prim_tex) beta = beta * tex_pattern(S, id, p);
                if (!absorbed) {
                    // NEE: Matte::DirectLighting (matte.cpp:54-82); Glossy only on its
                    // diffuse lobe, divided by kd_pdf (glossy.cpp:92-102)
                    const bool nee = S.n_lights > 0 && !walk_scatter &&
                                     (m.type == MAT_MATTE ||
                                      (m.type == MAT_GLOSSY && m.kd != 0.0f && b.xi <= m.kd_pdf));
                    if (nee) {
                        const LightSample ls = sample_light<!LEAN>(S, U0.u[3], U1.u[0], U1.u[1], p, nrm);
                        float3 wi;
                        float dist, G;
                        if (nee_setup(ls, p, wi, dist, G)) {
                            const float3 f = albedo * RUMI_INV_PI_F * m.kd;
                            const float cost = fmaxf(dot3(wi, nrm), 0.0f);
                            float3 direct = f * ls.Li * cost * G / ls.pdf;
                            if (m.type == MAT_GLOSSY) direct = direct * (1.0f / m.kd_pdf);
                            float tr = 1.0f;
                            if (!LEAN && V.present) {
                                const Uniform4 U2 = path_uniforms(path, bounce, 2, k0, k1);
                                float smax_sh = 0.0f;
                                tr = volume_shadow_tr(V, p, wi, dist, U2.u[2], &smax_sh);
                                if (ADJ) sh_score = make_float2(-smax_sh * 0.33333333333f, 0.0f);
                            }
                            // a shadow ray whose contribution is exactly zero (the light
                            // below the surface's horizon: cos = 0) cannot change the film
                            // and is not traced; NaN and inf contributions are
                            const float3 c = beta * direct;
                            if (tr > 0.0f && (c.x != 0.0f || c.y != 0.0f || c.z != 0.0f)) {
                                want_sh = true;
                                sh_o = p;
                                sh_d = wi;
                                sh_tmax = dist;
                                sh_c = c;
                            }
                        }
                    }
                    const float3 fr = walk_scatter ? mk3(1, 1, 1)
                                                   : material_fr(m, albedo, nrm, b.w, wo, inobj, b.xi, b.pdf_path,
                                                                 t, vol_ratio);
                    const float pdf = avg3(mk3(b.pdfw * b.pdf_path, b.pdfw * b.pdf_path, b.pdfw * b.pdf_path));
                    beta = beta * volw * fr * b.cost * (1.0f / pdf);
                    nx_o = p;
                    nx_d = b.w;
                    nx_flags = (b.le ? PFL_LE : 0) | (b.go_in ? PFL_IN : 0);
                    want_next = !last;
                }
            }
        }
        if (addL.x != 0.0f || addL.y != 0.0f || addL.z != 0.0f) {
            float4 l = P.L[slot];
            l.x += addL.x; l.y += addL.y; l.z += addL.z;
            P.L[slot] = l;
        }
    }
    // The next rays of this block go to the queue grouped by direction (octant x dominant
    // axis: 24 bins), in one contiguous range per block.  The traversal kernels take rays
    // in queue order, so a warp then holds rays from a few neighbouring pixels' hit points
    // that head the same way (closest-hit 2% faster per frame on the 1M-triangle
    // workload).  A path's result does not depend on its queue position.
#ifdef RUMI_HOST_BUILD
    // host build (one emulated thread per block): the block's group is its one ray
    const int kn = want_next ? atomicAdd(&P.cnt[nxt], 1) : -1;
#else
    __shared__ int s_bins[32];
    if (threadIdx.x < 32) s_bins[threadIdx.x] = 0;
    __syncthreads();
    int dkey = 0, drank = 0;
    if (want_next) {
        const float ax = fabsf(nx_d.x), ay = fabsf(nx_d.y), az = fabsf(nx_d.z);
        const int dom = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
        const int oct = (nx_d.x < 0.0f ? 1 : 0) | (nx_d.y < 0.0f ? 2 : 0) | (nx_d.z < 0.0f ? 4 : 0);
        dkey = oct * 3 + dom;
        drank = atomicAdd(&s_bins[dkey], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // exclusive scan of the bins, then the block's range of the queue
        const int v = s_bins[threadIdx.x];
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if ((int)threadIdx.x >= o) incl += u;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        int base = 0;
        if (threadIdx.x == 0 && total > 0) base = atomicAdd(&P.cnt[nxt], total);
        base = __shfl_sync(0xffffffffu, base, 0);
        s_bins[threadIdx.x] = base + incl - v;
    }
    __syncthreads();
    const int kn = want_next ? s_bins[dkey] + drank : -1;
#endif
    const int ks = warp_push(&P.cnt[C_SHADOW], want_sh);
    if (want_next) {
        P.ray_o[nxt][kn] = make_float4(nx_o.x, nx_o.y, nx_o.z, pack_slot(slot, nx_flags));
        P.ray_d[nxt][kn] = make_float4(nx_d.x, nx_d.y, nx_d.z, FLT_MAX);
        P.beta_q[nxt][kn] = make_float4(beta.x, beta.y, beta.z, pend_g);
    }
    if (want_sh) {
        P.sh_o[ks] = make_float4(sh_o.x, sh_o.y, sh_o.z, __int_as_float(slot));
        P.sh_d[ks] = make_float4(sh_d.x, sh_d.y, sh_d.z, sh_tmax);
        P.sh_c[ks] = make_float4(sh_c.x, sh_c.y, sh_c.z, 0.0f);
        if (ADJ) P.sh_s[ks] = sh_score;
    }
    if (ADJ) {
        warp_add3_by_key(P.g_albedo, alb_key, alb_grad);
        // medium: warp sums, then one atomic per parameter per block
        __shared__ float red[SHADE_THREADS / 32][GM_NUM];
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
        for (int k = 0; k < GM_NUM; ++k) {
            const float v = warp_sum(gm[k]);
            if (lane == 0) red[warp][k] = v;
        }
        __syncthreads();
        if (threadIdx.x < GM_NUM) {
            float v = 0.0f;
            for (int w = 0; w < SHADE_THREADS / 32; ++w) v += red[w][threadIdx.x];
            if (v != 0.0f) atomicAdd(&P.g_medium[threadIdx.x], v);
        }
    }
}

// RayTracer::Trace (src/Integrator/raytracer.cpp:37-72), the Whitted integrator, on the
// same queues as the path tracer.  A vertex at trace depth `bounce` (the camera ray is
// depth 0; depths up to max_depth are shaded, so the host runs max_depth + 1 bounces):
//   Specular   -> Specular::GlobalIllumination: mirror ray, weight kr * colour
//                 (specular.cpp:60-75);
//   Dielectric -> Dielectric::GlobalIllumination: reflection with probability kr, else
//                 refraction with weight 1 / eta^2, eta = in_object ? eta_in / eta_out
//                 : eta_out / eta_in; a ray that goes into the object is attenuated by
//                 Beer-Lambert over the length it travels, with the absorption of the
//                 material it entered (dielectric.cpp:105-159);
//   otherwise  -> the material's DirectLighting and the walk ends: Matte next-event
//                 estimation (matte.cpp:54-82), Glossy only when its Intersection::_rand
//                 (1.0 here, nothing samples a lobe) falls on the diffuse lobe
//                 (glossy.cpp:92-102), Emissive emission when le, outside objects and
//                 front-facing (emissive.cpp:61-74), Subsurface nothing.
// No medium event: the RayTracer sends rays through a volume unattenuated; only the
// shadow ray of next-event estimation sees it (HomogeneousVolume::ShadowRayTr).  beta.w
// carries the index of the material a refracted ray entered.
__global__ void __launch_bounds__(SHADE_THREADS) pt_shade_whitted(PtLaunch P, int bounce) {
    const int cur = bounce & 1, nxt = cur ^ 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = P.cnt[cur];
    const bool active = i < n;
    bool want_next = false, want_sh = false;
    float3 nx_o = mk3(0, 0, 0), nx_d = mk3(0, 0, 0);
    unsigned nx_flags = 0;
    float3 sh_o = mk3(0, 0, 0), sh_d = mk3(0, 0, 0), sh_c = mk3(0, 0, 0);
    float sh_tmax = 0.0f;
    int slot = 0, enter_mat = 0;
    float3 beta = mk3(0, 0, 0);
    if (active) {
        const float4 o4 = P.ray_o[cur][i];
        const float4 d4 = P.ray_d[cur][i];
        const float4 hv = P.hit[i];
        slot = slot_of(o4.w);
        const DevScene &S = P.s;
        const uint64_t path = (uint64_t)(P.path0 + slot);
        const float3 o = f4xyz(o4), d = f4xyz(d4);
        const float t = hv.x;
        const int code = __float_as_int(hv.y);
        const unsigned fl = flags_of(o4.w);
        const bool le = (fl & PFL_LE) != 0, inobj = (fl & PFL_IN) != 0;
        const float4 beta4 = P.beta_q[cur][i];
        beta = f4xyz(beta4);
        const bool last = bounce + 1 >= P.max_depth;
        float3 addL = mk3(0, 0, 0);
        if (t > 0.0f) {
            const int id = code & 0x7fffffff;
            const DevMaterial m = S.materials[prim_material(S, id)];
            const float3 p = rn_madd(o, d, t);
            const float3 nrm = surface_normal(S, id, code < 0, hv.z, hv.w, o, p, m);
            if (inobj) {  // BeerLambertLaw over the segment the previous vertex sent inside
                const float3 a = S.materials[__float_as_int(beta4.w)].rgb;
                beta = beta * mk3(expf(-a.x * t), expf(-a.y * t), expf(-a.z * t));
            }
            // Texture::Pattern scales what this vertex returns (raytracer.cpp:69-70)
            if (S.prim_tex) beta = beta * tex_pattern(S, id, p);
            const float3 wo = -d;
            const Uniform4 U0 = path_uniforms(path, bounce, 0, P.k0, P.k1);
            if (m.type == MAT_SPECULAR) {
                nx_d = mirror_dir(wo, nrm);
                float3 albedo = m.rgb;
                if (id < S.n_tris && S.tri_albedo) albedo = f4xyz(__ldg(&S.tri_albedo[id]));
                beta = beta * (albedo * m.kd);
                nx_o = p;
                nx_flags = PFL_LE;
                want_next = !last;
            } else if (m.type == MAT_DIELECTRIC) {
                const float kr = fresnel_kr(d, nrm, m.eta_in, m.eta_out);
                const float kt = 1.0f - kr;
                float c;
                bool entering;
                if (kr != 0.0f && U0.u[0] <= kr) {
                    nx_d = fresnel_reflect_dir(wo, nrm, c);
                    entering = c < 0.0f;
                    beta = beta * (kr * (1.0f / kr));
                } else {
                    nx_d = refract_dir(wo, nrm, m.eta_in, m.eta_out, c);
                    entering = c > 0.0f;
                    const float eta = inobj ? m.eta_in / m.eta_out : m.eta_out / m.eta_in;
                    beta = beta * (1.0f / (eta * eta) * kt * (1.0f / kt));
                }
                nx_o = p;
                nx_flags = PFL_LE | (entering ? PFL_IN : 0);
                enter_mat = prim_material(S, id);
                want_next = !last;
            } else if (m.type == MAT_EMISSIVE) {
                if (le && !inobj && -dot3(d, nrm) > 0.0f) addL = beta * m.le;
            } else if (S.n_lights > 0 && (m.type == MAT_MATTE || (m.type == MAT_GLOSSY && m.kd != 0.0f &&
                                                                  1.0f <= m.kd_pdf))) {
                const Uniform4 U1 = path_uniforms(path, bounce, 1, P.k0, P.k1);
                const LightSample ls = sample_light(S, U0.u[3], U1.u[0], U1.u[1], p, nrm);
                float3 wi;
                float dist, G;
                if (nee_setup(ls, p, wi, dist, G)) {
                    float3 albedo = m.rgb;
                    if (id < S.n_tris && S.tri_albedo) albedo = f4xyz(__ldg(&S.tri_albedo[id]));
                    const float3 f = albedo * RUMI_INV_PI_F * m.kd;
                    const float cost = fmaxf(dot3(wi, nrm), 0.0f);
                    float3 direct = f * ls.Li * cost * G / ls.pdf;
                    if (m.type == MAT_GLOSSY) direct = direct * (1.0f / m.kd_pdf);
                    float tr = 1.0f;
                    if (S.volume.present) {
                        const Uniform4 U2 = path_uniforms(path, bounce, 2, P.k0, P.k1);
                        float smax_sh = 0.0f;
                        tr = volume_shadow_tr(S.volume, p, wi, dist, U2.u[2], &smax_sh);
                    }
                    const float3 c = beta * direct;  // zero contributions are not traced
                    if (tr > 0.0f && (c.x != 0.0f || c.y != 0.0f || c.z != 0.0f)) {
                        want_sh = true;
                        sh_o = p;
                        sh_d = wi;
                        sh_tmax = dist;
                        sh_c = c;
                    }
                }
            }
        }
        if (addL.x != 0.0f || addL.y != 0.0f || addL.z != 0.0f) {
            float4 l = P.L[slot];
            l.x += addL.x; l.y += addL.y; l.z += addL.z;
            P.L[slot] = l;
        }
    }
    const int kn = warp_push(&P.cnt[nxt], want_next);
    const int ks = warp_push(&P.cnt[C_SHADOW], want_sh);
    if (want_next) {
        P.ray_o[nxt][kn] = make_float4(nx_o.x, nx_o.y, nx_o.z, pack_slot(slot, nx_flags));
        P.ray_d[nxt][kn] = make_float4(nx_d.x, nx_d.y, nx_d.z, FLT_MAX);
        P.beta_q[nxt][kn] = make_float4(beta.x, beta.y, beta.z, __int_as_float(enter_mat));
    }
    if (want_sh) {
        P.sh_o[ks] = make_float4(sh_o.x, sh_o.y, sh_o.z, __int_as_float(slot));
        P.sh_d[ks] = make_float4(sh_d.x, sh_d.y, sh_d.z, sh_tmax);
        P.sh_c[ks] = make_float4(sh_c.x, sh_c.y, sh_c.z, 0.0f);
    }
}

// One warp per pixel: the pixel's samples are summed in sample order by lane 0 after
// a coalesced load of up to 32 samples at a time.
__global__ void pt_resolve(PtLaunch P) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= P.n_pix) return;
    float3 acc = mk3(0.0f, 0.0f, 0.0f);
    int nan = 0;
    const long long gp = (long long)P.pix0 + warp;
    int spp = P.spp;
    size_t base = (size_t)warp * P.spp;
    if (P.scenes) {
        const int k = find_scene(P.scene_pix0, P.n_scenes, gp);
        spp = P.scene_spp[k];
        base = (size_t)(P.scene_path0[k] + (gp - P.scene_pix0[k]) * spp - P.path0);
    }
    for (int s0 = 0; s0 < spp; s0 += 32) {
        const int s = s0 + lane;
        float4 l = make_float4(0, 0, 0, 0);
        if (s < spp) l = P.L[base + s];
        const int cnt = min(32, spp - s0);
        for (int k = 0; k < cnt; ++k) {
            const float x = __shfl_sync(0xffffffffu, l.x, k);
            const float y = __shfl_sync(0xffffffffu, l.y, k);
            const float z = __shfl_sync(0xffffffffu, l.z, k);
            if (x != x || y != y || z != z)
                ++nan;
            else {
                acc.x += x; acc.y += y; acc.z += z;
            }
        }
    }
    if (lane == 0) {
        const size_t px = (size_t)gp * 3;
        P.film[px + 0] = acc.z;  // B
        P.film[px + 1] = acc.y;  // G
        P.film[px + 2] = acc.x;  // R
        if (nan) atomicAdd(&P.stats[S_NAN], (unsigned long long)nan);
    }
}

static inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }
static inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Traversal scheme index (traverse_queue MODE) from rumi_render_params.trace_mode:
// 1..4 select modes 0..3, 0 selects the default, the speculative while-while walk (mode 3),
// which measured fastest on the BVH-bound workload (238 vs 302 ms per 1024x1024x64 frame
// for mode 0).
static constexpr int DEFAULT_WALK_MODE = RUMI_WALK8 ? 4 : 3;
static inline int trace_scheme(int trace_mode) {
    return trace_mode >= 1 && trace_mode <= 5 ? trace_mode - 1 : DEFAULT_WALK_MODE;
}
bool uses_bvh8(int trace_mode) { return trace_scheme(trace_mode) == 4; }

using ExtendKernel = void (*)(PtLaunch, int);
using ShadowKernel = void (*)(PtLaunch);

// Shared-memory stack depth from rumi_render_params.stack_depth: 8, 16 or 32 entries per
// thread (0 = 16).  Only the while-while walks (schemes 3 and 4) come in all three depths.
// Measured on the 1024x1024x64 BVH-bound frame (binary walk, closest-hit ms): 8: 100.5,
// 16: 100.3, 32 with the L1 carveout sized to it: 107.0 -- the 32-entry stack takes L1 that
// node fetches use, and deeper entries are rare.
static inline int stack_entries(int stack_depth) { return stack_depth == 8 || stack_depth == 32 ? stack_depth : 16; }

// Kernel selection and launches.  A host build of this file (RUMI_HOST_BUILD: the kernels
// compiled as plain C++ for the CPU tests) leaves them out; it keeps the wave layout below.
#ifndef RUMI_HOST_BUILD
template <bool STATS>
static ExtendKernel extend_kernel(int mode, int smem) {
    switch (mode) {
        case 0: return pt_extend<0, STATS>;
        case 1: return pt_extend<1, STATS>;
        case 2: return pt_extend<2, STATS>;
        case 3: return smem == 8 ? pt_extend<3, STATS, 8> : smem == 16 ? pt_extend<3, STATS, 16> : pt_extend<3, STATS>;
        default: return smem == 8 ? pt_extend<4, STATS, 8> : smem == 16 ? pt_extend<4, STATS, 16> : pt_extend<4, STATS>;
    }
}

template <bool ADJ>
static ShadowKernel shadow_kernel(int mode, int smem) {
    switch (mode) {
        case 0: return pt_shadow<0, ADJ>;
        case 1: return pt_shadow<1, ADJ>;
        case 2: return pt_shadow<2, ADJ>;
        case 3: return smem == 8 ? pt_shadow<3, ADJ, 8> : smem == 16 ? pt_shadow<3, ADJ, 16> : pt_shadow<3, ADJ>;
        default: return smem == 8 ? pt_shadow<4, ADJ, 8> : smem == 16 ? pt_shadow<4, ADJ, 16> : pt_shadow<4, ADJ>;
    }
}

// Forward shading of one bounce.  lean: the instantiation without the medium, texture,
// image-based-light and subsurface branches, for scenes that have none of them.  Every
// forward pass of a scene (render, forward with or without kept radiance, the first pass of
// backward, a batch of such scenes) takes the same instantiation, so their paths agree bit
// for bit; the two instantiations differ in the compiler's FMA contraction, not in the
// algorithm.
static void launch_shade(bool lean, cudaStream_t st, const PtLaunch &L, int b) {
    if (lean)
        pt_shade<false, true><<<cdiv(L.n_paths, SHADE_THREADS), SHADE_THREADS, 0, st>>>(L, b);
    else
        pt_shade<false><<<cdiv(L.n_paths, SHADE_THREADS), SHADE_THREADS, 0, st>>>(L, b);
}

template <bool STATS>
static void launch_extend(int mode, int smem, int grid, cudaStream_t st, const PtLaunch &L, int b) {
    extend_kernel<STATS>(mode, smem)<<<grid, TRACE_THREADS, 0, st>>>(L, b);
}

template <bool ADJ>
static void launch_shadow(int mode, int smem, int grid, cudaStream_t st, const PtLaunch &L) {
    shadow_kernel<ADJ>(mode, smem)<<<grid, TRACE_THREADS, 0, st>>>(L);
}

// Asks for just the shared memory the resident blocks' stacks need (`blocks` blocks of smem
// entries per thread), so the rest of the unified L1 / shared storage stays L1.
template <typename K>
static void prefer_l1(K k, int smem, int blocks) {
    const int need = blocks * smem * TRACE_THREADS * (int)sizeof(int);
    int pct = (need * 100 + 228 * 1024 - 1) / (228 * 1024);
    if (pct > 100) pct = 100;
    cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
}

// Persistent grids: blocks per SM at the kernels' occupancy (capped by blocks_per_sm > 0).
static void trace_grids(int mode, int smem, int num_sms, int blocks_per_sm, bool adj, int &grid, int &grid_sh) {
    int occ = 0, occ_sh = 0;
    const ExtendKernel ke = extend_kernel<false>(mode, smem);
    const ShadowKernel ks = adj ? shadow_kernel<true>(mode, smem) : shadow_kernel<false>(mode, smem);
    prefer_l1(ke, smem, trace_min_blocks(mode, true));
    prefer_l1(extend_kernel<true>(mode, smem), smem, trace_min_blocks(mode, true));
    prefer_l1(ks, smem, trace_min_blocks(mode, false));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ke, TRACE_THREADS, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sh, ks, TRACE_THREADS, 0);
    if (occ < 1) occ = 1;
    if (occ_sh < 1) occ_sh = 1;
    if (blocks_per_sm > 0) {
        occ = blocks_per_sm < occ ? blocks_per_sm : occ;
        occ_sh = blocks_per_sm < occ_sh ? blocks_per_sm : occ_sh;
    }
    grid = num_sms * occ;
    grid_sh = num_sms * occ_sh;
}

#endif  // RUMI_HOST_BUILD

// Carves the wave state for Wp paths out of ws (pt_workspace_bytes(Wp) bytes) and clears
// every optional field; returns the first byte after it.
static char *carve_wave(PtLaunch &L, void *ws, size_t Wp) {
    memset(&L, 0, sizeof(L));
    const size_t f4 = align256(Wp * sizeof(float4));
    char *w = (char *)ws;
    L.ray_o[0] = (float4 *)w; w += f4;
    L.ray_o[1] = (float4 *)w; w += f4;
    L.ray_d[0] = (float4 *)w; w += f4;
    L.ray_d[1] = (float4 *)w; w += f4;
    L.hit = (float4 *)w; w += f4;
    L.sh_o = (float4 *)w; w += f4;
    L.sh_d = (float4 *)w; w += f4;
    L.sh_c = (float4 *)w; w += f4;
    L.beta_q[0] = (float4 *)w; w += f4;
    L.beta_q[1] = (float4 *)w; w += f4;
    L.L = (float4 *)w; w += f4;
    L.cnt = (int *)w; w += align256(C_NUM * sizeof(int));
    L.stats = (unsigned long long *)w; w += align256(S_NUM * sizeof(unsigned long long));
    return w;
}

// Device bytes of the wave state for `paths` paths in flight (queues, path state,
// counters): 176 bytes per path plus alignment and counters.
size_t pt_workspace_bytes(long long paths) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t Wp = (size_t)paths;
    return 11 * al(Wp * sizeof(float4)) + al(C_NUM * sizeof(int)) + al(S_NUM * sizeof(unsigned long long));
}

#ifndef RUMI_HOST_BUILD
// The scene's second stream and its fork / join events, made on first use.
static rumi_status ensure_aux(rumi_scene *sc) {
    if (sc->aux_stream) return RUMI_OK;
    cudaError_t e = cudaStreamCreateWithFlags(&sc->aux_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sc->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sc->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_status(e, "auxiliary stream");
    return RUMI_OK;
}

rumi_status pt_render(rumi_scene *sc, const rumi_render_params *p, float *film_dev, rumi_render_stats *stats,
                      cudaStream_t stream, float4 *keep_L) {
    const long long total_pix = (long long)sc->dev.width * sc->dev.height;
    long long wave = p->wave_paths > 0 ? p->wave_paths : RUMI_DEFAULT_WAVE_PATHS;
    long long pix_per_wave = wave / p->spp;
    if (pix_per_wave < 1) pix_per_wave = 1;
    if (pix_per_wave > total_pix) pix_per_wave = total_pix;
    const long long n_paths_max = pix_per_wave * p->spp;
    if (n_paths_max > 0x3fffffffLL) {  // slots are 30-bit (pack_slot)
        set_error("wave_paths too large");
        return RUMI_ERR_INVALID_ARG;
    }
    rumi_status st = ensure_workspace(sc, pt_workspace_bytes(n_paths_max));
    if (st != RUMI_OK) return st;
    if (uses_bvh8(p->trace_mode) && (st = ensure_bvh8(sc)) != RUMI_OK) return st;
    if ((st = ensure_aux(sc)) != RUMI_OK) return st;
    return pt_render_in(sc, p, film_dev, stats, stream, sc->ws, pix_per_wave,
                        RUMI_PT_OVERLAP != 0 && !(p->flags & RUMI_FLAG_SERIAL), keep_L);
}

// The frame loop over waves of pix_per_wave pixels, with the wave state carved out of
// `ws` (pt_workspace_bytes(pix_per_wave * spp) bytes).
rumi_status pt_render_in(rumi_scene *sc, const rumi_render_params *p, float *film_dev, rumi_render_stats *stats,
                         cudaStream_t stream, void *ws, long long pix_per_wave, bool overlap, float4 *keep_L) {
    const int W = sc->dev.width, H = sc->dev.height;
    const int spp = p->spp;
    const long long total_pix = (long long)W * H;
    const size_t Wp = (size_t)(pix_per_wave * spp);
    PtLaunch L;
    carve_wave(L, ws, Wp);
    L.s = sc->dev;
    L.spp = spp;
    // RayTracer::Trace shades trace depths 0..max_depth (raytracer.cpp:41-42)
    const bool whitted = p->integrator == RUMI_RAY_TRACER;
    const int bounces = whitted ? p->max_depth + 1 : p->max_depth;
    L.max_depth = bounces;
    L.k0 = (uint32_t)p->seed;
    L.k1 = (uint32_t)(p->seed >> 32) ^ 0x5851F42Du;
    int d = 0;
    while ((d + 1) * (d + 1) <= spp) ++d;
    L.grid_d = d;
    L.square = d * d == spp;
    L.film = film_dev;
    cudaMemsetAsync(L.cnt, 0, C_NUM * sizeof(int), stream);
    cudaMemsetAsync(L.stats, 0, S_NUM * sizeof(unsigned long long), stream);

    // traversal scheme and persistent grid (autotuner knobs; 0 = defaults)
    const int mode = trace_scheme(p->trace_mode);
    const int smem = stack_entries(p->stack_depth);
    L.refill_min = p->refill_min > 0 ? p->refill_min : 8;
    int trace_grid = 0, shadow_grid = 0;
    trace_grids(mode, smem, sc->num_sms, p->blocks_per_sm, false, trace_grid, shadow_grid);

    const bool timing = (p->flags & RUMI_FLAG_TIMING) != 0;
    const bool count_stats = (p->flags & RUMI_FLAG_STATS) != 0;
    const bool lean = shade_lean(sc);
    std::vector<cudaEvent_t> evs;
    auto mark_on = [&](cudaStream_t st_) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st_);
        evs.push_back(e);
    };
    auto mark = [&]() { mark_on(stream); };
    // event indices of (begin, end) per launch kind
    std::vector<std::pair<int, int>> ext_ev, shade_ev, sh_ev;
    if (timing) mark();
    long long waves = 0;
    for (long long pix0 = 0; pix0 < total_pix; pix0 += pix_per_wave) {
        const long long n_pix = pix0 + pix_per_wave <= total_pix ? pix_per_wave : total_pix - pix0;
        L.pix0 = (int)pix0;
        L.n_pix = (int)n_pix;
        L.n_paths = (int)(n_pix * spp);
        L.path0 = pix0 * spp;
        pt_generate<<<cdiv(L.n_paths, 256), 256, 0, stream>>>(L);
        if (overlap) {
            // shadow rays of bounce b are traced on the auxiliary stream while bounce b + 1's
            // closest-hit rays are traced here: neither reads what the other writes (shadow
            // queue and per-path radiance vs ray queue and hits); shading of b + 1 waits
            // for both, as it refills the shadow queue and adds to the radiance
            // (with timing, a closest-hit launch's events include the time it shares the
            // GPU with the previous bounce's any-hit launch)
            for (int b = 0; b < bounces; ++b) {
                pt_reset_extend<<<1, 1, 0, stream>>>(L, b);
                int e0 = 0;
                if (timing) { e0 = (int)evs.size(); mark(); }
                if (count_stats)
                    launch_extend<true>(mode, smem, trace_grid, stream, L, b);
                else
                    launch_extend<false>(mode, smem, trace_grid, stream, L, b);
                if (timing) { mark(); ext_ev.push_back({e0, e0 + 1}); }
                if (b > 0) cudaStreamWaitEvent(stream, sc->ev_join, 0);
                pt_reset_shade<<<1, 1, 0, stream>>>(L, b);
                if (timing) { e0 = (int)evs.size(); mark(); }
                if (whitted)
                    pt_shade_whitted<<<cdiv(L.n_paths, SHADE_THREADS), SHADE_THREADS, 0, stream>>>(L, b);
                else
                    launch_shade(lean, stream, L, b);
                if (timing) { mark(); shade_ev.push_back({e0, e0 + 1}); }
                const bool aside = b + 1 < bounces;
                cudaStream_t ss = aside ? sc->aux_stream : stream;
                if (aside) {
                    cudaEventRecord(sc->ev_fork, stream);
                    cudaStreamWaitEvent(sc->aux_stream, sc->ev_fork, 0);
                }
                if (timing) { e0 = (int)evs.size(); mark_on(ss); }
                launch_shadow<false>(mode, smem, shadow_grid, ss, L);
                if (timing) { mark_on(ss); sh_ev.push_back({e0, e0 + 1}); }
                if (aside) cudaEventRecord(sc->ev_join, sc->aux_stream);
            }
            pt_finish<<<1, 1, 0, stream>>>(L);
            pt_resolve<<<cdiv(L.n_pix * 32LL, 256), 256, 0, stream>>>(L);
            if (keep_L)
                cudaMemcpyAsync(keep_L + L.path0, L.L, sizeof(float4) * (size_t)L.n_paths, cudaMemcpyDeviceToDevice,
                                stream);
            ++waves;
            continue;
        }
        for (int b = 0; b < bounces; ++b) {
            pt_reset<<<1, 1, 0, stream>>>(L, b);
            int e0 = 0;
            if (timing) { e0 = (int)evs.size(); mark(); }
            if (count_stats)
                launch_extend<true>(mode, smem, trace_grid, stream, L, b);
            else
                launch_extend<false>(mode, smem, trace_grid, stream, L, b);
            if (timing) { mark(); ext_ev.push_back({e0, e0 + 1}); }
            if (timing) { e0 = (int)evs.size(); mark(); }
            if (whitted)
                pt_shade_whitted<<<cdiv(L.n_paths, SHADE_THREADS), SHADE_THREADS, 0, stream>>>(L, b);
            else
                launch_shade(lean, stream, L, b);
            if (timing) { mark(); shade_ev.push_back({e0, e0 + 1}); }
            if (timing) { e0 = (int)evs.size(); mark(); }
            launch_shadow<false>(mode, smem, shadow_grid, stream, L);
            if (timing) { mark(); sh_ev.push_back({e0, e0 + 1}); }
        }
        pt_finish<<<1, 1, 0, stream>>>(L);
        pt_resolve<<<cdiv(L.n_pix * 32LL, 256), 256, 0, stream>>>(L);
        if (keep_L)
            cudaMemcpyAsync(keep_L + L.path0, L.L, sizeof(float4) * (size_t)L.n_paths, cudaMemcpyDeviceToDevice,
                            stream);
        ++waves;
    }
    if (timing) mark();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "pt_render launch");
    unsigned long long h_stats[S_NUM];
    cudaMemcpyAsync(h_stats, L.stats, sizeof(h_stats), cudaMemcpyDeviceToHost, stream);
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        for (auto ev : evs) cudaEventDestroy(ev);
        return cuda_status(e, "pt_render");
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->paths = total_pix * spp;
        stats->nan_samples = (int64_t)h_stats[S_NAN];
        stats->rays_extend = (int64_t)h_stats[S_RAYS_EXT];
        stats->rays_shadow = (int64_t)h_stats[S_RAYS_SH];
        stats->extend_node_fetches = (int64_t)(h_stats[S_NODES] / 2);  // 16-byte units -> 32-byte nodes
        stats->extend_prim_tests = (int64_t)h_stats[S_PRIMS];
        stats->extend_launches = (int64_t)waves * bounces;
        stats->shade_launches = stats->extend_launches;
        stats->shadow_launches = stats->extend_launches;
        if (timing) {
            float ms;
            for (auto &pr : ext_ev) { cudaEventElapsedTime(&ms, evs[pr.first], evs[pr.second]); stats->extend_ms += ms; }
            for (auto &pr : shade_ev) { cudaEventElapsedTime(&ms, evs[pr.first], evs[pr.second]); stats->shade_ms += ms; }
            for (auto &pr : sh_ev) { cudaEventElapsedTime(&ms, evs[pr.first], evs[pr.second]); stats->shadow_ms += ms; }
            cudaEventElapsedTime(&ms, evs.front(), evs.back());
            stats->total_ms = ms;
        }
    }
    for (auto ev : evs) cudaEventDestroy(ev);
    return RUMI_OK;
}

// ---------------------------------------------------------------- path-replay adjoint
// Device bytes of the adjoint's wave state: the rendering wave state plus, per path, the
// first pass's radiance, the loss weights and the shadow-ray scores.
size_t pt_adjoint_workspace_bytes(long long paths) {
    const size_t Wp = (size_t)paths;
    return pt_workspace_bytes(paths) + 2 * align256(Wp * sizeof(float4)) + align256(Wp * sizeof(float2));
}

// Gradients of <dfilm, film> for the frame rumi_render produces with the same parameters:
// g_albedo (n_tris * 3, RGB; may be null) and g_medium (GM_NUM; may be null) are
// overwritten.  Each wave is traced twice: pass 1 records every path's radiance, pass 2
// replays the same random numbers with the scores of pt_shade<true> / pt_shadow<0, true>.
rumi_status pt_backward(rumi_scene *sc, const rumi_render_params *p, const float *dfilm_dev, float *g_albedo,
                        float *g_medium, rumi_render_stats *stats, cudaStream_t stream) {
    const int W = sc->dev.width, H = sc->dev.height;
    const int spp = p->spp;
    const long long total_pix = (long long)W * H;
    long long wave = p->wave_paths > 0 ? p->wave_paths : RUMI_DEFAULT_WAVE_PATHS;
    long long pix_per_wave = wave / spp;
    if (pix_per_wave < 1) pix_per_wave = 1;
    if (pix_per_wave > total_pix) pix_per_wave = total_pix;
    const size_t Wp = (size_t)(pix_per_wave * spp);
    if (Wp > 0x3fffffffULL) {
        set_error("wave_paths too large");
        return RUMI_ERR_INVALID_ARG;
    }
    rumi_status st = ensure_workspace(sc, pt_adjoint_workspace_bytes((long long)Wp));
    if (st != RUMI_OK) return st;
    if (uses_bvh8(p->trace_mode) && (st = ensure_bvh8(sc)) != RUMI_OK) return st;
    const bool overlap = RUMI_PT_OVERLAP != 0 && !(p->flags & RUMI_FLAG_SERIAL);
    if (overlap && (st = ensure_aux(sc)) != RUMI_OK) return st;
    // the forward pass of this very frame kept its per-path radiance: pass 1 is not traced
    const bool reuse = sc->kept_valid && sc->kept_seed == p->seed && sc->kept_spp == spp &&
                       sc->kept_depth == p->max_depth && sc->kept_cap >= total_pix * spp;
    float *gm_scratch = nullptr;
    cudaError_t e = cudaSuccess;
    if (!g_medium) {
        e = dalloc((void **)&gm_scratch, GM_NUM * sizeof(float), stream);
        if (e != cudaSuccess) return cuda_status(e, "adjoint scratch");
        g_medium = gm_scratch;
    }
    PtLaunch A;
    char *w = carve_wave(A, sc->ws, Wp);
    A.s = sc->dev;
    A.spp = spp;
    A.max_depth = p->max_depth;
    A.k0 = (uint32_t)p->seed;
    A.k1 = (uint32_t)(p->seed >> 32) ^ 0x5851F42Du;
    int d = 0;
    while ((d + 1) * (d + 1) <= spp) ++d;
    A.grid_d = d;
    A.square = d * d == spp;
    A.refill_min = 8;
    PtLaunch B = A;
    float4 *Lt = (float4 *)w; w += align256(Wp * sizeof(float4));
    B.Lt = Lt;
    B.dls = (float4 *)w; w += align256(Wp * sizeof(float4));
    B.sh_s = (float2 *)w;
    B.dfilm = dfilm_dev;
    B.g_albedo = g_albedo;
    B.g_medium = g_medium;
    cudaMemsetAsync(A.cnt, 0, C_NUM * sizeof(int), stream);
    cudaMemsetAsync(A.stats, 0, S_NUM * sizeof(unsigned long long), stream);
    cudaMemsetAsync(g_medium, 0, GM_NUM * sizeof(float), stream);
    if (g_albedo) cudaMemsetAsync(g_albedo, 0, sizeof(float) * 3 * (size_t)sc->dev.n_tris, stream);

    // the same traversal scheme as rumi_render, so both passes and the forward frame
    // resolve exact-distance ties alike
    const int mode = trace_scheme(p->trace_mode);
    const int smem = stack_entries(p->stack_depth);
    A.refill_min = B.refill_min = p->refill_min > 0 ? p->refill_min : 8;
    int grid = 0, grid_sh = 0, grid_dummy = 0, grid_sh_adj = 0;
    trace_grids(mode, smem, sc->num_sms, p->blocks_per_sm, false, grid, grid_sh);
    trace_grids(mode, smem, sc->num_sms, p->blocks_per_sm, true, grid_dummy, grid_sh_adj);

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (p->flags & RUMI_FLAG_TIMING) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, stream);
    }
    long long waves = 0;
    for (long long pix0 = 0; pix0 < total_pix; pix0 += pix_per_wave) {
        const long long n_pix = pix0 + pix_per_wave <= total_pix ? pix_per_wave : total_pix - pix0;
        for (PtLaunch *L : {&A, &B}) {
            L->pix0 = (int)pix0;
            L->n_pix = (int)n_pix;
            L->n_paths = (int)(n_pix * spp);
            L->path0 = pix0 * spp;
        }
        // both passes on the two-stream schedule of pt_render_in: each bounce's shadow rays
        // beside the next bounce's closest-hit rays, shading after both
        auto pass = [&](PtLaunch &X, bool adj) {
            pt_generate<<<cdiv(X.n_paths, 256), 256, 0, stream>>>(X);
            for (int b = 0; b < p->max_depth; ++b) {
                pt_reset_extend<<<1, 1, 0, stream>>>(X, b);
                launch_extend<false>(mode, smem, grid, stream, X, b);
                if (b > 0 && overlap) cudaStreamWaitEvent(stream, sc->ev_join, 0);
                pt_reset_shade<<<1, 1, 0, stream>>>(X, b);
                if (adj)
                    pt_shade<true><<<cdiv(X.n_paths, SHADE_THREADS), SHADE_THREADS, 0, stream>>>(X, b);
                else
                    launch_shade(shade_lean(sc), stream, X, b);
                const bool aside = overlap && b + 1 < p->max_depth;
                cudaStream_t ss = aside ? sc->aux_stream : stream;
                if (aside) {
                    cudaEventRecord(sc->ev_fork, stream);
                    cudaStreamWaitEvent(sc->aux_stream, sc->ev_fork, 0);
                }
                if (adj)
                    launch_shadow<true>(mode, smem, grid_sh_adj, ss, X);
                else
                    launch_shadow<false>(mode, smem, grid_sh, ss, X);
                if (aside) cudaEventRecord(sc->ev_join, sc->aux_stream);
            }
            pt_finish<<<1, 1, 0, stream>>>(X);
        };
        // pass 1: radiance of every path (or the radiance rumi_forward kept for this frame)
        if (reuse) {
            cudaMemcpyAsync(Lt, sc->kept_L + A.path0, sizeof(float4) * (size_t)A.n_paths, cudaMemcpyDeviceToDevice,
                            stream);
        } else {
            pass(A, false);
            cudaMemcpyAsync(Lt, A.L, sizeof(float4) * (size_t)A.n_paths, cudaMemcpyDeviceToDevice, stream);
        }
        // pass 2: replay with the scores
        pass(B, true);
        ++waves;
    }
    if (e1) cudaEventRecord(e1, stream);
    e = cudaGetLastError();
    unsigned long long h_stats[S_NUM];
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_stats, A.stats, sizeof(h_stats), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    dfree(gm_scratch, stream);
    if (e != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        return cuda_status(e, "pt_backward");
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->paths = total_pix * spp;
        stats->nan_samples = (int64_t)h_stats[S_NAN];
        stats->rays_extend = (int64_t)h_stats[S_RAYS_EXT];
        stats->rays_shadow = (int64_t)h_stats[S_RAYS_SH];
        stats->extend_launches = (reuse ? 1 : 2) * waves * p->max_depth;
        stats->shade_launches = stats->extend_launches;
        stats->shadow_launches = stats->extend_launches;
        if (e0) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            stats->total_ms = ms;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return RUMI_OK;
}

// ---------------------------------------------------------------- scene batches
// Device bytes of a multi-scene wave: the single-scene wave state plus each slot's scene.
size_t pt_batch_workspace_bytes(long long wave_paths) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return pt_workspace_bytes(wave_paths) + al((size_t)wave_paths * sizeof(int));
}

// Enqueues one frame of a multi-scene batch without synchronising, so the sequence can
// be captured into a CUDA graph: waves over the batch's global pixel / path index space,
// every stage serving all scenes from shared queues.
rumi_status pt_enqueue_batch(const BatchFrame &F, void *ws, float *films, cudaStream_t stream, int num_sms,
                             cudaStream_t aux, cudaEvent_t ev_fork, cudaEvent_t ev_join) {
    PtLaunch L;
    L.slot_scene = (int *)carve_wave(L, ws, (size_t)F.wave_paths);
    L.max_depth = F.max_depth;
    L.film = films;
    L.scenes = F.scenes;
    L.scene_path0 = F.scene_path0;
    L.scene_pix0 = F.scene_pix0;
    L.scene_key = F.scene_key;
    L.scene_spp = F.scene_spp;
    L.n_scenes = F.n_scenes;
    L.spp = 1;
    L.refill_min = 8;
    cudaMemsetAsync(L.cnt, 0, C_NUM * sizeof(int), stream);
    cudaMemsetAsync(L.stats, 0, S_NUM * sizeof(unsigned long long), stream);
    int occ = 0, occ_sh = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pt_trace_multi<false>, TRACE_THREADS, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sh, pt_trace_multi<true>, TRACE_THREADS, 0);
    if (occ < 1) occ = 1;
    if (occ_sh < 1) occ_sh = 1;
    if (F.blocks_per_sm > 0) {
        occ = F.blocks_per_sm < occ ? F.blocks_per_sm : occ;
        occ_sh = F.blocks_per_sm < occ_sh ? F.blocks_per_sm : occ_sh;
    }
    for (const BatchWave &wv : F.waves) {
        L.pix0 = (int)wv.pix0;
        L.n_pix = (int)(wv.pix1 - wv.pix0);
        L.path0 = wv.path0;
        L.n_paths = (int)(wv.path1 - wv.path0);
        pt_generate<<<cdiv(L.n_paths, 256), 256, 0, stream>>>(L);
        // the two-stream schedule of pt_render_in (a graph capture takes the auxiliary
        // stream in through the fork event and every fork is joined before shading)
        for (int b = 0; b < F.max_depth; ++b) {
            pt_reset_extend<<<1, 1, 0, stream>>>(L, b);
            pt_trace_multi<false><<<num_sms * occ, TRACE_THREADS, 0, stream>>>(L, b);
            if (b > 0 && aux) cudaStreamWaitEvent(stream, ev_join, 0);
            pt_reset_shade<<<1, 1, 0, stream>>>(L, b);
            launch_shade(F.lean, stream, L, b);
            const bool aside = aux && b + 1 < F.max_depth;
            if (aside) {
                cudaEventRecord(ev_fork, stream);
                cudaStreamWaitEvent(aux, ev_fork, 0);
            }
            pt_trace_multi<true><<<num_sms * occ_sh, TRACE_THREADS, 0, aside ? aux : stream>>>(L, b);
            if (aside) cudaEventRecord(ev_join, aux);
        }
        pt_finish<<<1, 1, 0, stream>>>(L);
        pt_resolve<<<cdiv(L.n_pix * 32LL, 256), 256, 0, stream>>>(L);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "batch launch");
    return RUMI_OK;
}

// Device address of the 64-bit statistics inside a batch workspace.
unsigned long long *pt_batch_stats_ptr(void *ws, long long wave_paths) {
    PtLaunch L;
    carve_wave(L, ws, (size_t)wave_paths);  // the same layout pt_enqueue_batch carves
    return L.stats;
}

// ---------------------------------------------------------------- ray batches
struct TraceLaunch {
    DevScene s;
    const float4 *rays;  // 2 float4 per ray: (o, in_object), (d, tmax)
    float *t;
    int32_t *prim;
    long long n;
    int anyhit;
    unsigned long long *counters;  // [0] fetch, [1] nodes, [2] prims
};

// Ray queries: the renderer's default traversal scheme (speculative while-while with
// per-lane refill) over a caller's ray array, in chunks of at most 2^30 rays.
template <int MODE, bool ANYHIT, bool STATS>
__global__ void __launch_bounds__(TRACE_THREADS, RUMI_TRACE_MIN_BLOCKS) trace_batch_kernel(TraceLaunch T, long long first,
                                                                                         int n, int *fetch_counter) {
    __shared__ int stack[STACK_SMEM * TRACE_THREADS];
    TraceStats st{0, 0};
    auto fetch = [&](int i, float3 &o, float3 &d, float &tmax, bool &in_obj) {
        const long long k = first + i;
        const float4 o4 = T.rays[2 * k], d4 = T.rays[2 * k + 1];
        o = f4xyz(o4);
        d = f4xyz(d4);
        tmax = d4.w;
        in_obj = o4.w != 0.0f;
    };
    auto finish = [&](int i, const HitRec &h) {
        const long long k = first + i;
        T.t[k] = h.t;
        T.prim[k] = ANYHIT ? (h.t > 0.0f ? 1 : 0) : (h.t > 0.0f ? h.id : -1);
    };
    traverse_queue<MODE, ANYHIT, STACK_SMEM, STATS>(T.s, n, fetch_counter, 8, stack + threadIdx.x, TRACE_THREADS,
                                                    fetch, finish, st);
    if (STATS) {
        atomicAdd(&T.counters[1], (unsigned long long)st.nodes);
        atomicAdd(&T.counters[2], (unsigned long long)st.prims);
    }
}

template <bool ANYHIT, bool STATS, int MODE = DEFAULT_WALK_MODE>
static void launch_trace_batch(const TraceLaunch &T, int num_sms, cudaStream_t stream) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, trace_batch_kernel<MODE, ANYHIT, STATS>, TRACE_THREADS, 0);
    if (occ < 1) occ = 1;
    const long long chunk = 1LL << 30;
    int k = 0;
    for (long long first = 0; first < T.n; first += chunk, ++k) {
        const int n = (int)(T.n - first < chunk ? T.n - first : chunk);
        // one fetch counter per chunk (counters[3 + k]; chunk count is bounded by the caller's n)
        int *ctr = reinterpret_cast<int *>(T.counters + 3) + k;
        trace_batch_kernel<MODE, ANYHIT, STATS><<<num_sms * occ, TRACE_THREADS, 0, stream>>>(T, first, n, ctr);
    }
}

rumi_status trace_rays(rumi_scene *sc, int64_t n, const float *rays_dev, int anyhit, float *t_dev, int32_t *prim_dev,
                       int64_t *node_visits, int64_t *prim_tests, cudaStream_t stream) {
    const long long chunks = (n + (1LL << 30) - 1) >> 30;
    if (chunks > 64) {
        set_error("trace_rays: at most 2^36 rays per call");
        return RUMI_ERR_INVALID_ARG;
    }
    rumi_status st = ensure_workspace(sc, 256 + 3 * sizeof(unsigned long long) + 64 * sizeof(int));
    if (st != RUMI_OK) return st;
    TraceLaunch T;
    T.s = sc->dev;
    T.rays = (const float4 *)rays_dev;
    T.t = t_dev;
    T.prim = prim_dev;
    T.n = n;
    T.anyhit = anyhit;
    T.counters = (unsigned long long *)sc->ws;
    cudaMemsetAsync(T.counters, 0, 3 * sizeof(unsigned long long) + 64 * sizeof(int), stream);
    const bool stats = node_visits != nullptr || prim_tests != nullptr;
    if (n > 0) {
        if (anyhit)
            stats ? launch_trace_batch<true, true>(T, sc->num_sms, stream)
                  : launch_trace_batch<true, false>(T, sc->num_sms, stream);
        else
            stats ? launch_trace_batch<false, true>(T, sc->num_sms, stream)
                  : launch_trace_batch<false, false>(T, sc->num_sms, stream);
    }
    unsigned long long h[3] = {0, 0, 0};
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, T.counters, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_status(e, "trace_rays");
    if (node_visits) *node_visits = (int64_t)(h[1] / 2);  // 16-byte units -> 32-byte nodes
    if (prim_tests) *prim_tests = (int64_t)h[2];
    return RUMI_OK;
}

// Ray queries through the traversal scheme trace_mode selects (1..5, as rumi_render_params;
// 0 = the default), so a test can compare every scheme's hits on the same rays.
rumi_status trace_rays_scheme(rumi_scene *sc, int64_t n, const float *rays_dev, int anyhit, int trace_mode,
                              float *t_dev, int32_t *prim_dev, cudaStream_t stream) {
    if (n < 0 || n > (1LL << 30)) {
        set_error("trace_rays_scheme: 0 <= n <= 2^30");
        return RUMI_ERR_INVALID_ARG;
    }
    rumi_status st = ensure_workspace(sc, 256 + 3 * sizeof(unsigned long long) + 64 * sizeof(int));
    if (st != RUMI_OK) return st;
    if (uses_bvh8(trace_mode) && (st = ensure_bvh8(sc)) != RUMI_OK) return st;
    TraceLaunch T;
    T.s = sc->dev;
    T.rays = (const float4 *)rays_dev;
    T.t = t_dev;
    T.prim = prim_dev;
    T.n = n;
    T.anyhit = anyhit;
    T.counters = (unsigned long long *)sc->ws;
    cudaMemsetAsync(T.counters, 0, 3 * sizeof(unsigned long long) + 64 * sizeof(int), stream);
    if (n > 0) {
        const int m = trace_scheme(trace_mode);
        auto go = [&](auto mode_tag) {
            constexpr int M = decltype(mode_tag)::value;
            if (anyhit)
                launch_trace_batch<true, false, M>(T, sc->num_sms, stream);
            else
                launch_trace_batch<false, false, M>(T, sc->num_sms, stream);
        };
        switch (m) {
            case 0: go(std::integral_constant<int, 0>()); break;
            case 1: go(std::integral_constant<int, 1>()); break;
            case 2: go(std::integral_constant<int, 2>()); break;
            case 3: go(std::integral_constant<int, 3>()); break;
            default: go(std::integral_constant<int, 4>()); break;
        }
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_status(e, "trace_rays_scheme");
    return RUMI_OK;
}

#endif  // RUMI_HOST_BUILD

}  // namespace rumi
