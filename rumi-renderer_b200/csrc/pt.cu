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

namespace rumi {

static constexpr int TRACE_THREADS = 128;
static constexpr int STACK_SMEM = 32;
static constexpr int SHADE_THREADS = 256;

enum { PFL_LE = 1, PFL_IN = 2 };
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
    float4 *beta, *L;
    unsigned *pflags;
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
};

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
    float3 o, d;
    if (P.scenes) {
        const long long g = P.path0 + j;
        const int k = find_scene(P.scene_path0, P.n_scenes, g);
        const DevScene &S = P.scenes[k];
        const int spp = P.scene_spp[k];
        const long long local = g - P.scene_path0[k];
        const long long pixel = local / spp;
        const int s = (int)(local % spp);
        const int gd = isqrt_floor(spp);
        const int w = (int)(pixel % S.width), h = (int)(pixel / S.width);
        const float2 smp = pixel_sample(s, spp, gd, gd * gd == spp, pixel, P.scene_key[2 * k], P.scene_key[2 * k + 1]);
        camera_ray(S.camera, S.width, S.height, w, h, smp.x, smp.y, o, d);
        P.slot_scene[j] = k;
    } else {
        const long long pixel = (long long)P.pix0 + j / P.spp;
        const int s = j % P.spp;
        const int W = P.s.width;
        const int w = (int)(pixel % W), h = (int)(pixel / W);
        const float2 smp = pixel_sample(s, P.spp, P.grid_d, P.square != 0, pixel, P.k0, P.k1);
        camera_ray(P.s.camera, W, P.s.height, w, h, smp.x, smp.y, o, d);
    }
    P.ray_o[0][j] = make_float4(o.x, o.y, o.z, __int_as_float(j));
    P.ray_d[0][j] = make_float4(d.x, d.y, d.z, FLT_MAX);
    P.beta[j] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    P.L[j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    P.pflags[j] = PFL_LE;
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

// Persistent traversal kernels: every block takes rays from the bounce's queue until it
// is empty (traverse_queue in traverse.cuh; MODE selects the scheme, see there).
template <int MODE, bool STATS>
__global__ void __launch_bounds__(TRACE_THREADS) pt_extend(PtLaunch P, int bounce) {
    __shared__ int stack[STACK_SMEM * TRACE_THREADS];
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
    traverse_queue<MODE, false, STACK_SMEM, STATS>(P.s, P.cnt[cur], &P.cnt[C_FETCH_EXT], P.refill_min,
                                                   stack + threadIdx.x, TRACE_THREADS, fetch, finish, st);
    if (STATS) {
        atomicAdd(&P.stats[S_NODES], (unsigned long long)st.nodes);
        atomicAdd(&P.stats[S_PRIMS], (unsigned long long)st.prims);
    }
}

template <int MODE>
__global__ void __launch_bounds__(TRACE_THREADS) pt_shadow(PtLaunch P) {
    __shared__ int stack[STACK_SMEM * TRACE_THREADS];
    TraceStats st{0, 0};
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
        }
    };
    traverse_queue<MODE, true, STACK_SMEM, false>(P.s, P.cnt[C_SHADOW], &P.cnt[C_FETCH_SH], P.refill_min,
                                                  stack + threadIdx.x, TRACE_THREADS, fetch, finish, st);
}

// Multi-scene batches: the warp-batch traversal with each ray's own scene.
template <bool ANYHIT>
__global__ void __launch_bounds__(TRACE_THREADS) pt_trace_multi(PtLaunch P, int bounce) {
    __shared__ int stack[STACK_SMEM * TRACE_THREADS];
    const int cur = bounce & 1;
    const int n = ANYHIT ? P.cnt[C_SHADOW] : P.cnt[cur];
    int *counter = ANYHIT ? &P.cnt[C_FETCH_SH] : &P.cnt[C_FETCH_EXT];
    const int lane = threadIdx.x & 31;
    TraceStats st{0, 0};
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(counter, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const int i = base + lane;
        if (i < n) {
            const float4 o4 = ANYHIT ? P.sh_o[i] : P.ray_o[cur][i];
            const float4 d4 = ANYHIT ? P.sh_d[i] : P.ray_d[cur][i];
            const int slot = __float_as_int(o4.w) & 0x7fffffff;
            const DevScene &S = P.scenes[P.slot_scene[slot]];
            const bool in_obj = !ANYHIT && (__float_as_uint(o4.w) >> 31) != 0;
            const HitRec h = trace_ray<ANYHIT, STACK_SMEM, false>(S, f4xyz(o4), f4xyz(d4), d4.w, in_obj,
                                                                 stack + threadIdx.x, TRACE_THREADS, st);
            if (ANYHIT) {
                if (h.t == 0.0f) {
                    const float4 c = P.sh_c[i];
                    float4 l = P.L[slot];
                    l.x += c.x; l.y += c.y; l.z += c.z;
                    P.L[slot] = l;
                }
            } else {
                const int code = h.t > 0.0f ? (h.id | (h.back ? (int)0x80000000 : 0)) : -1;
                P.hit[i] = make_float4(h.t, __int_as_float(code), h.u, h.v);
            }
        }
    }
}

// Next-event estimation toward one light sample from p.  Returns false when the light
// faces away or lies outside a spot cone (Scene::VisibilityTest's facing test,
// src/Scene/scene.cpp:99-123).  wi / dist: the shadow ray; G: AreaLight::G.
RUMI_D bool nee_setup(const LightSample &ls, float3 p, float3 &wi, float &dist, float &G) {
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

__global__ void __launch_bounds__(SHADE_THREADS) pt_shade(PtLaunch P, int bounce) {
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

    if (active) {
        const float4 o4 = P.ray_o[cur][i];
        const float4 d4 = P.ray_d[cur][i];
        const float4 hv = P.hit[i];
        slot = __float_as_int(o4.w) & 0x7fffffff;
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
        const unsigned fl = P.pflags[slot];
        const bool le = (fl & PFL_LE) != 0, inobj = (fl & PFL_IN) != 0;
        beta = f4xyz(P.beta[slot]);
        const Uniform4 U0 = path_uniforms(path, bounce, 0, k0, k1);
        const Uniform4 U1 = path_uniforms(path, bounce, 1, k0, k1);
        const bool last = bounce + 1 >= P.max_depth;
        float3 addL = mk3(0, 0, 0);
        bool done = false;

        // ---------------------------------------------- homogeneous medium
        const DevVolume &V = S.volume;
        if (V.present && !inobj) {
            float tn, tf;
            const float thit = hit ? t : 0.0f;
            if (volume_intersect(V, o, d, thit, tn, tf)) {
                const float smax = volume_max_distance(thit, tn, tf);
                const DistSample ds = distance_sample(V.sigma_t, V.avg_sigma_t, V.absorb, smax, U1.u[2], U1.u[3]);
                if (ds.outcome == 2) {
                    done = true;  // absorbed (pathtracer.cpp:164-167)
                } else if (ds.outcome == 1) {
                    const float3 p = o + d * (tn < 0.0f ? ds.s : tn + ds.s);
                    const float3 vol = ds.tau / ds.pdf;
                    // HomogeneousVolume::DirectLighting (homogeneousvolume.cpp:231-250)
                    if (S.n_lights > 0) {
                        const LightSample ls = sample_light(S, U0.u[3], U1.u[0], U1.u[1]);
                        float3 wi;
                        float dist, G;
                        if (nee_setup(ls, p, wi, dist, G)) {
                            const Uniform4 U2 = path_uniforms(path, bounce, 2, k0, k1);
                            const float tr = volume_shadow_tr(V, p, wi, dist, U2.u[2]);
                            if (tr > 0.0f) {
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
            float3 p = o + d * t;
            float3 nrm;
            float3 albedo = m.rgb;
            if (id < S.n_tris) {
                const float4 n0 = __ldg(&S.tri_shade[3 * id]), n1 = __ldg(&S.tri_shade[3 * id + 1]),
                             n2 = __ldg(&S.tri_shade[3 * id + 2]);
                const float u = hv.z, v = hv.w;
                nrm = f4xyz(n0) * (1.0f - u - v) + f4xyz(n1) * u + f4xyz(n2) * v;  // triangle.cpp:111 (Q3)
                if (back && material_opaque(m)) nrm = -nrm;
                if (S.tri_albedo) albedo = f4xyz(__ldg(&S.tri_albedo[id]));
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
                // Emissive::DirectLighting (emissive.cpp:61-74); the path ends here.
                if (le && !inobj && -dot3(d, nrm) > 0.0f) addL = beta * m.le;
            } else {
                const float3 wo = -d;
                BsdfSample b;
                float3 vol_ratio = mk3(1, 1, 1), volw = mk3(1, 1, 1);
                bool walk_scatter = false, absorbed = false;
                if (m.type == MAT_SUBSURFACE && inobj) {
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
                if (!absorbed) {
                    // NEE: Matte::DirectLighting (matte.cpp:54-82); Glossy only on its
                    // diffuse lobe, divided by kd_pdf (glossy.cpp:92-102)
                    const bool nee = S.n_lights > 0 && !walk_scatter &&
                                     (m.type == MAT_MATTE ||
                                      (m.type == MAT_GLOSSY && m.kd != 0.0f && b.xi <= m.kd_pdf));
                    if (nee) {
                        const LightSample ls = sample_light(S, U0.u[3], U1.u[0], U1.u[1]);
                        float3 wi;
                        float dist, G;
                        if (nee_setup(ls, p, wi, dist, G)) {
                            const float3 f = albedo * RUMI_INV_PI_F * m.kd;
                            const float cost = fmaxf(dot3(wi, nrm), 0.0f);
                            float3 direct = f * ls.Li * cost * G / ls.pdf;
                            if (m.type == MAT_GLOSSY) direct = direct * (1.0f / m.kd_pdf);
                            float tr = 1.0f;
                            if (V.present) {
                                const Uniform4 U2 = path_uniforms(path, bounce, 2, k0, k1);
                                tr = volume_shadow_tr(V, p, wi, dist, U2.u[2]);
                            }
                            if (tr > 0.0f) {
                                want_sh = true;
                                sh_o = p;
                                sh_d = wi;
                                sh_tmax = dist;
                                sh_c = beta * direct;
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
    const int kn = warp_push(&P.cnt[nxt], want_next);
    const int ks = warp_push(&P.cnt[C_SHADOW], want_sh);
    if (want_next) {
        P.ray_o[nxt][kn] = make_float4(nx_o.x, nx_o.y, nx_o.z,
                                       __int_as_float(slot | ((nx_flags & PFL_IN) ? (int)0x80000000 : 0)));
        P.ray_d[nxt][kn] = make_float4(nx_d.x, nx_d.y, nx_d.z, FLT_MAX);
        P.beta[slot] = make_float4(beta.x, beta.y, beta.z, 0.0f);
        P.pflags[slot] = nx_flags;
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

// Device bytes of the wave state for `paths` paths in flight (queues, path state,
// counters): 164 bytes per path plus alignment and counters.
size_t pt_workspace_bytes(long long paths) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t Wp = (size_t)paths;
    return 10 * al(Wp * sizeof(float4)) + al(Wp * sizeof(unsigned)) + al(C_NUM * sizeof(int)) +
           al(S_NUM * sizeof(unsigned long long));
}

rumi_status pt_render(rumi_scene *sc, const rumi_render_params *p, float *film_dev, rumi_render_stats *stats,
                      cudaStream_t stream) {
    const long long total_pix = (long long)sc->dev.width * sc->dev.height;
    long long wave = p->wave_paths > 0 ? p->wave_paths : (1 << 22);
    long long pix_per_wave = wave / p->spp;
    if (pix_per_wave < 1) pix_per_wave = 1;
    if (pix_per_wave > total_pix) pix_per_wave = total_pix;
    const long long n_paths_max = pix_per_wave * p->spp;
    if (n_paths_max > 0x7fffffffLL) {
        set_error("wave_paths too large");
        return RUMI_ERR_INVALID_ARG;
    }
    rumi_status st = ensure_workspace(sc, pt_workspace_bytes(n_paths_max));
    if (st != RUMI_OK) return st;
    return pt_render_in(sc, p, film_dev, stats, stream, sc->ws, pix_per_wave);
}

// The frame loop over waves of pix_per_wave pixels, with the wave state carved out of
// `ws` (pt_workspace_bytes(pix_per_wave * spp) bytes).
rumi_status pt_render_in(rumi_scene *sc, const rumi_render_params *p, float *film_dev, rumi_render_stats *stats,
                         cudaStream_t stream, void *ws, long long pix_per_wave) {
    const int W = sc->dev.width, H = sc->dev.height;
    const int spp = p->spp;
    const long long total_pix = (long long)W * H;
    const size_t Wp = (size_t)(pix_per_wave * spp);
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t f4 = al(Wp * sizeof(float4));
    char *w = (char *)ws;
    PtLaunch L;
    L.s = sc->dev;
    L.spp = spp;
    L.max_depth = p->max_depth;
    L.k0 = (uint32_t)p->seed;
    L.k1 = (uint32_t)(p->seed >> 32) ^ 0x5851F42Du;
    int d = 0;
    while ((d + 1) * (d + 1) <= spp) ++d;
    L.grid_d = d;
    L.square = d * d == spp;
    L.ray_o[0] = (float4 *)w; w += f4;
    L.ray_o[1] = (float4 *)w; w += f4;
    L.ray_d[0] = (float4 *)w; w += f4;
    L.ray_d[1] = (float4 *)w; w += f4;
    L.hit = (float4 *)w; w += f4;
    L.sh_o = (float4 *)w; w += f4;
    L.sh_d = (float4 *)w; w += f4;
    L.sh_c = (float4 *)w; w += f4;
    L.beta = (float4 *)w; w += f4;
    L.L = (float4 *)w; w += f4;
    L.pflags = (unsigned *)w; w += al(Wp * sizeof(unsigned));
    L.cnt = (int *)w; w += al(C_NUM * sizeof(int));
    L.stats = (unsigned long long *)w; w += al(S_NUM * sizeof(unsigned long long));
    L.film = film_dev;
    L.scenes = nullptr;
    L.scene_path0 = L.scene_pix0 = nullptr;
    L.scene_key = nullptr;
    L.scene_spp = nullptr;
    L.n_scenes = 0;
    L.slot_scene = nullptr;
    cudaMemsetAsync(L.cnt, 0, C_NUM * sizeof(int), stream);
    cudaMemsetAsync(L.stats, 0, S_NUM * sizeof(unsigned long long), stream);

    // traversal scheme and persistent grid (autotuner knobs; 0 = defaults)
    const int mode = p->trace_mode >= 1 && p->trace_mode <= 3 ? p->trace_mode - 1 : 0;
    L.refill_min = p->refill_min > 0 ? p->refill_min : 8;
    int occ = 0, occ_sh = 0;
    if (mode == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pt_extend<0, false>, TRACE_THREADS, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sh, pt_shadow<0>, TRACE_THREADS, 0);
    } else if (mode == 1) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pt_extend<1, false>, TRACE_THREADS, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sh, pt_shadow<1>, TRACE_THREADS, 0);
    } else {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pt_extend<2, false>, TRACE_THREADS, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sh, pt_shadow<2>, TRACE_THREADS, 0);
    }
    if (occ < 1) occ = 1;
    if (occ_sh < 1) occ_sh = 1;
    if (p->blocks_per_sm > 0) {
        occ = p->blocks_per_sm < occ ? p->blocks_per_sm : occ;
        occ_sh = p->blocks_per_sm < occ_sh ? p->blocks_per_sm : occ_sh;
    }
    const int trace_grid = sc->num_sms * occ;
    const int shadow_grid = sc->num_sms * occ_sh;

    const bool timing = (p->flags & RUMI_FLAG_TIMING) != 0;
    const bool count_stats = (p->flags & RUMI_FLAG_STATS) != 0;
    std::vector<cudaEvent_t> evs;
    auto mark = [&]() {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, stream);
        evs.push_back(e);
    };
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
        for (int b = 0; b < p->max_depth; ++b) {
            pt_reset<<<1, 1, 0, stream>>>(L, b);
            int e0 = 0;
            if (timing) { e0 = (int)evs.size(); mark(); }
            if (count_stats)
                pt_extend<0, true><<<trace_grid, TRACE_THREADS, 0, stream>>>(L, b);
            else if (mode == 0)
                pt_extend<0, false><<<trace_grid, TRACE_THREADS, 0, stream>>>(L, b);
            else if (mode == 1)
                pt_extend<1, false><<<trace_grid, TRACE_THREADS, 0, stream>>>(L, b);
            else
                pt_extend<2, false><<<trace_grid, TRACE_THREADS, 0, stream>>>(L, b);
            if (timing) { mark(); ext_ev.push_back({e0, e0 + 1}); }
            if (timing) { e0 = (int)evs.size(); mark(); }
            pt_shade<<<cdiv(L.n_paths, SHADE_THREADS), SHADE_THREADS, 0, stream>>>(L, b);
            if (timing) { mark(); shade_ev.push_back({e0, e0 + 1}); }
            if (timing) { e0 = (int)evs.size(); mark(); }
            if (mode == 0)
                pt_shadow<0><<<shadow_grid, TRACE_THREADS, 0, stream>>>(L);
            else if (mode == 1)
                pt_shadow<1><<<shadow_grid, TRACE_THREADS, 0, stream>>>(L);
            else
                pt_shadow<2><<<shadow_grid, TRACE_THREADS, 0, stream>>>(L);
            if (timing) { mark(); sh_ev.push_back({e0, e0 + 1}); }
        }
        pt_finish<<<1, 1, 0, stream>>>(L);
        pt_resolve<<<cdiv(L.n_pix * 32LL, 256), 256, 0, stream>>>(L);
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
        stats->extend_node_fetches = (int64_t)h_stats[S_NODES];
        stats->extend_prim_tests = (int64_t)h_stats[S_PRIMS];
        stats->extend_launches = (int64_t)waves * p->max_depth;
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

// ---------------------------------------------------------------- scene batches
// Device bytes of a multi-scene wave: the single-scene wave state plus each slot's scene.
size_t pt_batch_workspace_bytes(long long wave_paths) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return pt_workspace_bytes(wave_paths) + al((size_t)wave_paths * sizeof(int));
}

// Enqueues one frame of a multi-scene batch without synchronising, so the sequence can
// be captured into a CUDA graph: waves over the batch's global pixel / path index space,
// every stage serving all scenes from shared queues.
rumi_status pt_enqueue_batch(const BatchFrame &F, void *ws, float *films, cudaStream_t stream, int num_sms) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t Wp = (size_t)F.wave_paths;
    const size_t f4 = al(Wp * sizeof(float4));
    char *w = (char *)ws;
    PtLaunch L;
    memset(&L, 0, sizeof(L));
    L.max_depth = F.max_depth;
    L.ray_o[0] = (float4 *)w; w += f4;
    L.ray_o[1] = (float4 *)w; w += f4;
    L.ray_d[0] = (float4 *)w; w += f4;
    L.ray_d[1] = (float4 *)w; w += f4;
    L.hit = (float4 *)w; w += f4;
    L.sh_o = (float4 *)w; w += f4;
    L.sh_d = (float4 *)w; w += f4;
    L.sh_c = (float4 *)w; w += f4;
    L.beta = (float4 *)w; w += f4;
    L.L = (float4 *)w; w += f4;
    L.pflags = (unsigned *)w; w += al(Wp * sizeof(unsigned));
    L.cnt = (int *)w; w += al(C_NUM * sizeof(int));
    L.stats = (unsigned long long *)w; w += al(S_NUM * sizeof(unsigned long long));
    L.slot_scene = (int *)w;
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
        for (int b = 0; b < F.max_depth; ++b) {
            pt_reset<<<1, 1, 0, stream>>>(L, b);
            pt_trace_multi<false><<<num_sms * occ, TRACE_THREADS, 0, stream>>>(L, b);
            pt_shade<<<cdiv(L.n_paths, SHADE_THREADS), SHADE_THREADS, 0, stream>>>(L, b);
            pt_trace_multi<true><<<num_sms * occ_sh, TRACE_THREADS, 0, stream>>>(L, b);
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
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t Wp = (size_t)wave_paths;
    const size_t off = 10 * al(Wp * sizeof(float4)) + al(Wp * sizeof(unsigned)) + al(C_NUM * sizeof(int));
    return (unsigned long long *)((char *)ws + off);
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

template <bool ANYHIT>
__global__ void __launch_bounds__(TRACE_THREADS) trace_batch_kernel(TraceLaunch T) {
    __shared__ int stack[STACK_SMEM * TRACE_THREADS];
    const int lane = threadIdx.x & 31;
    TraceStats st{0, 0};
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&T.counters[0], 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= (unsigned long long)T.n) break;
        const long long i = (long long)base + lane;
        if (i < T.n) {
            const float4 o4 = T.rays[2 * i], d4 = T.rays[2 * i + 1];
            const HitRec h = trace_ray<ANYHIT, STACK_SMEM, true>(T.s, f4xyz(o4), f4xyz(d4), d4.w, o4.w != 0.0f,
                                                                 stack + threadIdx.x, TRACE_THREADS, st);
            T.t[i] = h.t;
            T.prim[i] = ANYHIT ? (h.t > 0.0f ? 1 : 0) : (h.t > 0.0f ? h.id : -1);
        }
    }
    atomicAdd(&T.counters[1], (unsigned long long)st.nodes);
    atomicAdd(&T.counters[2], (unsigned long long)st.prims);
}

rumi_status trace_rays(rumi_scene *sc, int64_t n, const float *rays_dev, int anyhit, float *t_dev, int32_t *prim_dev,
                       int64_t *node_visits, int64_t *prim_tests, cudaStream_t stream) {
    rumi_status st = ensure_workspace(sc, 256);
    if (st != RUMI_OK) return st;
    TraceLaunch T;
    T.s = sc->dev;
    T.rays = (const float4 *)rays_dev;
    T.t = t_dev;
    T.prim = prim_dev;
    T.n = n;
    T.anyhit = anyhit;
    T.counters = (unsigned long long *)sc->ws;
    cudaMemsetAsync(T.counters, 0, 3 * sizeof(unsigned long long), stream);
    int occ = 0;
    if (anyhit)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, trace_batch_kernel<true>, TRACE_THREADS, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, trace_batch_kernel<false>, TRACE_THREADS, 0);
    if (occ < 1) occ = 1;
    const int grid = sc->num_sms * occ;
    if (n > 0) {
        if (anyhit)
            trace_batch_kernel<true><<<grid, TRACE_THREADS, 0, stream>>>(T);
        else
            trace_batch_kernel<false><<<grid, TRACE_THREADS, 0, stream>>>(T);
    }
    unsigned long long h[3] = {0, 0, 0};
    cudaMemcpyAsync(h, T.counters, sizeof(h), cudaMemcpyDeviceToHost, stream);
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_status(e, "trace_rays");
    if (node_visits) *node_visits = (int64_t)h[1];
    if (prim_tests) *prim_tests = (int64_t)h[2];
    return RUMI_OK;
}

}  // namespace rumi
