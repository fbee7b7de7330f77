// Bidirectional path tracing with multiple importance sampling, restating
// BidirectionalPathTracer (src/Integrator/bidirectionalpathtracer.cpp):
//   Trace                 :121-394  all (s, t) strategies of one camera sample
//   ConstructViewPath     :396-711  camera subpath with area-measure pdfs and throughput
//   ConstructLightPath    :713-1016 light subpath
//   VisibilityTest        :1018-1050
//   VolumetricTest        :1052-1094
//   MISWeight             :1096-1586 balance heuristic over pdf ratios, "locked" rule
// One thread renders one camera sample: both subpaths live in per-thread arrays
// (the reference's Path[] / Color[] members), pdfs are RGB because medium pdfs are.
// Light-tracing strategies (t = 1, the camera vertex) splat through the film plane
// into a separate buffer with atomic adds, added to the pixel sums at the end (the
// reference's Film::LightPixel + CombineBuffer, src/Camera/film.cpp:99-150).
#include "renderer.h"
#include "traverse.cuh"
#include "shading.cuh"
#include "camera.cuh"

namespace rumi {


// Every index this file forms into a local subpath array or a scene array goes through
// bd_index: none can leave its range by construction, and an index that did would be
// recorded here (check code, index, bound, sample thread) and replaced by 0, and
// bdpt_render would return RUMI_ERR_INTERNAL naming it, instead of the kernel reading or
// writing out of range.  The kernel builds without these checks raised illegal-address
// faults in some configurations (a scene with two area lights in a medium, among others)
// without any index leaving its range in the checked build; the checked build runs them
// all.  One word for the process: a check that fires during concurrent BDPT renders on
// several streams is reported by whichever render reads it first.
__device__ int g_bd_range[4];
// Records the first out-of-range index; out of line, so each checked access costs a
// compare and a branch.
__device__ RUMI_NOINLINE void bd_index_fail(int idx, int n, int code) {
    if (atomicCAS(&g_bd_range[0], 0, code) == 0) {
        g_bd_range[1] = idx;
        g_bd_range[2] = n;
        g_bd_range[3] = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    }
}
// idx when it lies in [0, n); otherwise the failure is recorded and 0 is used instead.
RUMI_D int bd_index(int idx, int n, int code) {
    if (__builtin_expect((unsigned)idx < (unsigned)n, 1)) return idx;
    bd_index_fail(idx, n, code);
    return 0;
}
static constexpr int BD_THREADS = 64;
static constexpr int BD_STACK = 32;
static constexpr int BD_MAXV = 16;  // vertices per subpath (nE, nL <= 16)
// The kernel is instantiated for MAXV = 8 and 16: its per-thread subpath arrays live in
// local memory, and sizing them to the request halves that traffic for nL, nE <= 8.

struct BVert {
    float3 p, n;
    float3 pdf_fwd, pdf_bwd;  // _pdf_pforward / _pdf_pbackward (area measure)
    float pdf_dir;            // _pdf_wi (eye) / _pdf_wo (light) of the sampled outgoing direction
    float pdf_path;           // _pdf_path (lobe probability)
    float cos_a;              // eye: _costheta_i, light: _costheta_o (outgoing side)
    float cos_b;              // eye: _costheta_o, light: _costheta_i (arriving side)
    bool dirac, onsurface;
    // Intersection of the segment arriving at this vertex
    int mat;                  // material index of the hit surface (-1: none)
    int prim;
    float xi;                 // _rand
    bool in_obj;              // _in_object
    float t_in;               // ray _tmin
    float3 d_in;              // direction of the arriving segment
    float3 vtau, vpdf;        // _volumetric_tau / _volumetric_pdf
};

RUMI_D void bvert_clear(BVert &v) {
    v.p = v.n = mk3(0, 0, 0);
    v.pdf_fwd = v.pdf_bwd = mk3(1, 1, 1);
    v.pdf_dir = 1.0f;
    v.pdf_path = 1.0f;
    v.cos_a = v.cos_b = 1.0f;
    v.dirac = false;
    v.onsurface = true;
    v.mat = -1;
    v.prim = -1;
    v.xi = 1.0f;
    v.in_obj = false;
    v.t_in = 0.0f;
    v.d_in = mk3(0, 0, 0);
    v.vtau = v.vpdf = mk3(1, 1, 1);
}

struct BdLaunch {
    DevScene s;
    int nL, nE, spp;
    uint32_t k0, k1;
    int grid_d, square;
    long long path0;
    int n_paths, pix0;
    float4 *L;           // per-path radiance (sample value of Trace)
    float *light_film;   // H*W*3 (B,G,R) light-tracing splats
    float3 right, up;    // camera basis (film plane)
};

RUMI_D float3 c3(float v) { return mk3(v, v, v); }

// Spot lights (not in the reference): a point at `position` emitting intensity I (per
// steradian) uniformly inside the cone of half-angle acos(cos_cone) about `direction`.
// As the light vertex of a subpath it is a delta position: no eye subpath can hit it,
// its "emission" is I, it has no cosine of its own, and its emission directions are
// drawn uniformly from the cone.
RUMI_D float3 light_emission(const DevLight &l) { return l.type == LIGHT_SPOT ? l.intensity : l.le; }

RUMI_D float spot_pdf_dir(const DevLight &l) { return 1.0f / (2.0f * RUMI_PI_F * (1.0f - l.cos_cone)); }

RUMI_D float3 spot_sample_dir(const DevLight &l, float u1, float u2) {
    float3 u, w;
    onb_ref(l.direction, u, w);
    const float ct = 1.0f - u2 * (1.0f - l.cos_cone);
    const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float sphi, cphi;
    sincosf(u1 * 2.0f * RUMI_PI_F, &sphi, &cphi);
    return normalize_ref(frame_dir(u, l.direction, w, st * sphi, ct, st * cphi));
}

// HomogeneousVolume::Tr over [0, s] (homogeneousvolume.cpp:46-54)
RUMI_D float3 vol_tr(const DevVolume &V, float s) {
    return mk3(expf(V.sigma_t.x * -s), expf(V.sigma_t.y * -s), expf(V.sigma_t.z * -s));
}
// HomogeneousVolume::PdfDistance (homogeneousvolume.cpp:100-111)
RUMI_D float3 vol_pdf_distance(const DevVolume &V, float s) {
    float3 pdf = vol_tr(V, s) * V.sigma_t;
    if (pdf.x == 0.0f && pdf.y == 0.0f && pdf.z == 0.0f) pdf = c3(1e-4f);
    return pdf;
}
// Scattering-ray segment as MISWeight / the subpath loops form it: Intersect (return
// value ignored where the reference ignores it), MaxDistance.
RUMI_D float vol_segment(const DevVolume &V, float3 o, float3 d, float tmax, bool &hit) {
    float tn, tf;
    hit = volume_intersect(V, o, d, 0.0f, tn, tf);
    return volume_max_distance(tmax, tn, tf);
}

// Pinhole::FilmPlaneIntersection (pinhole.cpp:138-167) with the film plane of
// Pinhole::AddFilmPlane (pinhole.cpp:64-82).
RUMI_D bool film_plane_pixel(const BdLaunch &P, float3 pos, int &wi, int &hi) {
    const DevCamera &c = P.s.camera;
    const float width = 2.0f * c.tanfov, height = 2.0f * c.tanfov * c.y_ratio;
    float3 sp = c.p - P.right * (0.5f * width);
    sp = sp - P.up * (0.5f * height);
    sp = sp + c.dir * c.plane_dist;
    const float3 lv = P.right * width, wv = P.up * height;
    const float3 d = normalize_ref(c.p - pos);
    float t;
    // the film plane Rect carries no material: two-sided
    if (!isect_rect(pos, d, FLT_MAX, 0.0f, make_float4(sp.x, sp.y, sp.z, 0), make_float4(lv.x, lv.y, lv.z, 0),
                    make_float4(wv.x, wv.y, wv.z, 0), true, t))
        return false;
    const float3 ip = pos + d * t;
    const float3 on = ip - sp;
    const float llen = sqrtf(dot3(lv, lv)), wlen = sqrtf(dot3(wv, wv));
    float u = dot3(on, lv) / (llen * llen);
    float v = dot3(on, wv) / (wlen * wlen);
    u = (float)P.s.width * (1.0f - u);
    v = (float)P.s.height * (1.0f - v);
    if (u == (float)P.s.width) u -= 1.0f;
    if (v == (float)P.s.height) v -= 1.0f;
    wi = (int)u;
    hi = (int)v;
    return true;
}

// Hit -> vertex fields (position, normal, material).
RUMI_D void record_hit(const DevScene &S, const HitRec &h, float3 o, float3 d, BVert &v) {
    v.p = rn_madd(o, d, h.t);
    v.prim = h.id;
    v.mat = prim_material(S, bd_index(h.id, S.n_prims, 31));
    v.n = surface_normal(S, h.id, h.back != 0, h.u, h.v, o, v.p, S.materials[bd_index(v.mat, S.n_materials, 1)]);
}

RUMI_D float3 vert_albedo(const DevScene &S, const BVert &v, const DevMaterial &m) {
    if (S.tri_albedo && v.prim >= 0 && v.prim < S.n_tris) return f4xyz(__ldg(&S.tri_albedo[v.prim]));
    return m.rgb;
}

// Material::Fr with the vertex's arriving Intersection state.
RUMI_D float3 vert_fr(const DevScene &S, const BVert &v, float3 n, float3 wi, float3 wo) {
    const DevMaterial m = S.materials[bd_index(v.mat, S.n_materials, 2)];
    return material_fr(m, vert_albedo(S, v, m), n, wi, wo, v.in_obj, v.xi, v.pdf_path, v.t_in, v.vtau / v.vpdf);
}

// Subpath construction shared by both directions.  eye: ConstructViewPath, else
// ConstructLightPath.  V[0] is prepared by the caller; seg_d[k] receives the direction of
// the segment from V[k] to V[k+1]; alpha[] the subpath throughputs.  Returns the vertex count.
// The direction is a run-time argument: the caller's one call site serves both subpaths,
// so the kernel holds one copy of this code (the kernel is bound by instruction fetch).
RUMI_D int construct_subpath(const BdLaunch &P, bool eye, int max_depth, uint64_t path, uint32_t stream_base,
                             float3 o, float3 d, BVert *V, float3 *seg_d, float3 *alpha, const DevLight &light,
                             float3 light_n, int *stack, TraceStats &st) {
    const DevScene &S = P.s;
    const DevVolume &vol = S.volume;
    bool in_object = false;
    alpha[0] = c3(1.0f);
    int n_vertex = 1;
    float3 prev_w = mk3(0, 0, 0);  // prev_wo (eye) / prev_wi (light)
    const int max_seg = max_depth - 1;  // the reference's Path[max_depth - 1] array
    for (int depth = 0; depth < max_depth && depth < max_seg; ++depth) {
        BVert &start = V[depth];
        BVert &end = V[bd_index(depth + 1, max_depth, 28)];
        bvert_clear(end);
        end.in_obj = in_object;
        end.d_in = d;
        seg_d[bd_index(depth, max_depth, 30)] = d;
        const Uniform4 U0 = path_uniforms(path, stream_base + depth, 0, P.k0, P.k1);
        const Uniform4 U1 = path_uniforms(path, stream_base + depth, 1, P.k0, P.k1);
        const HitRec h = trace_ray<false, BD_STACK, false>(S, o, d, FLT_MAX, in_object, stack, BD_THREADS, st);
        const bool hit = h.t > 0.0f;
        end.t_in = h.t;
        if (hit) record_hit(S, h, o, d, end);
        float vol_s = 0.0f;
        bool absorb = false;
        if (vol.present && !in_object) {
            float tn, tf;
            if (volume_intersect(vol, o, d, h.t, tn, tf)) {
                const float smax = volume_max_distance(h.t, tn, tf);
                const DistSample ds = distance_sample(vol.sigma_t, vol.avg_sigma_t, vol.absorb, smax, U1.u[2], U1.u[3]);
                if (ds.outcome == 2) {
                    absorb = true;
                } else {
                    end.vtau = ds.tau;
                    end.vpdf = ds.pdf;
                    if (ds.outcome == 1) {
                        vol_s = ds.s;
                        end.p = o + d * (tn < 0.0f ? ds.s : tn + ds.s);
                        end.onsurface = false;
                    }
                }
            }
            if (absorb) break;
        }
        if (!hit && vol_s == 0.0f) break;
        ++n_vertex;
        const bool has_mat = end.mat >= 0;
        DevMaterial m;
        if (has_mat) m = S.materials[bd_index(end.mat, S.n_materials, 3)];
        const float3 wrev = -d;  // wo (eye) / wi (light)
        float3 w, n;
        float pdf_dir = 1.0f;
        if (end.onsurface) {
            n = end.n;
            const BsdfSample b = material_sample(m, wrev, n, U0.u[0], U0.u[1], U0.u[2]);
            w = b.w;
            in_object = b.go_in;
            end.xi = b.xi;
            end.pdf_path = b.pdf_path;
            end.cos_a = b.cost;
            pdf_dir = b.pdfw;
            end.pdf_dir = pdf_dir;
            end.dirac = material_dirac(m, b.xi);
        } else {
            n = mk3(0, 0, 0);
            if (vol.g == 0.0f) {
                w = isotropic_dir(d, U0.u[1], U0.u[2]);
                pdf_dir = 1.0f / (4.0f * RUMI_PI_F);
            } else {
                w = hg_sample(d, vol.g, U0.u[1], U0.u[2], pdf_dir);
            }
            in_object = false;
            end.pdf_dir = pdf_dir;
            end.dirac = false;
        }
        // cosine at the start vertex on its outgoing side
        float cos_s;
        if (start.onsurface) {
            const bool use_stored = eye ? (depth == 0 || !start.dirac) : !start.dirac;
            if (use_stored) {
                cos_s = start.cos_a;
            } else {
                cos_s = !end.in_obj ? dot3(d, start.n) : -dot3(d, start.n);
                if (cos_s <= 0.0f) cos_s = 1e-4f;
                start.cos_a = cos_s;
            }
        } else {
            cos_s = 1.0f;
            start.cos_a = 1.0f;
        }
        // cosine at the end vertex on its arriving side
        float cos_e;
        if (end.onsurface) {
            cos_e = !end.in_obj ? -dot3(d, end.n) : dot3(d, end.n);
            if (cos_e <= 0.0f) cos_e = 1e-4f;
        } else {
            cos_e = 1.0f;
        }
        end.cos_b = cos_e;
        // forward pdf of the end vertex
        const float3 se = end.p - start.p;
        const float dist = sqrtf(dot3(se, se));
        float dwda = cos_e / (dist * dist);
        float fwd;
        if (start.onsurface) {
            const bool plain = eye ? (depth == 0 || !start.dirac) : !start.dirac;
            fwd = plain ? start.pdf_dir * dwda : start.pdf_dir * dwda * start.cos_a;
        } else {
            fwd = start.pdf_dir * dwda * start.cos_a;
        }
        end.pdf_fwd = c3(fwd);
        if (vol.present && !end.in_obj) end.pdf_fwd = end.pdf_fwd * end.vpdf;
        // backward pdf of the start vertex
        dwda = cos_s / (dist * dist);
        const bool end_le = has_mat && m.type == MAT_EMISSIVE;
        // the end surface's pdf of the reversed direction (both start kinds use it)
        const float pw_end = end.onsurface && !end_le ? material_pdfw(m, end.xi, n, w, wrev) : 0.0f;
        float3 bwd;
        if (start.onsurface) {
            if (end.onsurface) {
                float pw;
                if (end_le) {
                    // AreaLight::Pdfw(w) with the light's stored normal
                    float c = dot3(wrev, light_n);
                    if (c <= 0.0f) c = 1e-4f;
                    pw = RUMI_INV_PI_F * c;
                    if (pw <= 0.0f) pw = 1e-4f;
                    bwd = c3(pw * dwda);
                } else {
                    pw = pw_end;
                    bwd = end.dirac ? c3(pw * dwda * end.cos_b) : c3(pw * dwda);
                }
                if (vol.present && !end.in_obj) bwd = bwd * end.vpdf;
            } else {
                bool vh;
                const float sm = vol_segment(vol, end.p, -d, dist, vh);
                bwd = vol_tr(vol, sm) * (phase_value(vol, w, wrev) * dwda * end.cos_b);
            }
        } else {
            bool vh;
            const float sm = vol_segment(vol, end.p, -d, dist, vh);
            const float3 pdf_s = vol_pdf_distance(vol, sm);
            if (end.onsurface) {
                if (end_le) {
                    float c = dot3(wrev, light_n);
                    if (c <= 0.0f) c = 1e-4f;
                    float pw = RUMI_INV_PI_F * c;
                    if (pw <= 0.0f) pw = 1e-4f;
                    bwd = pdf_s * (pw * dwda);
                } else {
                    const float pw = pw_end;
                    bwd = end.dirac ? pdf_s * (pw * dwda * end.cos_b) : pdf_s * (pw * dwda);
                }
            } else {
                bwd = pdf_s * (phase_value(vol, w, wrev) * dwda * end.cos_b);
            }
        }
        start.pdf_bwd = bwd;
        // throughput
        const float G = cos_s * cos_e / (dist * dist);
        float3 a = alpha[depth];
        if (start.onsurface) {
            if (depth == 0) {
                if (eye) {
                    const DevCamera &c = S.camera;
                    const float cs = start.cos_a;
                    const float We = c.plane_dist * c.plane_dist / (c.film_area * cs * cs * cs * cs);
                    a = a * (We / avg3(start.pdf_fwd) * G);
                } else {
                    a = a * (light_emission(light) / start.pdf_fwd * G);  // Light::L / pick pdf
                }
            } else {
                const float3 fr = vert_fr(S, start, start.n, eye ? d : prev_w, eye ? prev_w : d);
                a = a * (fr / (start.pdf_fwd * start.pdf_path) * G);
                // the surface's texture (bidirectionalpathtracer.cpp:660-661, 971-972)
                if (S.prim_tex && start.prim >= 0) a = a * tex_pattern(S, start.prim, start.p);
            }
        } else {
            const float fp = phase_value(vol, eye ? d : prev_w, eye ? prev_w : d);
            a = a * ((vol.sigma_s * fp) / (start.pdf_fwd * start.pdf_path) * G);
        }
        if (vol.present && !end.in_obj) a = a * end.vtau;
        alpha[depth + 1] = a;
        if (eye) {
            if (end_le) {
                const float3 fr = end.onsurface ? vert_fr(S, end, n, w, wrev) : mk3(0, 0, 0);
                alpha[bd_index(depth + 2, max_depth + 1, 29)] = a * (fr / (end.pdf_fwd * end.pdf_path));
                end.pdf_bwd = c3(light.inv_area * (float)S.n_lights);  // Light::Pdf() * LightCount()
                break;
            }
        } else {
            if (end.onsurface && end_le) break;
        }
        prev_w = wrev;
        o = end.p;
        d = w;
    }
    return n_vertex;
}

// AreaLight::Pdfw (arealight.cpp:62-73) with the light's normal.
RUMI_D float light_pdfw(float3 w, float3 light_n) {
    float c = dot3(w, light_n);
    if (c <= 0.0f) c = 1e-4f;
    float pdf = RUMI_INV_PI_F * c;
    return pdf <= 0.0f ? 1e-4f : pdf;
}

// Pinhole::Pdfw (pinhole.cpp:58-62)
RUMI_D float camera_pdfw(const DevCamera &c, float3 w) {
    const float ct = dot3(w, c.dir);
    return c.plane_dist * c.plane_dist / (ct * ct * ct * c.film_area);
}

// BidirectionalPathTracer::MISWeight (bidirectionalpathtracer.cpp:1096-1586).
// ns / nt: vertices used on the light / eye side; VL / VE the subpaths, segL / segE
// their segment directions.
template <int MAXV>
RUMI_D float mis_weight(const BdLaunch &P, const BVert *VL, const float3 *segL, const BVert *VE, const float3 *segE,
                        int ns, int nt, float3 connect_wi, float3 connect_wo, float3 light_n, const DevLight &light) {
    if (ns + nt <= 2) return 1.0f;
    const DevScene &S = P.s;
    const DevVolume &vol = S.volume;
    float3 sb[MAXV], sf[MAXV], tb[MAXV], tf[MAXV];
    const BVert *s_connect = nullptr, *s_prev = nullptr, *t_connect = nullptr, *t_prev = nullptr;
    float3 s_wi = mk3(0, 0, 0), t_wo = mk3(0, 0, 0);
    if (ns > 0) {
        s_connect = &VL[bd_index(ns - 1, MAXV, 17)];
        if (ns >= 2) {
            s_prev = &VL[bd_index(ns - 2, MAXV, 17)];
            s_wi = -segL[bd_index(ns - 2, MAXV, 19)];
        }
    }
    if (nt > 0) {
        t_connect = &VE[bd_index(nt - 1, MAXV, 18)];
        if (nt >= 2) {
            t_prev = &VE[bd_index(nt - 2, MAXV, 18)];
            t_wo = -segE[bd_index(nt - 2, MAXV, 20)];
        }
    }
    float connect_d = 1.0f, sd = 1.0f, td = 1.0f;
    if (s_connect && t_connect) connect_d = sqrtf(dot3(s_connect->p - t_connect->p, s_connect->p - t_connect->p));
    if (s_connect && s_prev) sd = sqrtf(dot3(s_connect->p - s_prev->p, s_connect->p - s_prev->p));
    if (t_connect && t_prev) td = sqrtf(dot3(t_connect->p - t_prev->p, t_connect->p - t_prev->p));

    // The two connection-side blocks of MISWeight mirror each other: side 0 gives the light
    // vertex X = s_connect the pdf of being sampled from Y = t_connect (sb / sf) and its
    // predecessor the pdf of being sampled from X; side 1 the same with the roles swapped
    // (tb / tf).  One loop body serves both, so the kernel holds one copy of this code.
    // pdf of sampling X from Y along the connection in the reference's form: Tr (surface
    // end) or PdfDistance (medium end) of the segment, times the density of the direction
    // at Y (a material, the camera or the light at a subpath's first vertex, or the phase
    // function in the medium).
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        const bool sl = side == 0;
        const BVert *X = sl ? s_connect : t_connect, *Y = sl ? t_connect : s_connect;
        const BVert *Xp = sl ? s_prev : t_prev;
        if (!X || !Y) continue;                                       // ns == 0: side 1 below
        const int nx = sl ? ns : nt, ny = sl ? nt : ns;
        const float3 y_to_x = sl ? connect_wi : connect_wo, x_to_y = sl ? connect_wo : connect_wi;
        const float3 y_in = sl ? t_wo : s_wi, x_in = sl ? s_wi : t_wo;  // toward Y's / X's predecessor
        const float xd = sl ? sd : td;
        float3 *xb = sl ? sb : tb, *xf = sl ? sf : tf;
        float3 pdf_s = c3(1.0f);
        float dwda;
        if (X->onsurface) {
            if (vol.present) {
                bool vh;
                const float sm = vol_segment(vol, Y->p, y_to_x, connect_d, vh);
                if (vh) pdf_s = vol_tr(vol, sm);
            }
            dwda = dot3(X->n, x_to_y) / (connect_d * connect_d);
        } else {
            dwda = 1.0f / (connect_d * connect_d);
            bool vh;
            const float sm = vol_segment(vol, Y->p, y_to_x, connect_d, vh);
            if (vh) pdf_s = vol_pdf_distance(vol, sm);
        }
        float pw;
        if (Y->onsurface) {
            if (ny > 1)
                pw = material_pdfw(S.materials[bd_index(Y->mat, S.n_materials, 4)], Y->xi, Y->n, y_in, y_to_x);
            else if (sl)
                pw = camera_pdfw(S.camera, connect_wi);
            else
                pw = light.type == LIGHT_SPOT ? spot_pdf_dir(light) : light_pdfw(connect_wo, light_n);
        } else {
            pw = phase_value(vol, y_in, y_to_x);
        }
        xb[bd_index(nx - 1, MAXV, 11)] = pdf_s * (pw * dwda);
        xf[bd_index(nx - 1, MAXV, 11)] = X->pdf_fwd;
        if (Xp) {
            if (Xp->onsurface && Xp->dirac) {
                xb[nx - 2] = c3(1.0f);
                xf[nx - 2] = c3(1.0f);
            } else {
                float3 ps = c3(1.0f);
                float dw;
                if (Xp->onsurface) {
                    if (vol.present) {
                        bool vh;
                        const float sm = vol_segment(vol, X->p, x_in, xd, vh);
                        if (vh) ps = vol_tr(vol, sm);
                    }
                    dw = -dot3(Xp->n, x_in) / (xd * xd);
                } else {
                    dw = 1.0f / (xd * xd);
                    bool vh;
                    const float sm = vol_segment(vol, X->p, x_in, xd, vh);
                    if (vh) ps = vol_pdf_distance(vol, sm);
                }
                const float pw2 = X->onsurface
                                      ? material_pdfw(S.materials[bd_index(X->mat, S.n_materials, 5)], X->xi, X->n, x_to_y, x_in)
                                      : phase_value(vol, x_to_y, x_in);
                xb[bd_index(nx - 2, MAXV, 12)] = ps * (pw2 * dw);
                xf[bd_index(nx - 2, MAXV, 12)] = Xp->pdf_fwd;
            }
        }
    }
    if (t_connect && ns == 0) {
        // the eye subpath reached a light by itself ("kajiya" strategy)
        tb[bd_index(nt - 1, MAXV, 13)] = VE[nt - 1].pdf_bwd;
        tf[nt - 1] = VE[nt - 1].pdf_fwd;
        if (t_prev->dirac) {
            tb[nt - 2] = c3(1.0f);
            tf[nt - 2] = c3(1.0f);
        } else {
            tb[bd_index(nt - 2, MAXV, 14)] = VE[nt - 2].pdf_bwd;
            tf[nt - 2] = VE[nt - 2].pdf_fwd;
        }
    }
    for (int i = 0; i < ns - 2; ++i) {
        if (VL[i].dirac) {
            sf[i] = sb[i] = c3(1.0f);
        } else {
            sf[i] = VL[i].pdf_fwd;
            sb[i] = VL[i].pdf_bwd;
        }
    }
    for (int i = 0; i < nt - 2; ++i) {
        if (VE[i].dirac) {
            tf[i] = tb[i] = c3(1.0f);
        } else {
            tf[i] = VE[i].pdf_fwd;
            tb[i] = VE[i].pdf_bwd;
        }
    }
    // leading specular chain seen from the camera ("locked", :1523-1540)
    int locked = -1;
    if (VE[0].dirac && VE[1].dirac) {
        int i = 0;
        for (; i < nt - 1; ++i) {
            if (VE[i].dirac || VE[i + 1].dirac) continue;
            locked = i;
            break;
        }
        if (i == nt - 1) locked = i;
    }
    float sum = 1.0f, pi = 1.0f;
    for (int i = nt - 1; i >= 0; --i) {
        pi *= avg3(tb[i] / tf[i]);
        if (locked != -1 && i <= locked) break;
        if (i < nt - 1 && VE[i].dirac) continue;
        if (i == 0 && VE[0].dirac) continue;
        sum += pi;
    }
    pi = 1.0f;
    for (int i = ns - 1; i >= 0; --i) {
        pi *= avg3(sb[i] / sf[i]);
        if (0 < i && i < ns - 1 && VL[i].dirac) continue;
        if (i == 0 && VL[0].dirac) continue;
        sum += pi;
    }
    return 1.0f / sum;
}

// VolumetricTest (:1052-1094): binary transmittance between the vertices.
RUMI_D bool volumetric_ok(const DevVolume &V, float3 sp, float3 tp, float xi) {
    if (!V.present) return true;
    const float3 dir = normalize_ref(tp - sp);
    const float tmax = sqrtf(dot3(tp - sp, tp - sp));
    float tn, tf;
    if (!volume_intersect(V, sp, dir, 0.0f, tn, tf)) return true;
    const float sm = volume_max_distance(tmax, tn, tf);
    return !(xi < 1.0f - expf(avg3(V.sigma_t) * -sm));
}

// The light a sample picked and its sampled point (Scene::LightsUniformSampling +
// AreaLight::SolidAngleSampling's position).
struct BdLight {
    int li;
    float3 n;
};

// Both subpaths of camera sample j (ConstructViewPath / ConstructLightPath with their
// starts, bidirectionalpathtracer.cpp:121-180).  Returns the light; nE / nLv receive the
// vertex counts.
template <int MAXV>
RUMI_D BdLight build_subpaths(const BdLaunch &P, int j, BVert *VE, float3 *segE, float3 *aE, BVert *VL, float3 *segL,
                              float3 *aL, int &nE, int &nLv, int *stk, TraceStats &st) {
    const DevScene &S = P.s;
    const uint64_t path = (uint64_t)(P.path0 + j);
    const long long pixel = (long long)P.pix0 + j / P.spp;
    const int sidx = j % P.spp;
    const int W = S.width, H = S.height;
    const int pw_ = (int)(pixel % W), ph_ = (int)(pixel / W);
    const Uniform4 UL = path_uniforms(path, 1000u, 0, P.k0, P.k1);
    const Uniform4 UD = path_uniforms(path, 1000u, 1, P.k0, P.k1);
    const int li = pick_light(S, UL.u[0]);
    const DevLight light = S.lights[bd_index(li, S.n_lights, 6)];
    const LightSample ls = sample_light(S, UL.u[0], UL.u[1], UL.u[2]);
    const float3 light_n = ls.nL;
    // eye subpath start (Pinhole::CastViewRay, pinhole.cpp:97-136)
    const float2 smp = pixel_sample(sidx, P.spp, P.grid_d, P.square != 0, pixel, P.k0, P.k1);
    float3 eo, ed;
    {
        // the reference's BDPT turns depth of field off when it is constructed
        // (BidirectionalPathTracer's constructor, bidirectionalpathtracer.cpp:56)
        DevCamera pin = S.camera;
        pin.focal_distance = 0.0f;
        camera_ray(pin, W, H, pw_, ph_, smp.x, smp.y, 0.0f, 0.0f, eo, ed);
    }
    {
        const DevCamera &c = S.camera;
        const float hw = W * 0.5f, hh = H * 0.5f;
        const float x = -(((float)pw_ - hw) + smp.x) / hw * c.tanfov;
        const float y = -(((float)ph_ - hh) + smp.y) / hh * c.tanfov * c.y_ratio;
        const float3 l = normalize_ref(mk3(x, y, c.plane_dist));
        bvert_clear(VE[0]);
        VE[0].p = eo;
        VE[0].n = c.dir;
        VE[0].dirac = true;
        VE[0].cos_a = l.z;
        VE[0].pdf_dir = c.plane_dist * c.plane_dist / (l.z * l.z * l.z * c.film_area);
        VE[0].pdf_fwd = c3(1.0f);
    }
    // light subpath start: cosine-weighted emission from an area light
    // (AreaLight::SolidAngleSampling), uniform in the cone from a spot
    const bool spot = light.type == LIGHT_SPOT;
    bvert_clear(VL[0]);
    VL[0].p = ls.P;
    VL[0].n = light_n;
    VL[0].pdf_fwd = c3(ls.pdf);
    float3 emit_w;
    if (spot) {
        emit_w = spot_sample_dir(light, UD.u[0], UD.u[1]);
        VL[0].pdf_dir = spot_pdf_dir(light);
        VL[0].cos_a = 1.0f;
    } else {
        const LobeSample emit = lambert_sample(light_n, UD.u[0], UD.u[1]);
        emit_w = emit.wi;
        VL[0].pdf_dir = emit.pdf;
        VL[0].cos_a = dot3(emit.wi, light_n);
    }
    // the eye subpath, then the light subpath, through one call site
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        const bool eye = side == 0;
        const int nv = construct_subpath(P, eye, eye ? P.nE : P.nL, path, eye ? 2000u : 3000u, eye ? eo : ls.P,
                                         eye ? ed : emit_w, eye ? VE : VL, eye ? segE : segL, eye ? aE : aL, light,
                                         light_n, stk, st);
        if (eye)
            nE = nv;
        else
            nLv = nv;
    }
    // a delta position: the strategies in which the eye subpath reaches the light carry
    // no weight (the MIS sums skip a dirac first light vertex)
    if (spot) VL[0].dirac = true;
    BdLight bl;
    bl.li = li;
    bl.n = light_n;
    return bl;
}

// One strategy of Trace's double loop (bidirectionalpathtracer.cpp:182-390): eye subpath
// vertex t and light subpath vertex s = len - (t + 1).  Returns
//   STRAT_NONE   nothing to add (rejected, or a skipped combination);
//   STRAT_ADD    `lo` is added to the sample as it is (the eye subpath reached a light);
//   STRAT_SHADOW `lo` counts once the shadow ray (o, dir, tmax) is unoccluded; t == 0 splats
//                it onto film pixel `px`.
// *stop: Trace leaves the t loop of this length here (t past the eye subpath, or an eye
// vertex on a light).  VisibilityTest is the caller's.
enum { STRAT_NONE = 0, STRAT_ADD = 1, STRAT_SHADOW = 2 };

struct StratOut {
    float3 lo, o, dir;
    float tmax;
    int px;
};

template <int MAXV>
RUMI_D int strategy(const BdLaunch &P, int j, int len, int t, const BVert *VE, const float3 *segE, const float3 *aE,
                    int nE, const BVert *VL, const float3 *segL, const float3 *aL, int nLv, const DevLight &light,
                    float3 light_n, bool &stop, StratOut &out) {
    const DevScene &S = P.s;
    const uint64_t path = (uint64_t)(P.path0 + j);
    const int W = S.width, H = S.height;
    const bool spot = light.type == LIGHT_SPOT;
    if (t >= nE) {
        stop = true;
        return STRAT_NONE;
    }
    const BVert &tc = VE[bd_index(t, MAXV, 21)];
    float3 t_wo = mk3(0, 0, 0);
    if (t > 0) {
        t_wo = -segE[bd_index(t - 1, MAXV, 26)];
        if (tc.onsurface && tc.mat >= 0 && S.materials[bd_index(tc.mat, S.n_materials, 8)].type == MAT_EMISSIVE) {
            stop = true;
            if (len == nE - 1) {
                const float w = mis_weight<MAXV>(P, VL, segL, VE, segE, 0, t + 1, mk3(0, 0, 0), mk3(0, 0, 0), light_n, light);
                out.lo = aE[bd_index(t + 1, MAXV + 2, 23)] * w;
                return STRAT_ADD;
            }
            return STRAT_NONE;
        }
        if (tc.dirac) return STRAT_NONE;
    }
    const int s = len - (t + 1);
    if (s >= nLv || s <= -1) return STRAT_NONE;
    const BVert &sc = VL[bd_index(s, MAXV, 22)];
    float3 s_wi = mk3(0, 0, 0);
    if (s > 0) {
        s_wi = -segL[bd_index(s - 1, MAXV, 27)];
        if (sc.onsurface && sc.mat >= 0 && S.materials[bd_index(sc.mat, S.n_materials, 9)].type == MAT_EMISSIVE) return STRAT_NONE;
        if (sc.dirac) return STRAT_NONE;
    }
    // the geometric rejections come before the two visibility tests: they read no random
    // numbers and change nothing, so the order only saves traversals
    const float3 cwi = normalize_ref(sc.p - tc.p);
    const float3 cwo = normalize_ref(tc.p - sc.p);
    const float ci = tc.onsurface ? dot3(cwi, tc.n) : 1.0f;
    if (ci < 1e-4f) return STRAT_NONE;
    float co = sc.onsurface ? dot3(cwo, sc.n) : 1.0f;
    if (s == 0 && spot) {
        if (dot3(cwo, light.direction) < light.cos_cone) return STRAT_NONE;  // outside the cone
        co = 1.0f;                                                         // no cosine at a point
    }
    if (co < 1e-4f) return STRAT_NONE;
    const float dist = sqrtf(dot3(tc.p - sc.p, tc.p - sc.p));
    if (dist <= 0.0f) return STRAT_NONE;
    const float G = ci * co / (dist * dist);
    if (G <= 0.0f) return STRAT_NONE;
    int film_w = 0, film_h = 0;
    if (t == 0) {
        if (!film_plane_pixel(P, sc.p, film_w, film_h)) return STRAT_NONE;
        if (film_w == W || film_h == H) return STRAT_NONE;
        if (film_w < 0 || film_h < 0 || film_w > W || film_h > H) return STRAT_NONE;
    }
    // VolumetricTest reads its own uniform, so it may come before the visibility test
    const Uniform4 UC = path_uniforms(path, 4000u + (uint32_t)(s * 64 + t), 0, P.k0, P.k1);
    if (!volumetric_ok(S.volume, sc.p, tc.p, UC.u[0])) return STRAT_NONE;
    // the eye end's and the light end's factors through one loop body (one copy of the
    // material code in the kernel)
    float3 cf[2];
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        const bool ee = side == 0;
        const BVert &v = ee ? tc : sc;
        const int k = ee ? t : s;
        const float3 wa = ee ? cwi : s_wi, wb = ee ? t_wo : cwo;
        float3 c;
        if (k == 0) {
            if (ee) {
                const DevCamera &cam = S.camera;
                const float cs = dot3(tc.n, cwi);
                const float We = cam.plane_dist * cam.plane_dist / (cam.film_area * cs * cs * cs * cs);
                c = c3(We / avg3(tc.pdf_fwd));
            } else {
                c = light_emission(light) / sc.pdf_fwd;
            }
        } else if (v.onsurface) {
            c = vert_fr(S, v, v.n, wa, wb) / (v.pdf_fwd * v.pdf_path);
        } else {
            c = (S.volume.sigma_s * phase_value(S.volume, wa, wb)) / (v.pdf_fwd * v.pdf_path);
        }
        // Texture::Pattern of the connecting vertex's object (bidirectionalpathtracer.cpp:
        // 350-351): a medium vertex takes the texture of the surface its segment was
        // headed for, evaluated at the medium point; none without such a surface
        if (k > 0 && S.prim_tex && v.prim >= 0) c = c * tex_pattern(S, v.prim, v.p);
        cf[side] = c;
    }
    const float3 cE = cf[0], cL = cf[1];
    const float3 lo = aE[bd_index(t, MAXV + 2, 24)] * cE * G * cL * aL[bd_index(s, MAXV + 2, 25)];
    out.lo = lo * mis_weight<MAXV>(P, VL, segL, VE, segE, s + 1, t + 1, cwi, cwo, light_n, light);
    // the shadow ray of VisibilityTest (:1018-1050): from the eye vertex unless the eye
    // vertex is the camera
    if (t == 0) {
        out.o = sc.p;
        out.dir = normalize_ref(tc.p - sc.p);
    } else {
        out.o = tc.p;
        out.dir = normalize_ref(sc.p - tc.p);
    }
    out.tmax = sqrtf(dot3(tc.p - sc.p, tc.p - sc.p));
    out.px = t == 0 ? film_h * W + film_w : -1;
    return STRAT_SHADOW;
}

// Every strategy of one sample in Trace's order, visibility traced by this thread; splats
// go to the light film.  Returns the sample's radiance.
template <int MAXV>
RUMI_D float3 connect_strategies(const BdLaunch &P, int j, const BVert *VE, const float3 *segE, const float3 *aE,
                                 int nE, const BVert *VL, const float3 *segL, const float3 *aL, int nLv,
                                 const BdLight &bl, int *stk, TraceStats &st) {
    const DevScene &S = P.s;
    const DevLight light = S.lights[bd_index(bl.li, S.n_lights, 7)];
    float3 L = mk3(0, 0, 0);
    const int max_len = nE + nLv - 1;
    for (int len = 1; len <= max_len; ++len) {
        for (int t = 0; t <= len; ++t) {
            bool stop = false;
            StratOut out;
            const int r = strategy<MAXV>(P, j, len, t, VE, segE, aE, nE, VL, segL, aL, nLv, light, bl.n, stop, out);
            if (r == STRAT_ADD) {
                L = L + out.lo;
            } else if (r == STRAT_SHADOW) {
                const HitRec h = trace_ray<true, BD_STACK, false>(S, out.o, out.dir, out.tmax, false, stk, BD_THREADS, st);
                if (!(h.t > 0.0f && out.tmax - h.t > 1e-4f)) {
                    if (out.px >= 0) {
                        float *dst = P.light_film + (size_t)bd_index(out.px, P.s.width * P.s.height, 10) * 3;
                        atomicAdd(dst + 0, out.lo.z);
                        atomicAdd(dst + 1, out.lo.y);
                        atomicAdd(dst + 2, out.lo.x);
                    } else {
                        L = L + out.lo;
                    }
                }
            }
            if (stop) break;
        }
    }
    return L;
}


// One thread renders one camera sample: both subpaths and every strategy.
template <int MAXV>
__global__ void __launch_bounds__(BD_THREADS) bdpt_kernel(BdLaunch P) {
    __shared__ int stack[BD_STACK * BD_THREADS];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= P.n_paths) return;
    TraceStats st{0, 0};
    int *stk = stack + threadIdx.x;
    BVert VE[MAXV], VL[MAXV];
    float3 segE[MAXV], segL[MAXV], aE[MAXV + 2], aL[MAXV + 2];
    int nE, nLv;
    const BdLight bl = build_subpaths<MAXV>(P, j, VE, segE, aE, VL, segL, aL, nE, nLv, stk, st);
    const float3 L = connect_strategies<MAXV>(P, j, VE, segE, aE, nE, VL, segL, aL, nLv, bl, stk, st);
    P.L[j] = make_float4(L.x, L.y, L.z, 0.0f);
}

__global__ void bdpt_write_film(BdLaunch P, int n_pix, float *film, unsigned long long *nan_count) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_pix) return;
    float3 acc = mk3(0, 0, 0);
    int nan = 0;
    for (int s = 0; s < P.spp; ++s) {
        const float4 l = P.L[(size_t)q * P.spp + s];
        if (l.x != l.x || l.y != l.y || l.z != l.z)
            ++nan;
        else {
            acc.x += l.x; acc.y += l.y; acc.z += l.z;
        }
    }
    const size_t px = (size_t)(P.pix0 + q) * 3;
    film[px + 0] = acc.z;
    film[px + 1] = acc.y;
    film[px + 2] = acc.x;
    if (nan) atomicAdd(nan_count, (unsigned long long)nan);
}

__global__ void add_light_film(float *film, const float *light, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        film[i] += light[i];
}

// The launch sequence.  A host build of this file (RUMI_HOST_BUILD: the kernel body
// compiled as plain C++ for address and undefined-behaviour checks on the CPU) leaves it out.
#ifndef RUMI_HOST_BUILD
rumi_status bdpt_render(rumi_scene *sc, const rumi_render_params *p, float *film_dev, rumi_render_stats *stats,
                        cudaStream_t stream) {
    const DevScene &S = sc->dev;
    if (sc->has_ibl) {
        set_error("BDPT does not support image-based lights");
        return RUMI_ERR_INVALID_ARG;
    }
    if (p->n_light < 2 || p->n_eye < 2 || p->n_light > BD_MAXV || p->n_eye > BD_MAXV) {
        set_error("BDPT needs 2 <= n_light, n_eye <= 16");
        return RUMI_ERR_INVALID_ARG;
    }
    if (S.n_lights <= 0) {
        set_error("BDPT needs a light");
        return RUMI_ERR_INVALID_ARG;
    }
    const int W = S.width, H = S.height, spp = p->spp;
    const long long total_pix = (long long)W * H;
    long long wave = p->wave_paths > 0 ? p->wave_paths : (1 << 20);
    long long pix_per_wave = wave / spp;
    if (pix_per_wave < 1) pix_per_wave = 1;
    if (pix_per_wave > total_pix) pix_per_wave = total_pix;
    const size_t npaths = (size_t)(pix_per_wave * spp);
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t film_bytes = sizeof(float) * 3 * (size_t)total_pix;
    const size_t bytes = al(npaths * sizeof(float4)) + al(film_bytes) + al(64);
    rumi_status st = ensure_workspace(sc, bytes);
    if (st != RUMI_OK) return st;
    char *w = (char *)sc->ws;
    BdLaunch B;
    B.s = S;
    B.nL = p->n_light;
    B.nE = p->n_eye;
    B.spp = spp;
    B.k0 = (uint32_t)p->seed;
    B.k1 = (uint32_t)(p->seed >> 32) ^ 0x5851F42Du;
    int d = 0;
    while ((d + 1) * (d + 1) <= spp) ++d;
    B.grid_d = d;
    B.square = d * d == spp;
    B.L = (float4 *)w; w += al(npaths * sizeof(float4));
    B.light_film = (float *)w; w += al(film_bytes);
    unsigned long long *nan_count = (unsigned long long *)w;
    const DevCamera &c = S.camera;
    B.right = mk3(c.m[0] + c.m[3], c.m[4] + c.m[7], c.m[8] + c.m[11]);
    B.up = mk3(c.m[1] + c.m[3], c.m[5] + c.m[7], c.m[9] + c.m[11]);
    {
        const int z[4] = {0, 0, 0, 0};
        cudaStreamSynchronize(stream);
        cudaMemcpyToSymbol(g_bd_range, z, sizeof(z));
    }
    cudaMemsetAsync(B.light_film, 0, film_bytes, stream);
    cudaMemsetAsync(nan_count, 0, sizeof(unsigned long long), stream);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const bool timing = (p->flags & RUMI_FLAG_TIMING) != 0;
    if (timing) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, stream);
    }
    long long launches = 0;
    for (long long pix0 = 0; pix0 < total_pix; pix0 += pix_per_wave) {
        const long long n_pix = pix0 + pix_per_wave <= total_pix ? pix_per_wave : total_pix - pix0;
        B.pix0 = (int)pix0;
        B.n_paths = (int)(n_pix * spp);
        B.path0 = pix0 * spp;
        const int blocks = (B.n_paths + BD_THREADS - 1) / BD_THREADS;
        if (p->n_light <= 8 && p->n_eye <= 8)
            bdpt_kernel<8><<<blocks, BD_THREADS, 0, stream>>>(B);
        else
            bdpt_kernel<BD_MAXV><<<blocks, BD_THREADS, 0, stream>>>(B);
        bdpt_write_film<<<(int)((n_pix + 255) / 256), 256, 0, stream>>>(B, (int)n_pix, film_dev, nan_count);
        launches += 2;
    }
    add_light_film<<<sc->num_sms * 4, 256, 0, stream>>>(film_dev, B.light_film, (size_t)total_pix * 3);
    if (timing) cudaEventRecord(e1, stream);
    unsigned long long h_nan = 0;
    cudaMemcpyAsync(&h_nan, nan_count, sizeof(h_nan), cudaMemcpyDeviceToHost, stream);
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_status(e, "bdpt_render");
    {
        int chk[4] = {0, 0, 0, 0};
        cudaMemcpyFromSymbol(chk, g_bd_range, sizeof(chk));
        if (chk[0]) {
            set_error("bdpt_render: index check " + std::to_string(chk[0]) + " failed: index " +
                      std::to_string(chk[1]) + " of " + std::to_string(chk[2]) + " (sample thread " +
                      std::to_string(chk[3]) + ")");
            return RUMI_ERR_INTERNAL;
        }
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->paths = total_pix * spp;
        stats->nan_samples = (int64_t)h_nan;
        stats->extend_launches = launches;
        if (timing) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            stats->total_ms = ms;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return RUMI_OK;
}
#endif  // RUMI_HOST_BUILD

}  // namespace rumi
