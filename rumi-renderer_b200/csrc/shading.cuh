// Scattering, emission and medium routines of the renderer, restated from the
// reference with explicit uniforms (the reference draws them from a global rand()).
//   OrthonormalBasis        src/Kernel/vector.h:70-95
//   Lambertian              src/Kernel/bsdf.cpp:24-69
//   Phong                   src/Kernel/bsdf.cpp:86-170
//   PerfectReflection       src/Kernel/bsdf.cpp:182-207
//   FresnelReflection       src/Kernel/bsdf.cpp:219-283
//   FresnelTransparency     src/Kernel/bsdf.cpp:306-342
//   Isotropic phase         src/Kernel/phase.cpp:34-71
//   materials               src/Material/{matte,glossy,specular,emissive,dielectric,subsurface}.cpp
//   AreaLight               src/Light/arealight.cpp:31-117
//   HomogeneousVolume       src/Volume/homogeneousvolume.cpp:46-229
// Sampling uses closed forms of the reference's angle formulas (cos(acos(1-2u)/2) =
// sqrt(1-u), cos(acos(x)) = x), equal up to float rounding.
#pragma once
#include "scene.cuh"
#include "traverse.cuh"

// ----------------------------------------------------------------- frames
RUMI_D void onb_ref(float3 v0, float3 &v1, float3 &v2) {
    if (v0.x == 0.0f && v0.z == 0.0f && (v0.y == 1.0f || v0.y == -1.0f)) {
        v1 = mk3(1.0f, 0.0f, 0.0f);
        v2 = mk3(0.0f, 0.0f, -1.0f);  // the reference's v0.y == 0 branch is unreachable here
        return;
    }
    v1 = normalize_ref(cross3(v0, mk3(0.0f, 1.0f, 0.0f)));
    if (any_nan3(v1)) v1 = mk3(1.0f, 0.0f, 0.0f);
    v2 = cross3(v0, v1);
}

// local (su, sv, sw) in frame (u, v, w): u*su + v*sv + w*sw
RUMI_D float3 frame_dir(float3 u, float3 v, float3 w, float su, float sv, float sw) {
    return u * su + v * sv + w * sw;
}

// ---------------------------------------------------------------- BSDF lobes
struct LobeSample {
    float3 wi;
    float cost;
    float pdf;
};

// Lambertian::BSDFSampling: phi = 2 pi u1, theta = acos(1 - 2 u2) / 2.
RUMI_D LobeSample lambert_sample(float3 n, float u1, float u2) {
    float3 u, w;
    onb_ref(n, u, w);
    float sphi, cphi;
    sincosf(u1 * 2.0f * RUMI_PI_F, &sphi, &cphi);
    const float sint = sqrtf(u2), cost = sqrtf(1.0f - u2);
    LobeSample s;
    s.wi = frame_dir(u, n, w, sint * sphi, cost, sint * cphi);
    s.cost = dot3(s.wi, n);
    if (s.cost <= 0.0f) s.cost = 1e-4f;
    s.pdf = RUMI_INV_PI_F * s.cost;
    if (s.pdf <= 0.0f) s.pdf = 1e-4f;
    return s;
}

RUMI_D float lambert_pdf(float3 n, float3 w_pdf) {
    float pdf = RUMI_INV_PI_F * dot3(n, w_pdf);
    return pdf <= 0.0f ? 1e-4f : pdf;
}

// Phong lobe about the mirror direction of w (Phong::BSDFSampling / F / Pdfw).
RUMI_D LobeSample phong_sample(float3 wo, float3 n, float e, float norm, float u1, float u2) {
    float won = dot3(wo, n);
    if (won <= 0.0f) won = 1e-4f;
    const float3 v = -wo + n * won * 2.0f;
    float3 u, w;
    onb_ref(v, u, w);
    float sphi, cphi;
    sincosf(u1 * 2.0f * RUMI_PI_F, &sphi, &cphi);
    const float cth = powf(u2, 1.0f / (1.0f + e));
    const float sth = sqrtf(fmaxf(0.0f, 1.0f - cth * cth));
    const float su = sth * sphi, sv = cth, sw = sth * cphi;
    LobeSample s;
    s.wi = frame_dir(u, v, w, su, sv, sw);
    float c = dot3(s.wi, n);
    if (c < 0.0f) {
        c = -c;
        s.wi = frame_dir(u, v, w, -su, sv, -sw);
    }
    const float ca = powf(dot3(s.wi, v), e);
    s.pdf = ca >= 1e-4f ? norm * ca : norm * 1e-4f;
    if (s.pdf <= 0.0f) s.pdf = 1e-4f;
    s.cost = 1.0f;
    return s;
}

RUMI_D float phong_f(float3 n, float3 wi, float3 wo, float e, float norm) {
    float c = dot3(wi, n);
    if (c <= 0.0f) c = 1e-4f;
    const float3 r = -wi + n * (c * 2.0f);
    const float ca = powf(dot3(wo, r), e);
    return ca >= 1e-4f ? norm * ca : norm * 1e-4f;
}

RUMI_D float phong_pdf(float3 n, float3 w, float3 w_pdf, float e, float norm) {
    float won = dot3(w, n);
    if (won <= 0.0f) won = 1e-4f;
    const float3 v = -w + n * (won * 2.0f);
    const float ca = powf(dot3(w_pdf, v), e);
    float pdf = ca >= 1e-4f ? norm * ca : norm * 1e-4f;
    return pdf <= 0.0f ? 1e-4f : pdf;
}

RUMI_D float3 mirror_dir(float3 wo, float3 n) {  // PerfectReflection::BSDFSampling
    float won = dot3(wo, n);
    if (won <= 0.0f) won = 1e-4f;
    return -wo + n * (2.0f * won);
}

// FresnelReflection::BSDFSampling: reflect about the side of n that wo is on.
// cost_out = Dot(wo, n) (the caller's go-into-object test reads its sign).
RUMI_D float3 fresnel_reflect_dir(float3 wo, float3 normal, float &cost_out) {
    cost_out = dot3(wo, normal);
    float3 n = normal;
    float won = cost_out;
    if (won < 1e-4f) {
        if (won > -1e-4f)
            won = 1e-4f;
        else {
            n = -n;
            won = -won;
        }
    }
    return -wo + n * (2.0f * won);
}

// FresnelReflection::Fresnel: unpolarised dielectric reflectance, 1 on total internal
// reflection.  direction is the incident ray direction (-wo).
RUMI_D float fresnel_kr(float3 direction, float3 normal, float eta_in, float eta_out) {
    float eta_i = eta_out, eta_t = eta_in;
    float ci = -dot3(direction, normal);
    if (ci < 0.0f) {
        eta_i = eta_in;
        eta_t = eta_out;
        ci = -ci;
    }
    const float inv_eta = 1.0f / (eta_t / eta_i);
    float ct = 1.0f - (1.0f - ci * ci) * (inv_eta * inv_eta);
    if (ct <= 0.0f) return 1.0f;
    ct = sqrtf(ct);
    const float rs = (eta_i * ci - eta_t * ct) / (eta_i * ci + eta_t * ct);
    const float rp = (eta_i * ct - eta_t * ci) / (eta_i * ct + eta_t * ci);
    return (rs * rs + rp * rp) * 0.5f;
}

// FresnelTransparency::BSDFSampling.  cost_out = Dot(wo, n) before flipping.
RUMI_D float3 refract_dir(float3 wo, float3 normal, float eta_in, float eta_out, float &cost_out) {
    float eta = eta_in / eta_out;
    float3 n = normal;
    float ci = dot3(wo, n);
    cost_out = ci;
    if (ci < 0.0f) {
        n = -n;
        eta = eta_out / eta_in;
        ci = -ci;
    }
    const float inv_eta = 1.0f / eta;
    const float ct = sqrtf(1.0f - (1.0f - ci * ci) * (inv_eta * inv_eta));
    return -wo * inv_eta + n * (ci * inv_eta - ct);
}

// Isotropic::IsotropicSampling about v = -wo: phi = 2 pi u1, theta = acos(2 u2 - 1).
RUMI_D float3 isotropic_dir(float3 wo, float u1, float u2) {
    const float3 v = -wo;
    float3 u, w;
    onb_ref(v, u, w);
    float sphi, cphi;
    sincosf(u1 * 2.0f * RUMI_PI_F, &sphi, &cphi);
    const float cth = u2 * 2.0f - 1.0f;
    const float sth = sqrtf(fmaxf(0.0f, 1.0f - cth * cth));
    return frame_dir(u, v, w, sth * sphi, cth, sth * cphi);
}

// Henyey-Greenstein phase (Henyey & Greenstein 1941), not in the reference.  The
// scattering angle is measured from the propagation direction d (cos = dot(d, wi)),
// g > 0 forward.  Sampled by inverting its CDF; reduces to isotropic_dir at g = 0.
RUMI_D float hg_eval(float cos_theta, float g) {
    const float denom = 1.0f + g * g - 2.0f * g * cos_theta;
    return (1.0f - g * g) / (4.0f * RUMI_PI_F * denom * sqrtf(fmaxf(denom, 1e-12f)));
}

RUMI_D float3 hg_sample(float3 d, float g, float u1, float u2, float &pdf) {
    if (fabsf(g) < 1e-3f) {
        pdf = 1.0f / (4.0f * RUMI_PI_F);
        return isotropic_dir(-d, u1, u2);
    }
    const float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * u2);
    const float cth = fminf(1.0f, fmaxf(-1.0f, (1.0f + g * g - sq * sq) / (2.0f * g)));
    const float sth = sqrtf(fmaxf(0.0f, 1.0f - cth * cth));
    float3 u, w;
    onb_ref(d, u, w);
    float sphi, cphi;
    sincosf(u1 * 2.0f * RUMI_PI_F, &sphi, &cphi);
    pdf = hg_eval(cth, g);
    return frame_dir(u, d, w, sth * sphi, cth, sth * cphi);
}

// ------------------------------------------------------------ material sample
struct BsdfSample {
    float3 w;
    bool le;        // next vertex may count emission (specular-like bounce)
    bool go_in;     // next segment travels inside the object
    float xi;       // lobe record (Intersection::_rand)
    float pdf_path; // lobe probability
    float cost;
    float pdfw;
};

// Material::BSDFSampling for every surface material.  u = (lobe, u1, u2).
RUMI_D BsdfSample material_sample(const DevMaterial &m, float3 wo, float3 n, float ulobe, float u1, float u2) {
    BsdfSample b;
    b.xi = 1.0f;
    b.pdf_path = 1.0f;
    b.cost = 1.0f;
    b.pdfw = 1.0f;
    b.le = false;
    b.go_in = false;
    b.w = mk3(0.0f, 0.0f, 0.0f);
    switch (m.type) {
    case MAT_MATTE: {
        LobeSample s = lambert_sample(n, u1, u2);
        b.w = s.wi; b.cost = s.cost; b.pdfw = s.pdf;
        break;
    }
    case MAT_GLOSSY: {
        b.xi = ulobe;
        if (m.kd != 0.0f && ulobe <= m.kd_pdf) {
            LobeSample s = lambert_sample(n, u1, u2);
            b.w = s.wi; b.cost = s.cost; b.pdfw = s.pdf;
            b.le = false;
            b.pdf_path = m.kd_pdf;
        } else {
            LobeSample s = phong_sample(wo, n, m.e, m.phong_norm, u1, u2);
            b.w = s.wi; b.cost = s.cost; b.pdfw = s.pdf;
            b.le = true;
            b.pdf_path = 1.0f - m.kd_pdf;
        }
        break;
    }
    case MAT_SPECULAR: {
        b.w = mirror_dir(wo, n);
        b.le = true;
        break;
    }
    case MAT_EMISSIVE: {
        b.w = mk3(0.0f, 0.0f, 0.0f);
        break;
    }
    case MAT_DIELECTRIC:
    case MAT_SUBSURFACE: {
        const float kr = fresnel_kr(-wo, n, m.eta_in, m.eta_out);
        const float kt = 1.0f - kr;
        float c;
        if (kr != 0.0f && ulobe <= kr) {
            b.w = fresnel_reflect_dir(wo, n, c);
            b.go_in = c < 0.0f;
            b.xi = 1.0f;
            b.pdf_path = kr;
        } else {
            b.w = refract_dir(wo, n, m.eta_in, m.eta_out, c);
            b.go_in = c > 0.0f;
            b.xi = 0.0f;
            b.pdf_path = kt;
        }
        b.le = true;
        b.cost = 1.0f;
        b.pdfw = 1.0f;
        break;
    }
    }
    return b;
}

// Material::Fr at a surface vertex.  albedo: the Matte/Glossy/Specular colour (per
// triangle when overridden).  in_object: the arriving ray was inside the object;
// t_in: its length (Beer-Lambert); vol_ratio: subsurface tau / pdf of the arriving
// inside segment.
RUMI_D float3 material_fr(const DevMaterial &m, float3 albedo, float3 n, float3 wi, float3 wo, bool in_object,
                          float xi, float pdf_path, float t_in, float3 vol_ratio) {
    switch (m.type) {
    case MAT_MATTE:
        return albedo * RUMI_INV_PI_F * m.kd;
    case MAT_GLOSSY:
        if (m.kd != 0.0f && xi <= m.kd_pdf) return albedo * RUMI_INV_PI_F * m.kd;
        {
            const float f = phong_f(n, wi, wo, m.e, m.phong_norm) * m.ks;
            return mk3(f, f, f);
        }
    case MAT_SPECULAR:
        return albedo * m.kd;
    case MAT_EMISSIVE:
        if (in_object) return mk3(0.0f, 0.0f, 0.0f);
        if (dot3(n, wo) <= 0.0f) return mk3(0.0f, 0.0f, 0.0f);
        return m.le;
    case MAT_DIELECTRIC:
    case MAT_SUBSURFACE: {
        float3 fr;
        if (xi == 1.0f) {
            fr = mk3(pdf_path, pdf_path, pdf_path);
        } else {
            const float eta = in_object ? m.eta_in / m.eta_out : m.eta_out / m.eta_in;
            const float f = 1.0f / (eta * eta) * pdf_path;
            fr = mk3(f, f, f);
        }
        if (in_object) {
            if (m.type == MAT_DIELECTRIC) {
                fr = fr * mk3(expf(-m.rgb.x * t_in), expf(-m.rgb.y * t_in), expf(-m.rgb.z * t_in));
            } else {
                fr = fr * vol_ratio;
            }
        }
        return fr;
    }
    }
    return mk3(0.0f, 0.0f, 0.0f);
}

RUMI_D bool material_opaque(const DevMaterial &m) { return m.type != MAT_DIELECTRIC && m.type != MAT_SUBSURFACE; }

// ------------------------------------------------------------------ lights
struct LightSample {
    float3 P;       // point on the light
    float3 nL;      // light normal at P (area lights)
    float3 Li;      // emitted radiance / intensity
    float pdf;      // (1 / n_lights) * (1 / area), or 1 / n_lights for a spot
    bool is_delta;  // spot light: no area pdf, no cosine at the light
    float cos_cone;
    float3 spot_dir;
    bool is_ibl;    // image-based light: wi sampled about the shading normal, G = 1
    float3 wi;
};

// ------------------------------------------------------------------ textures
// Checker::Pixel (checker.cpp:24-32), ImageTexture::Pixel (imagetexture.cpp:32-61),
// HDRTexture::Pixel (hdrtexture.cpp:46-59) at (u, v), with the reference's conversions:
// the index products are float, truncated to int.  Out-of-range indices (only a NaN
// coordinate produces them) read the first pixel.
RUMI_D float3 tex_pixel(const DevTexture &t, float u, float v) {
    if (t.type == TEX_CHECKER) {
        const int a = (int)(u * t.rep_u) % 2, b = (int)(v * t.rep_v) % 2;
        if (a == 0 && b == 0) return t.c2;
        if (a != 0 && b != 0) return t.c2;
        return t.c1;
    }
    if (t.type == TEX_IMAGE) {
        if (!t.img) return mk3(1.0f, 1.0f, 1.0f);
        const int row = (int)(__fmul_rn(__fsub_rn(1.0f, v), (float)(unsigned)(t.ih - 1)));
        const int col = (int)(__fmul_rn(u, (float)(unsigned)(t.iw - 1)));
        long long idx = (long long)(t.ih - 1 - row) * t.iw * t.bpp + (long long)col * t.bpp;
        if (idx < 0 || idx + 2 >= (long long)t.iw * t.ih * t.bpp) idx = 0;
        const float inv = 1.0f / 255.0f;
        float b = __fmul_rn((float)t.img[idx], inv), g = __fmul_rn((float)t.img[idx + 1], inv),
              r = __fmul_rn((float)t.img[idx + 2], inv);
        if (t.gamma != 1.0f) {
            b = powf(b, t.gamma);
            g = powf(g, t.gamma);
            r = powf(r, t.gamma);
        }
        return mk3(r, g, b);
    }
    const int row = (int)(__fmul_rn(__fsub_rn(1.0f, v), (float)(t.ih - 1)));
    const int col = (int)(__fmul_rn(__fsub_rn(1.0f, u), (float)(t.iw - 1)));
    long long idx = (long long)row * t.iw * 3 + (long long)col * 3;
    if (idx < 0 || idx + 2 >= (long long)t.iw * t.ih * 3) idx = 0;
    return mk3(t.hdr[idx], t.hdr[idx + 1], t.hdr[idx + 2]);
}

// Shape::TextureMapping of canonical primitive `id` at p: (0, 0) for triangles
// (shape.cpp:86-92); Rect::TextureMapping (rect.cpp:183-196); Sphere::TextureMapping
// (sphere.cpp:172-192), oriented by the rows of the sphere's _transform, with the
// reference's double-precision divisions by PI.
RUMI_D void tex_mapping(const DevScene &S, int id, float3 p, float &u, float &v) {
    u = 0.0f;
    v = 0.0f;
    if (id < S.n_tris) return;
    if (id < S.n_tris + S.n_rects) {
        const int r = id - S.n_tris;
        const float3 rp = f4xyz(S.rects[3 * r]), l = f4xyz(S.rects[3 * r + 1]), w = f4xyz(S.rects[3 * r + 2]);
        const float len = __fsqrt_rn(rn_dot(l, l)), wid = __fsqrt_rn(rn_dot(w, w));
        const float3 on = rn_sub(p, rp);
        u = __fdiv_rn(rn_dot(on, l), __fmul_rn(len, len));
        v = __fdiv_rn(rn_dot(on, w), __fmul_rn(wid, wid));
        if (u >= 1.0f) u = 1.0f;
        if (u <= 0.0f) u = 0.0f;
        if (v >= 1.0f) v = 1.0f;
        if (v <= 0.0f) v = 0.0f;
        return;
    }
    const int k = id - S.n_tris - S.n_rects;
    const float3 c = f4xyz(S.spheres[k]);
    float3 uu = mk3(1.0f, 0.0f, 0.0f), vv = mk3(0.0f, 1.0f, 0.0f), ww = mk3(0.0f, 0.0f, 1.0f);
    if (S.sphere_frame) {
        uu = f4xyz(S.sphere_frame[3 * k]);
        vv = f4xyz(S.sphere_frame[3 * k + 1]);
        ww = f4xyz(S.sphere_frame[3 * k + 2]);
    }
    const float3 pc = normalize_ref(rn_sub(p, c));
    const float theta = acosf(rn_dot(pc, vv));
    const float st = sinf(theta);
    const float3 pcxz = mk3(__fmul_rn(pc.x, st), __fmul_rn(pc.y, st), __fmul_rn(pc.z, st));
    const float phi = atan2f(rn_dot(pcxz, uu), rn_dot(pcxz, ww));
    const double two_pi = 2.0 * 3.14159265358979323846;
    u = phi >= 0.0f ? (float)__ddiv_rn((double)phi, two_pi) : (float)__ddiv_rn(__dadd_rn((double)phi, two_pi), two_pi);
    v = (float)__dsub_rn(1.0, __ddiv_rn((double)theta, 3.14159265358979323846));
}

// Texture::Pattern (texture.cpp:17-23): the texture of primitive `id` at p; 1 without one.
RUMI_D float3 tex_pattern(const DevScene &S, int id, float3 p) {
    if (!S.prim_tex) return mk3(1.0f, 1.0f, 1.0f);
    const int t = __ldg(&S.prim_tex[id]);
    if (t < 0) return mk3(1.0f, 1.0f, 1.0f);
    float u, v;
    tex_mapping(S, id, p, u, v);
    return tex_pixel(S.textures[t], u, v);
}

// ImageBasedLight::UniformSampling (imagebasedlight.cpp:38-69): a cosine-weighted direction
// about the shading normal n (first uniform: angle about n, second: elevation), the point
// where it leaves through the light's sphere (Sphere::Intersect without an Intersection:
// from inside, the far root), the sphere's texture there as radiance.  A ray that misses
// the sphere leaves the point at p (Ray::_tmin stays 0).
RUMI_D void sample_ibl(const DevScene &s, const DevLight &L, float3 p, float3 n, float u1, float u2,
                       LightSample &ls) {
    float3 uu, ww;
    onb_ref(n, uu, ww);
    const float phi = (float)__dmul_rn((double)__fmul_rn(u1, 2.0f), 3.14159265358979323846);
    const float theta = acosf(__fsqrt_rn(__fsub_rn(1.0f, u2)));
    const float st = sinf(theta);
    const float su = __fmul_rn(st, sinf(phi)), sv = cosf(theta), sw = __fmul_rn(st, cosf(phi));
    const float3 wi = mk3(__fadd_rn(__fadd_rn(__fmul_rn(uu.x, su), __fmul_rn(n.x, sv)), __fmul_rn(ww.x, sw)),
                          __fadd_rn(__fadd_rn(__fmul_rn(uu.y, su), __fmul_rn(n.y, sv)), __fmul_rn(ww.y, sw)),
                          __fadd_rn(__fadd_rn(__fmul_rn(uu.z, su), __fmul_rn(n.z, sv)), __fmul_rn(ww.z, sw)));
    const float4 c = s.spheres[L.shape_index];
    float t = 0.0f;
    if (!isect_sphere(p, wi, FLT_MAX, 0.0f, make_float4(c.x, c.y, c.z, 0.0f), make_float4(c.w, 0.0f, 0.0f, 0.0f),
                      false, true, t))
        t = 0.0f;
    ls.P = rn_madd(p, wi, t);
    ls.nL = -wi;
    ls.wi = wi;
    ls.Li = tex_pattern(s, s.n_tris + s.n_rects + L.shape_index, ls.P);
    float cost = rn_dot(wi, n);
    if (cost <= 0.0f) cost = 1e-4f;
    float pdf = (float)__dmul_rn(0.3183098865475128, (double)cost);  // INV_PI is a double literal
    if (pdf <= 0.0f) pdf = 1e-4f;
    ls.pdf = (1.0f / (float)s.n_lights) * pdf;
    ls.is_ibl = true;
    ls.is_delta = false;
}

RUMI_D int pick_light(const DevScene &s, float u) {
    int k = (int)(u * (float)s.n_lights);
    return k >= s.n_lights ? s.n_lights - 1 : k;
}

// Scene::VisibilityTest's light part: pick a light, sample a point on it
// (AreaLight::Sampling -> Shape::ShapeSampling, uniform over the shape; an image-based
// light samples a direction about the shading normal n at p instead).
// IBL = false compiles the image-based branch out, for scenes without such a light.
template <bool IBL = true>
RUMI_D LightSample sample_light(const DevScene &s, float ul, float u1, float u2, float3 p = mk3(0.0f, 0.0f, 0.0f),
                                float3 n = mk3(0.0f, 1.0f, 0.0f)) {
    LightSample ls;
    const DevLight L = s.lights[pick_light(s, ul)];
    ls.is_delta = false;
    ls.is_ibl = false;
    if (IBL && L.type == LIGHT_IBL) {
        sample_ibl(s, L, p, n, u1, u2, ls);
        return ls;
    }
    ls.pdf = (1.0f / (float)s.n_lights) * L.inv_area;
    ls.Li = L.le;
    if (L.type == LIGHT_SPOT) {
        ls.is_delta = true;
        ls.P = L.position;
        ls.nL = L.direction;
        ls.Li = L.intensity;
        ls.pdf = 1.0f / (float)s.n_lights;
        ls.cos_cone = L.cos_cone;
        ls.spot_dir = L.direction;
        return ls;
    }
    if (L.shape_type == SHAPE_RECT) {
        const float4 p = s.rects[3 * L.shape_index], l = s.rects[3 * L.shape_index + 1],
                     w = s.rects[3 * L.shape_index + 2];
        ls.P = f4xyz(p) + f4xyz(l) * u1 + f4xyz(w) * u2;
        ls.nL = normalize_ref(cross3(f4xyz(l), f4xyz(w)));
    } else if (L.shape_type == SHAPE_SPHERE) {
        const float4 c = s.spheres[L.shape_index];
        const float z = 1.0f - 2.0f * u2;
        const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
        float sp, cp;
        sincosf(2.0f * RUMI_PI_F * u1, &sp, &cp);
        const float3 dir = mk3(r * sp, z, r * cp);
        ls.P = f4xyz(c) + dir * c.w;
        ls.nL = normalize_ref(ls.P - f4xyz(c));
    } else {
        // emissive triangles are not light sources in this path
        ls.P = mk3(0.0f, 0.0f, 0.0f);
        ls.nL = mk3(0.0f, 1.0f, 0.0f);
    }
    return ls;
}

// ----------------------------------------------------------------- medium
// BBox::Intersect (src/Kernel/bbox.cpp:30-92) as the reference evaluates it.
RUMI_D bool bbox_intersect_ref(float3 pmin, float3 pmax, float3 o, float3 d, float &tnear, float &tfar) {
    const float ix = 1.0f / d.x, iy = 1.0f / d.y, iz = 1.0f / d.z;
    float t0 = (pmin.x - o.x) * ix, t1 = (pmax.x - o.x) * ix, tmp;
    if (t0 > t1) { tmp = t0; t0 = t1; t1 = tmp; }
    tnear = t0;
    tfar = t1;
    t0 = (pmin.y - o.y) * iy;
    t1 = (pmax.y - o.y) * iy;
    if (t0 > t1) { tmp = t0; t0 = t1; t1 = tmp; }
    if (tnear > t1 || t0 > tfar) return false;
    if (tnear < t0) tnear = t0;
    if (tfar > t1) tfar = t1;
    t0 = (pmin.z - o.z) * iz;
    t1 = (pmax.z - o.z) * iz;
    if (t0 > t1) { tmp = t0; t0 = t1; t1 = tmp; }
    if (tnear > t1 || t0 > tfar) return false;
    if (tnear < t0) tnear = t0;
    if (tfar > t1) tfar = t1;
    return true;
}

// HomogeneousVolume::Intersect: box hit, not blocked by a nearer surface (ray_tmin =
// the closest surface hit, 0 = none), not behind.
RUMI_D bool volume_intersect(const DevVolume &v, float3 o, float3 d, float ray_tmin, float &tnear, float &tfar) {
    tnear = 0.0f;
    tfar = 0.0f;
    if (!bbox_intersect_ref(v.bmin, v.bmax, o, d, tnear, tfar)) return false;
    if (tnear != tnear || tfar != tfar) return false;
    if (0.0f < ray_tmin && ray_tmin < tnear) return false;
    if (tfar < 0.0f) return false;
    return true;
}

RUMI_D float volume_max_distance(float thit, float tnear, float tfar) {
    if (tnear < 0.0f) {
        if (thit == 0.0f) return tfar;
        return thit < tfar ? thit : tfar;
    }
    if (thit == 0.0f) return tfar - tnear;
    return thit < tfar ? thit - tnear : tfar - tnear;
}

struct DistSample {
    int outcome;    // 0 pass through, 1 scatter at s, 2 absorbed
    float s;
    float3 tau, pdf;
};

// HomogeneousVolume::DistanceSampling / Subsurface::DistanceSampling: free flight with
// the mean extinction, then analog absorption with probability `absorb`.
RUMI_D DistSample distance_sample(float3 sigma_t, float avg_sigma_t, float absorb, float smax, float xi,
                                  float xi_absorb) {
    DistSample r;
    r.s = 0.0f;
    r.outcome = 0;
    const float3 e_max = mk3(expf(sigma_t.x * -smax), expf(sigma_t.y * -smax), expf(sigma_t.z * -smax));
    if (xi >= 1.0f - expf(avg_sigma_t * -smax)) {
        r.tau = e_max;
        if (r.tau.x == 0.0f && r.tau.y == 0.0f && r.tau.z == 0.0f) r.tau = mk3(1e-4f, 1e-4f, 1e-4f);
        r.pdf = r.tau;
        return r;
    }
    const float ds = -logf(1.0f - xi) / avg_sigma_t;
    if (smax - ds < 1e-4f) {
        r.tau = e_max;
        if (r.tau.x == 0.0f && r.tau.y == 0.0f && r.tau.z == 0.0f) r.tau = mk3(1e-4f, 1e-4f, 1e-4f);
        r.pdf = r.tau;
        return r;
    }
    if (xi_absorb < absorb || ds < 1e-4f) {
        r.outcome = 2;
        r.s = -1.0f;
        r.tau = mk3(1.0f, 1.0f, 1.0f);
        r.pdf = mk3(1.0f, 1.0f, 1.0f);
        return r;
    }
    r.outcome = 1;
    r.s = ds;
    r.tau = mk3(expf(sigma_t.x * -ds), expf(sigma_t.y * -ds), expf(sigma_t.z * -ds));
    r.pdf = r.tau * sigma_t;
    if (r.pdf.x == 0.0f && r.pdf.y == 0.0f && r.pdf.z == 0.0f) r.pdf = mk3(1e-4f, 1e-4f, 1e-4f);
    return r;
}

// HomogeneousVolume::ShadowRayTr: binary transmittance of an unblocked shadow ray of
// length tmax.  Returns 0 (scattered away) or 1.
// smax_out (optional): the length of the ray inside the medium (0 when it misses it).
RUMI_D float volume_shadow_tr(const DevVolume &v, float3 o, float3 d, float tmax, float xi,
                              float *smax_out = nullptr) {
    float tn, tf;
    if (!volume_intersect(v, o, d, 0.0f, tn, tf)) return 1.0f;
    const float smax = volume_max_distance(tmax, tn, tf);
    if (smax_out) *smax_out = smax;
    if (xi < 1.0f - expf(v.avg_sigma_t * -smax)) return 0.0f;
    return 1.0f;
}

// Material::Pdfw (Matte: Lambertian::Pdfw; Glossy: the lobe recorded in xi; Dirac,
// emissive and subsurface materials: 1), src/Material/{matte,glossy,specular,dielectric,
// material}.cpp.
RUMI_D float material_pdfw(const DevMaterial &m, float xi, float3 n, float3 w, float3 w_pdf) {
    if (m.type == MAT_MATTE) return lambert_pdf(n, w_pdf);
    if (m.type == MAT_GLOSSY) {
        if (m.kd != 0.0f && xi <= m.kd_pdf) return lambert_pdf(n, w_pdf);
        return phong_pdf(n, w, w_pdf, m.e, m.phong_norm);
    }
    return 1.0f;
}

// Material::IsDirac: Specular and Dielectric always (specular.cpp:30-33,
// dielectric.cpp:33-36), Glossy on its Phong lobe (glossy.cpp:35-41).  Subsurface derives
// from Material and keeps its default (material.cpp:33-36): not dirac, so BDPT connects
// through its vertices with its constant Fresnel Fr and the default Pdfw of 1.
RUMI_D bool material_dirac(const DevMaterial &m, float xi) {
    if (m.type == MAT_SPECULAR || m.type == MAT_DIELECTRIC) return true;
    if (m.type == MAT_GLOSSY) return !(m.kd != 0.0f && xi <= m.kd_pdf);
    return false;
}

// Phase value / pdf for directions a and b pointing away from the scattering point
// toward its two neighbours (the scattering cosine is -dot(a, b)).  g = 0: the
// reference's Isotropic (1 / 4 pi).
RUMI_D float phase_value(const DevVolume &v, float3 a, float3 b) {
    return v.g == 0.0f ? 1.0f / (4.0f * RUMI_PI_F) : hg_eval(-dot3(a, b), v.g);
}

// Surface normal at a hit as the shapes' Intersect routines record it
// (triangle.cpp:109-115 with the Q3 barycentric order, rect.cpp:113-119,
// sphere.cpp:111-128).  o: ray origin, p: hit point.
RUMI_D float3 surface_normal(const DevScene &S, int id, bool back, float u, float v, float3 o, float3 p,
                             const DevMaterial &m) {
    if (id < S.n_tris) {
        const float4 n0 = __ldg(&S.tri_shade[3 * id]), n1 = __ldg(&S.tri_shade[3 * id + 1]),
                     n2 = __ldg(&S.tri_shade[3 * id + 2]);
        float3 nrm = bary_ref(f4xyz(n0), f4xyz(n1), f4xyz(n2), u, v);
        if (back && material_opaque(m)) nrm = -nrm;
        return nrm;
    }
    if (id < S.n_tris + S.n_rects) {
        const int r = id - S.n_tris;
        return normalize_ref(cross3(f4xyz(S.rects[3 * r + 1]), f4xyz(S.rects[3 * r + 2])));
    }
    const float4 c = S.spheres[id - S.n_tris - S.n_rects];
    const float3 cc = f4xyz(c);
    if (m.type == MAT_EMISSIVE) {
        const float3 oc = o - cc;
        return sqrtf(dot3(oc, oc)) > c.w ? normalize_ref(p - cc) : normalize_ref(cc - p);
    }
    return normalize_ref(p - cc);
}
