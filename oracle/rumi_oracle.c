/* CPU restatement of Rumi-Renderer's rendering path -- TEST INFRASTRUCTURE ONLY.
 *
 * Used by tests/ (as the checker of the GPU kernels) and by nothing in the product.
 * Plain C99, float arithmetic, compiled with -ffp-contract=off so every operation
 * rounds as the reference's x86 build does.  Each routine cites the reference code it
 * restates.  It is pinned to the reference itself (oracle/_ref, built from the
 * reference's sources by oracle/build_ref.py) by tests/test_oracle_golden.py and
 * tests/test_textures.py, and to the golden vectors under tests/golden/.
 *
 * Randomness: the reference draws from a global rand().  The oracle instead consumes
 * the same counter-based Philox4x32-10 stream layout the GPU renderer uses -- counter
 * (path, bounce, group), key from the seed -- so a GPU frame and an oracle frame of the
 * same seed compare pixel by pixel.  What is sampled from those uniforms, and how, is the
 * reference's.
 *
 * Scene input: orc_scene_desc has the same field layout as rumi_scene_desc of
 * include/rumi_b200.h so one flattened description drives both; the oracle keeps its own
 * copy of the layout and links nothing of the product.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EPS 1e-4f
#define PI_D 3.14159265358979323846
#define INV_PI_F 0.3183098865475128f

typedef struct { float x, y, z; } V3;

static V3 v3(float x, float y, float z) { V3 r = {x, y, z}; return r; }
static V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
static V3 mul(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static V3 vmul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static V3 vdiv(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
/* Dot / Cross / Length / Normalize: src/Kernel/vector.h:33-68 */
static float dot(V3 u, V3 v) { return u.x * v.x + u.y * v.y + u.z * v.z; }
static V3 cross(V3 u, V3 v) { return v3(u.y * v.z - v.y * u.z, u.z * v.x - v.z * u.x, u.x * v.y - v.x * u.y); }
static float length(V3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
static V3 normalize(V3 v) {
    float inv = 1.0f / sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return v3(v.x * inv, v.y * inv, v.z * inv);
}
static int isnan3(V3 a) { return a.x != a.x || a.y != a.y || a.z != a.z; }
/* Average(Color) = (b + g + r) * 0.33333333333f; V3 colours hold (r, g, b). */
static float average(V3 c) { return (c.z + c.y + c.x) * 0.33333333333f; }

/* ------------------------------------------------------------------ Philox4x32-10
 * Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11):
 * round (c0..c3) -> (hi(M1*c2) ^ c1 ^ k0, lo(M1*c2), hi(M0*c0) ^ c3 ^ k1, lo(M0*c0)),
 * key += (0x9E3779B9, 0xBB67AE85) between rounds, 10 rounds. */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1, n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static float u24(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

static void path_u(uint64_t path, uint32_t bounce, uint32_t group, const uint32_t key[2], float u[4]) {
    uint32_t c[4] = {(uint32_t)path, (uint32_t)(path >> 32), bounce, group}, o[4];
    orc_philox(c, key, o);
    for (int i = 0; i < 4; ++i) u[i] = u24(o[i]);
}

/* ------------------------------------------------------------------ scene layout */
typedef struct {
    int32_t type;
    float kd, ks, exponent;
    float rgb[3];
    float eta_in, eta_out;
    float rgb2[3];
    float density;
} orc_material;

typedef struct {
    int32_t type, shape_type, shape_index;
    float position[3], direction[3], cone_deg, intensity[3];
} orc_light;

typedef struct {
    int32_t present;
    float pmin[3], pmax[3], sigma_s[3], sigma_a[3], g;
} orc_volume;

typedef struct {
    float position[3];
    float basis[16];
    float y_ratio, fov_deg;
    float focal_distance, lens_radius;
} orc_camera;

typedef struct {
    int32_t type;
    float repeat_u, repeat_v, color1[3], color2[3], gamma;
    int32_t img_width, img_height, bytes_per_pixel;
    const void *pixels;
} orc_texture;

typedef struct {
    int32_t width, height;
    int32_t n_triangles;
    const float *tri_vertices, *tri_normals;
    const int32_t *tri_material;
    const float *tri_albedo;
    int32_t n_rects;
    const float *rects;
    const int32_t *rect_material;
    int32_t n_spheres;
    const float *spheres;
    const int32_t *sphere_material;
    int32_t n_materials;
    const orc_material *materials;
    int32_t n_lights;
    const orc_light *lights;
    orc_volume volume;
    orc_camera camera;
    int32_t n_textures;
    const orc_texture *textures;
    const int32_t *tri_texture, *rect_texture, *sphere_texture;
    const float *sphere_frame;
} orc_scene_desc;

enum { MATTE = 0, GLOSSY = 1, SPECULAR = 2, EMISSIVE = 3, DIELECTRIC = 4, SUBSURFACE = 5 };

static V3 fv(const float *p) { return v3(p[0], p[1], p[2]); }

static const orc_material *prim_mat(const orc_scene_desc *s, int id) {
    if (id < s->n_triangles) return &s->materials[s->tri_material[id]];
    id -= s->n_triangles;
    if (id < s->n_rects) return &s->materials[s->rect_material[id]];
    return &s->materials[s->sphere_material[id - s->n_rects]];
}
static V3 mat_le(const orc_material *m) { return v3(m->rgb[0] * m->kd, m->rgb[1] * m->kd, m->rgb[2] * m->kd); }
static int is_emitting(const orc_material *m) {
    V3 le = mat_le(m);
    return m->type == EMISSIVE && (le.x != 0.0f || le.y != 0.0f || le.z != 0.0f);
}

/* ------------------------------------------------------------------ intersection
 * Ray state as the reference keeps it: tbest plays Ray::_tmin (0 = nothing yet). */
typedef struct { V3 o, d; float tmax; int in_object; } Ray;

/* Triangle::Intersect, src/Shape/triangle.cpp:41-118 */
static int tri_isect(const Ray *r, V3 v0, V3 v1, V3 v2, float tbest, float *t_out, float *u_out, float *v_out,
                     int *back) {
    V3 e1 = sub(v1, v0), e2 = sub(v2, v0);
    V3 P = cross(r->d, e2);
    float det = dot(P, e1);
    if (-1e-8f < det && det < 1e-8f) return 0;
    float inv = 1.0f / det;
    V3 T = sub(r->o, v0);
    float u = dot(P, T) * inv;
    if (u < 0.0f || u > 1.0f) return 0;
    V3 Q = cross(T, e1);
    float v = dot(Q, r->d) * inv;
    if (v < 0.0f || u + v > 1.0f) return 0;
    float t = dot(Q, e2) * inv;
    if (t < EPS) return 0;
    if (tbest > EPS && t > tbest) return 0;
    if (r->tmax - t < EPS) return 0;
    *t_out = t; *u_out = u; *v_out = v; *back = det < 0.0f;
    return 1;
}

/* Rect constructor + Rect::Intersect, src/Shape/rect.cpp:12-20, 51-122 */
static int rect_isect(const Ray *r, V3 p, V3 l, V3 w, int emitting, float tbest, float *t_out) {
    V3 n = normalize(cross(l, w));
    float len = length(l), wid = length(w);
    float inv_area = 1.0f / (len * wid);
    float c = dot(r->d, n);
    if (c == 0.0f) return 0;
    float t = -dot(sub(r->o, p), n) / c;
    if (t < 0.0f) return 0;
    if (t < EPS) return 0;
    if (r->tmax - t < EPS) return 0;
    if (!emitting && (0.0f < c && c < 1.0f)) return 0;
    if (t > tbest && tbest > 0.0f) return 0;
    V3 ip = add(r->o, mul(r->d, t));
    V3 on = sub(ip, p);
    float il = dot(on, l) * (inv_area * wid);
    if (il < 0.0f || il > len) return 0;
    float iw = dot(on, w) * (inv_area * len);
    if (iw < 0.0f || iw > wid) return 0;
    *t_out = t;
    return 1;
}

/* Sphere::Intersect + SolveQuadratic, src/Shape/sphere.cpp:51-132, src/Kernel/clibrary.h:62-87;
 * ibl: an emissive, textured sphere, whose roots swap (again) for a ray starting inside */
static int sphere_isect(const Ray *r, V3 c, float rad, int swap, int ibl, float tbest, float *t_out) {
    V3 roc = sub(r->o, c);
    float A = 1.0f, B = 2.0f * dot(r->d, roc), C = dot(roc, roc) - rad * rad;
    float disc = B * B - 4 * A * C, t0, t1;
    if (disc < 0.0f) return 0;
    float inv2a = 1.0f / (2.0f * A);
    if (disc == 0.0f) {
        t0 = t1 = -B * inv2a;
    } else {
        float sq = sqrtf(disc);
        t0 = (-B - sq) * inv2a;
        t1 = (-B + sq) * inv2a;
    }
    if (t0 < 0.0f && t1 < 0.0f) return 0;
    if (swap) { float tmp = t0; t0 = t1; t1 = tmp; }
    if (ibl && length(roc) < rad) { float tmp = t0; t0 = t1; t1 = tmp; }
    if (t0 < EPS) return 0;
    if (r->tmax - t0 < EPS) return 0;
    if (t0 > tbest && tbest > 0.0f) return 0;
    *t_out = t0;
    return 1;
}

typedef struct { float t; int id; float u, v; int back; } Hit;

/* Material::IsLe() and a texture: Sphere::Intersect's image-based-light branch */
static int sphere_ibl(const orc_scene_desc *s, int i) {
    return s->materials[s->sphere_material[i]].type == EMISSIVE && s->n_textures > 0 && s->sphere_texture &&
           s->sphere_texture[i] >= 0;
}

/* Brute-force stand-in for BVHAccel::Travel (src/Acceleration/bvh.cpp:150-213) over all
 * primitives in canonical order (triangles, rects, spheres), same acceptance rules.
 * anyhit returns at the first accepted primitive. */
static Hit closest(const orc_scene_desc *s, const Ray *r, int anyhit) {
    Hit h = {0.0f, -1, 0.0f, 0.0f, 0};
    if (r->d.x == 0.0f && r->d.y == 0.0f && r->d.z == 0.0f) return h;
    float t, u, v;
    int back;
    for (int i = 0; i < s->n_triangles; ++i) {
        const float *q = s->tri_vertices + 9 * (size_t)i;
        if (tri_isect(r, fv(q), fv(q + 3), fv(q + 6), h.t, &t, &u, &v, &back)) {
            h.t = t; h.id = i; h.u = u; h.v = v; h.back = back;
            if (anyhit) return h;
        }
    }
    for (int i = 0; i < s->n_rects; ++i) {
        const float *q = s->rects + 9 * (size_t)i;
        if (rect_isect(r, fv(q), fv(q + 3), fv(q + 6), is_emitting(&s->materials[s->rect_material[i]]), h.t, &t)) {
            h.t = t; h.id = s->n_triangles + i; h.u = h.v = 0.0f; h.back = 0;
            if (anyhit) return h;
        }
    }
    for (int i = 0; i < s->n_spheres; ++i) {
        const float *q = s->spheres + 4 * (size_t)i;
        if (sphere_isect(r, fv(q), q[3], r->in_object && !anyhit, sphere_ibl(s, i), h.t, &t)) {
            h.t = t; h.id = s->n_triangles + s->n_rects + i; h.u = h.v = 0.0f; h.back = 0;
            if (anyhit) return h;
        }
    }
    return h;
}

/* rays: n*8 (o, in_object, d, tmax) as in rumi_trace_rays */
void orc_trace(const orc_scene_desc *s, int64_t n, const float *rays, int anyhit, float *t, int32_t *prim) {
    for (int64_t i = 0; i < n; ++i) {
        const float *q = rays + 8 * i;
        Ray r = {fv(q), fv(q + 4), q[7], q[3] != 0.0f};
        Hit h = closest(s, &r, anyhit);
        t[i] = h.t;
        prim[i] = anyhit ? (h.t > 0.0f) : (h.t > 0.0f ? h.id : -1);
    }
}

/* ------------------------------------------------------------------ BSDFs */
/* OrthonormalBasis, src/Kernel/vector.h:70-95 */
static void onb(V3 v0, V3 *v1, V3 *v2) {
    if (v0.x == 0.0f && v0.z == 0.0f && (v0.y == 1.0f || v0.y == -1.0f)) {
        *v1 = v3(1, 0, 0);
        *v2 = v0.y == 0.0f ? v3(0, 0, 1) : v3(0, 0, -1);
    } else {
        *v1 = normalize(cross(v0, v3(0, 1, 0)));
        if (isnan3(*v1)) *v1 = v3(1, 0, 0);
        *v2 = cross(v0, *v1);
    }
}

/* 2 pi u as the reference forms it: (u * 2.0f) * PI in double, stored as float */
static float two_pi_u(float u) { return (float)((double)(u * 2.0f) * PI_D); }

/* Lambertian::BSDFSampling, src/Kernel/bsdf.cpp:44-69 */
static V3 lambert_sample(V3 n, float u1, float u2, float *cost, float *pdf) {
    V3 u, w;
    onb(n, &u, &w);
    float phi = two_pi_u(u1);
    float theta = acosf(1.0f - u2 * 2.0f) * 0.5f;
    float st = sinf(theta);
    V3 wi = add(add(mul(u, st * sinf(phi)), mul(n, cosf(theta))), mul(w, st * cosf(phi)));
    *cost = dot(wi, n);
    if (*cost <= 0.0f) *cost = 1e-4f;
    *pdf = INV_PI_F * *cost;
    if (*pdf <= 0.0f) *pdf = 1e-4f;
    return wi;
}

/* Phong::BSDFSampling / F / Pdfw, src/Kernel/bsdf.cpp:86-170 */
static float phong_norm(float e) { return (float)((e + 1.0f) / (2.0f * PI_D)); }
static V3 phong_sample(V3 wo, V3 n, float e, float u1, float u2, float *cost, float *pdf) {
    float won = dot(wo, n);
    if (won <= 0.0f) won = 1e-4f;
    V3 v = add(neg(wo), mul(mul(n, won), 2.0f));
    V3 u, w;
    onb(v, &u, &w);
    float phi = two_pi_u(u1);
    float theta = acosf(powf(u2, 1.0f / (1.0f + e)));
    float su = sinf(theta) * sinf(phi), sv = cosf(theta), sw = sinf(theta) * cosf(phi);
    V3 wi = add(add(mul(u, su), mul(v, sv)), mul(w, sw));
    *cost = dot(wi, n);
    if (*cost < 0.0f) {
        *cost = -*cost;
        wi = add(add(mul(u, -su), mul(v, sv)), mul(w, -sw));
    }
    float ca = powf(dot(wi, v), e);
    float nm = phong_norm(e);
    *pdf = ca >= 1e-4f ? nm * ca : nm * 1e-4f;
    if (*pdf <= 0.0f) *pdf = 1e-4f;
    *cost = 1.0f;
    return wi;
}
static float phong_f(V3 n, V3 wi, V3 wo, float e) {
    float c = dot(wi, n);
    if (c <= 0.0f) c = 1e-4f;
    V3 r = add(neg(wi), mul(n, c * 2.0f));
    float ca = powf(dot(wo, r), e);
    return ca >= 1e-4f ? phong_norm(e) * ca : phong_norm(e) * 1e-4f;
}

/* FresnelReflection::Fresnel, src/Kernel/bsdf.cpp:256-283 */
float orc_fresnel(const float *direction, const float *normal, float eta_in, float eta_out) {
    float eta_i = eta_out, eta_t = eta_in;
    float ci = -dot(fv(direction), fv(normal));
    if (ci < 0.0f) { eta_i = eta_in; eta_t = eta_out; ci = -ci; }
    float inv_eta = 1.0f / (eta_t / eta_i);
    float ct = 1.0f - (1.0f - ci * ci) * (inv_eta * inv_eta);
    if (ct <= 0.0f) return 1.0f;
    ct = sqrtf(ct);
    float rs = (eta_i * ci - eta_t * ct) / (eta_i * ci + eta_t * ct);
    float rp = (eta_i * ct - eta_t * ci) / (eta_i * ct + eta_t * ci);
    return (rs * rs + rp * rp) * 0.5f;
}

/* Isotropic::IsotropicSampling, src/Kernel/phase.cpp:43-58 */
static V3 isotropic(V3 wo, float u1, float u2) {
    V3 v = neg(wo), u, w;
    onb(v, &u, &w);
    float phi = two_pi_u(u1);
    float theta = acosf(u2 * 2.0f - 1.0f);
    float st = sinf(theta);
    return add(add(mul(u, st * sinf(phi)), mul(v, cosf(theta))), mul(w, st * cosf(phi)));
}

/* Henyey-Greenstein (not in the reference): inverse-CDF sampling about d. */
static float hg_eval(float c, float g) {
    float den = 1.0f + g * g - 2.0f * g * c;
    return (1.0f - g * g) / (4.0f * (float)PI_D * den * sqrtf(den));
}
static V3 hg_sample(V3 d, float g, float u1, float u2, float *pdf) {
    if (fabsf(g) < 1e-3f) {
        *pdf = (float)(1.0 / (4.0 * PI_D));
        return isotropic(neg(d), u1, u2);
    }
    float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * u2);
    float c = (1.0f + g * g - sq * sq) / (2.0f * g);
    if (c > 1.0f) c = 1.0f;
    if (c < -1.0f) c = -1.0f;
    float s = sqrtf(fmaxf(0.0f, 1.0f - c * c));
    V3 u, w;
    onb(d, &u, &w);
    float phi = two_pi_u(u1);
    *pdf = hg_eval(c, g);
    return add(add(mul(u, s * sinf(phi)), mul(d, c)), mul(w, s * cosf(phi)));
}

typedef struct { V3 w; int le, go_in; float xi, pdf_path, cost, pdfw; } Bsdf;

/* Material::BSDFSampling of every material (the src/Material/ sources) */
static Bsdf mat_sample(const orc_material *m, V3 wo, V3 n, float ulobe, float u1, float u2) {
    Bsdf b;
    memset(&b, 0, sizeof(b));
    b.xi = 1.0f; b.pdf_path = 1.0f; b.cost = 1.0f; b.pdfw = 1.0f;
    switch (m->type) {
    case MATTE: /* matte.cpp:38-46 */
        b.w = lambert_sample(n, u1, u2, &b.cost, &b.pdfw);
        break;
    case GLOSSY: { /* glossy.cpp:45-69 */
        float kd_pdf = m->kd / (m->kd + m->ks);
        b.xi = ulobe;
        if (m->kd != 0.0f && ulobe <= kd_pdf) {
            b.w = lambert_sample(n, u1, u2, &b.cost, &b.pdfw);
            b.pdf_path = kd_pdf;
        } else {
            b.w = phong_sample(wo, n, m->exponent, u1, u2, &b.cost, &b.pdfw);
            b.le = 1;
            b.pdf_path = 1.0f - kd_pdf;
        }
        break;
    }
    case SPECULAR: { /* specular.cpp:36-44, bsdf.cpp:198-207 */
        float won = dot(wo, n);
        if (won <= 0.0f) won = 1e-4f;
        b.w = add(neg(wo), mul(n, 2.0f * won));
        b.le = 1;
        break;
    }
    case DIELECTRIC:
    case SUBSURFACE: { /* dielectric.cpp:45-74, subsurface.cpp:99-120, bsdf.cpp:230-250, 321-342 */
        float nd[3] = {-wo.x, -wo.y, -wo.z}, nn[3] = {n.x, n.y, n.z};
        float kr = orc_fresnel(nd, nn, m->eta_in, m->eta_out), kt = 1.0f - kr;
        if (kr != 0.0f && ulobe <= kr) {
            float c = dot(wo, n), won = c;
            V3 nr = n;
            if (won < 1e-4f) {
                if (won > -1e-4f) won = 1e-4f;
                else { nr = neg(nr); won = -won; }
            }
            b.w = add(neg(wo), mul(nr, 2.0f * won));
            b.go_in = c < 0.0f;
            b.xi = 1.0f;
            b.pdf_path = kr;
        } else {
            float eta = m->eta_in / m->eta_out;
            V3 nr = n;
            float ci = dot(wo, nr), c = ci;
            if (ci < 0.0f) { nr = neg(nr); eta = m->eta_out / m->eta_in; ci = -ci; }
            float inv = 1.0f / eta;
            float ct = sqrtf(1.0f - (1.0f - ci * ci) * (inv * inv));
            b.w = add(mul(neg(wo), inv), mul(nr, ci * inv - ct));
            b.go_in = c > 0.0f;
            b.xi = 0.0f;
            b.pdf_path = kt;
        }
        b.le = 1;
        b.cost = 1.0f;
        b.pdfw = 1.0f;
        break;
    }
    default:
        break;
    }
    return b;
}

/* Material::Fr, src/Material/{matte,glossy,specular,emissive,dielectric,subsurface}.cpp */
static V3 mat_fr(const orc_material *m, V3 albedo, V3 n, V3 wi, V3 wo, int in_object, float xi, float pdf_path,
                 float t_in, V3 vol_ratio) {
    switch (m->type) {
    case MATTE:
        return mul(mul(albedo, INV_PI_F), m->kd);
    case GLOSSY: {
        float kd_pdf = m->kd / (m->kd + m->ks);
        if (m->kd != 0.0f && xi <= kd_pdf) return mul(mul(albedo, INV_PI_F), m->kd);
        float f = phong_f(n, wi, wo, m->exponent) * m->ks;
        return v3(f, f, f);
    }
    case SPECULAR:
        return mul(albedo, m->kd);
    case EMISSIVE:
        if (in_object || dot(n, wo) <= 0.0f) return v3(0, 0, 0);
        return mat_le(m);
    case DIELECTRIC:
    case SUBSURFACE: {
        V3 fr;
        if (xi == 1.0f) {
            fr = v3(pdf_path, pdf_path, pdf_path);
        } else {
            float eta = in_object ? m->eta_in / m->eta_out : m->eta_out / m->eta_in;
            float f = 1.0f / (eta * eta) * pdf_path;
            fr = v3(f, f, f);
        }
        if (in_object) {
            if (m->type == DIELECTRIC)
                fr = vmul(fr, v3(expf(-m->rgb[0] * t_in), expf(-m->rgb[1] * t_in), expf(-m->rgb[2] * t_in)));
            else
                fr = vmul(fr, vol_ratio);
        }
        return fr;
    }
    }
    return v3(0, 0, 0);
}

/* ------------------------------------------------------------------ medium
 * HomogeneousVolume, src/Volume/homogeneousvolume.cpp:46-215 */
static int bbox_isect(V3 pmin, V3 pmax, V3 o, V3 d, float *tn, float *tf) {
    float ix = 1.0f / d.x, iy = 1.0f / d.y, iz = 1.0f / d.z, t0, t1, tmp;
    t0 = (pmin.x - o.x) * ix; t1 = (pmax.x - o.x) * ix;
    if (t0 > t1) { tmp = t0; t0 = t1; t1 = tmp; }
    *tn = t0; *tf = t1;
    t0 = (pmin.y - o.y) * iy; t1 = (pmax.y - o.y) * iy;
    if (t0 > t1) { tmp = t0; t0 = t1; t1 = tmp; }
    if (*tn > t1 || t0 > *tf) return 0;
    if (*tn < t0) *tn = t0;
    if (*tf > t1) *tf = t1;
    t0 = (pmin.z - o.z) * iz; t1 = (pmax.z - o.z) * iz;
    if (t0 > t1) { tmp = t0; t0 = t1; t1 = tmp; }
    if (*tn > t1 || t0 > *tf) return 0;
    if (*tn < t0) *tn = t0;
    if (*tf > t1) *tf = t1;
    return 1;
}
static int vol_isect(const orc_volume *v, V3 o, V3 d, float ray_tmin, float *tn, float *tf) {
    *tn = 0.0f; *tf = 0.0f;
    if (!bbox_isect(fv(v->pmin), fv(v->pmax), o, d, tn, tf)) return 0;
    if (*tn != *tn || *tf != *tf) return 0;
    if (0.0f < ray_tmin && ray_tmin < *tn) return 0;
    if (*tf < 0.0f) return 0;
    return 1;
}
static float vol_smax(float thit, float tn, float tf) {
    if (tn < 0.0f) return thit == 0.0f ? tf : (thit < tf ? thit : tf);
    return thit == 0.0f ? tf - tn : (thit < tf ? thit - tn : tf - tn);
}
/* outcome: 0 pass, 1 scatter, 2 absorbed */
static int dist_sample(V3 st, float avg_st, float absorb, float smax, float xi, float xa, float *s, V3 *tau, V3 *pdf) {
    *s = 0.0f;
    if (xi >= 1.0f - expf(avg_st * -smax)) {
        *tau = v3(expf(st.x * -smax), expf(st.y * -smax), expf(st.z * -smax));
        if (tau->x == 0.0f && tau->y == 0.0f && tau->z == 0.0f) *tau = v3(1e-4f, 1e-4f, 1e-4f);
        *pdf = *tau;
        return 0;
    }
    float ds = -logf(1.0f - xi) / avg_st;
    if (smax - ds < 1e-4f) {
        *tau = v3(expf(st.x * -smax), expf(st.y * -smax), expf(st.z * -smax));
        if (tau->x == 0.0f && tau->y == 0.0f && tau->z == 0.0f) *tau = v3(1e-4f, 1e-4f, 1e-4f);
        *pdf = *tau;
        return 0;
    }
    if (xa < absorb || ds < 1e-4f) {
        *s = -1.0f;
        *tau = v3(1, 1, 1);
        *pdf = v3(1, 1, 1);
        return 2;
    }
    *s = ds;
    *tau = v3(expf(st.x * -ds), expf(st.y * -ds), expf(st.z * -ds));
    *pdf = vmul(*tau, st);
    if (pdf->x == 0.0f && pdf->y == 0.0f && pdf->z == 0.0f) *pdf = v3(1e-4f, 1e-4f, 1e-4f);
    return 1;
}

/* ------------------------------------------------------------------ lights */
typedef struct { V3 P, nL, Li; float pdf; int delta; float cos_cone; V3 dir; int ibl; V3 wi; } LSample;

/* ------------------------------------------------------------------ textures
 * Checker::Pixel (checker.cpp:24-32), ImageTexture::Pixel (imagetexture.cpp:32-61),
 * HDRTexture::Pixel (hdrtexture.cpp:46-59). */
static V3 tex_pixel(const orc_texture *t, float u, float v) {
    if (t->type == 0) {
        if ((int)(u * t->repeat_u) % 2 == 0 && (int)(v * t->repeat_v) % 2 == 0) return fv(t->color2);
        if ((int)(u * t->repeat_u) % 2 != 0 && (int)(v * t->repeat_v) % 2 != 0) return fv(t->color2);
        return fv(t->color1);
    }
    if (t->type == 1) {
        const unsigned char *b = (const unsigned char *)t->pixels;
        unsigned H = (unsigned)t->img_height, W = (unsigned)t->img_width, bpp = (unsigned)t->bytes_per_pixel;
        if (!b) return v3(1, 1, 1);
        int row = (int)((1.0f - v) * (float)(H - 1));
        int col = (int)(u * (float)(W - 1));
        int idx = (int)((H - 1 - (unsigned)row) * W * bpp) + col * (int)bpp;
        float inv = 1.0f / 255.0f;
        float cb = (float)b[idx] * inv, cg = (float)b[idx + 1] * inv, cr = (float)b[idx + 2] * inv;
        if (t->gamma != 1.0f) {
            cb = powf(cb, t->gamma);
            cg = powf(cg, t->gamma);
            cr = powf(cr, t->gamma);
        }
        return v3(cr, cg, cb);
    }
    const float *h = (const float *)t->pixels;
    int row = (int)((1.0f - v) * (float)(t->img_height - 1));
    int col = (int)((1.0f - u) * (float)(t->img_width - 1));
    int idx = row * t->img_width * 3 + col * 3;
    return v3(h[idx], h[idx + 1], h[idx + 2]);
}

/* Shape::TextureMapping (shape.cpp:86-92: (0, 0)), Rect::TextureMapping (rect.cpp:183-196),
 * Sphere::TextureMapping (sphere.cpp:172-192) */
static void tex_mapping(const orc_scene_desc *s, int id, V3 p, float *u, float *v) {
    *u = 0.0f;
    *v = 0.0f;
    if (id < s->n_triangles) return;
    if (id < s->n_triangles + s->n_rects) {
        const float *q = s->rects + 9 * (size_t)(id - s->n_triangles);
        V3 l = fv(q + 3), w = fv(q + 6);
        float len = length(l), wid = length(w);
        V3 on = sub(p, fv(q));
        *u = dot(on, l) / (len * len);
        *v = dot(on, w) / (wid * wid);
        if (*u >= 1.0f) *u = 1.0f;
        if (*u <= 0.0f) *u = 0.0f;
        if (*v >= 1.0f) *v = 1.0f;
        if (*v <= 0.0f) *v = 0.0f;
        return;
    }
    int k = id - s->n_triangles - s->n_rects;
    const float *c = s->spheres + 4 * (size_t)k;
    V3 uu = v3(1, 0, 0), vv = v3(0, 1, 0), ww = v3(0, 0, 1);
    if (s->sphere_frame) {
        const float *f = s->sphere_frame + 9 * (size_t)k;
        uu = fv(f);
        vv = fv(f + 3);
        ww = fv(f + 6);
    }
    V3 pc = normalize(sub(p, fv(c)));
    float theta = acosf(dot(pc, vv));
    V3 pcxz = mul(pc, sinf(theta));
    float phi = atan2f(dot(pcxz, uu), dot(pcxz, ww));
    if (phi >= 0.0f)
        *u = (float)(phi / (2.0f * PI_D));
    else
        *u = (float)((phi + 2.0f * PI_D) / (2.0f * PI_D));
    *v = (float)(1.0f - theta / PI_D);
}

/* Texture::Pattern (texture.cpp:17-23) of primitive id at p; 1 without a texture */
static V3 tex_pattern(const orc_scene_desc *s, int id, V3 p) {
    int t = -1;
    if (s->n_textures <= 0) return v3(1, 1, 1);
    if (id < s->n_triangles) t = s->tri_texture ? s->tri_texture[id] : -1;
    else if (id < s->n_triangles + s->n_rects) t = s->rect_texture ? s->rect_texture[id - s->n_triangles] : -1;
    else t = s->sphere_texture ? s->sphere_texture[id - s->n_triangles - s->n_rects] : -1;
    if (t < 0) return v3(1, 1, 1);
    float u, v;
    tex_mapping(s, id, p, &u, &v);
    return tex_pixel(&s->textures[t], u, v);
}

static float rect_inv_area(const float *r) { return 1.0f / (length(fv(r + 3)) * length(fv(r + 6))); }

/* p, n: the shading point and normal, read by an image-based light
 * (ImageBasedLight::UniformSampling, imagebasedlight.cpp:38-69) */
static LSample light_sample(const orc_scene_desc *s, float ul, float u1, float u2, V3 p, V3 n) {
    LSample ls;
    memset(&ls, 0, sizeof(ls));
    int k = (int)(ul * (float)s->n_lights);
    if (k >= s->n_lights) k = s->n_lights - 1;
    const orc_light *L = &s->lights[k];
    if (L->type == 2) { /* image-based light */
        V3 uu, ww;
        onb(n, &uu, &ww);
        float phi = (float)((double)(u1 * 2.0f) * PI_D);
        float theta = acosf(sqrtf(1.0f - u2));
        float st = sinf(theta);
        float su = st * sinf(phi), sv = cosf(theta), sw = st * cosf(phi);
        V3 wi = add(add(mul(uu, su), mul(n, sv)), mul(ww, sw));
        const float *c = s->spheres + 4 * (size_t)L->shape_index;
        Ray r = {p, wi, 3.402823466e+38f, 0};
        float t = 0.0f;
        if (!sphere_isect(&r, fv(c), c[3], 0, sphere_ibl(s, L->shape_index), 0.0f, &t)) t = 0.0f;
        ls.P = add(p, mul(wi, t));
        ls.nL = neg(wi);
        ls.wi = wi;
        ls.ibl = 1;
        ls.Li = tex_pattern(s, s->n_triangles + s->n_rects + L->shape_index, ls.P);
        float cost = dot(wi, n);
        if (cost <= 0.0f) cost = 1e-4f;
        float pdf = (float)(0.3183098865475128 * cost);
        if (pdf <= 0.0f) pdf = 1e-4f;
        ls.pdf = 1.0f / (float)s->n_lights * pdf;
        return ls;
    }
    if (L->type == 1) { /* spot */
        ls.delta = 1;
        ls.P = fv(L->position);
        ls.dir = fv(L->direction);
        ls.Li = fv(L->intensity);
        ls.cos_cone = (float)cos(L->cone_deg * PI_D / 180.0);
        ls.pdf = 1.0f / (float)s->n_lights;
        return ls;
    }
    if (L->shape_type == 1) { /* Rect::ShapeSampling, rect.cpp:176-181 */
        const float *r = s->rects + 9 * (size_t)L->shape_index;
        ls.P = add(add(fv(r), mul(fv(r + 3), u1)), mul(fv(r + 6), u2));
        ls.nL = normalize(cross(fv(r + 3), fv(r + 6)));
        ls.pdf = (1.0f / (float)s->n_lights) * rect_inv_area(r);
        ls.Li = mat_le(&s->materials[s->rect_material[L->shape_index]]);
    } else { /* sphere: uniform over the surface */
        const float *c = s->spheres + 4 * (size_t)L->shape_index;
        float z = 1.0f - 2.0f * u2, rr = sqrtf(fmaxf(0.0f, 1.0f - z * z)), ph = 2.0f * (float)PI_D * u1;
        ls.P = add(fv(c), mul(v3(rr * sinf(ph), z, rr * cosf(ph)), c[3]));
        ls.nL = normalize(sub(ls.P, fv(c)));
        ls.pdf = (1.0f / (float)s->n_lights) * (float)(1.0f / (4.0f * PI_D * c[3] * c[3]));
        ls.Li = mat_le(&s->materials[s->sphere_material[L->shape_index]]);
    }
    return ls;
}

/* Scene::VisibilityTest's geometry + AreaLight::G (scene.cpp:99-123, arealight.cpp:106-112) */
static int nee_geom(const LSample *ls, V3 p, V3 *wi, float *dist, float *G) {
    if (ls->ibl) { /* Wi = the sampled direction, G = ImageBasedLight::G = 1 */
        *wi = ls->wi;
        *dist = length(sub(ls->P, p));
        *G = 1.0f;
        return dot(*wi, ls->nL) < 0.0f;
    }
    *wi = normalize(sub(ls->P, p));
    *dist = length(sub(p, ls->P));
    if (ls->delta) {
        if (dot(neg(*wi), ls->dir) < ls->cos_cone) return 0;
        *G = 1.0f / (*dist * *dist);
        return 1;
    }
    if (dot(*wi, ls->nL) >= 0.0f) return 0;
    float c = -dot(*wi, ls->nL);
    *G = (c > 0.0f ? c : 0.0f) / (*dist * *dist);
    return 1;
}

/* ------------------------------------------------------------------ pixel sampler
 * The reference's sampler (src/Sample/uniformsample.cpp:32-58, src/Sample/sampler.cpp:17-38):
 * a jittered sqrt(n)^2 grid per frame, each pixel drawing x and y coordinates without
 * replacement.  Draw order = keyed permutations (balanced Feistel + cycle walking). */
static uint32_t mix(uint32_t y) {
    y ^= y >> 16; y *= 0x7FEB352Du; y ^= y >> 15; y *= 0x846CA68Bu; y ^= y >> 16;
    return y;
}
static int perm(int i, int n, uint32_t key) {
    if (n <= 1) return 0;
    int bits = 0;
    while ((1 << bits) < n) ++bits;
    if (bits & 1) ++bits;
    if (bits < 2) bits = 2;
    int half = bits >> 1;
    uint32_t mask = (1u << half) - 1u, x = (uint32_t)i;
    for (int walk = 0; walk < 4096; ++walk) {
        uint32_t L = x >> half, R = x & mask;
        for (int r = 0; r < 4; ++r) {
            uint32_t F = mix(R ^ (key + 0x9E3779B9u * (uint32_t)(r + 1))) & mask;
            uint32_t nl = R;
            R = L ^ F;
            L = nl;
        }
        x = (L << half) | R;
        if ((int)x < n) return (int)x;
    }
    return i;
}

static void pixel_sample(int s, int spp, long long pixel, const uint32_t key[2], float *sx, float *sy) {
    int d = 0;
    while ((d + 1) * (d + 1) <= spp) ++d;
    uint32_t pk = (uint32_t)pixel * 0x9E3779B1u ^ (uint32_t)(pixel >> 32);
    int kx = perm(s, spp, mix(pk ^ key[0]) ^ 0x68E31DA4u);
    int ky = perm(s, spp, mix(pk ^ key[1]) ^ 0xB5297A4Du);
    uint32_t cx[4] = {(uint32_t)kx, 0u, 0xFFFFFFFFu, 0u}, cy[4] = {(uint32_t)ky, 0u, 0xFFFFFFFFu, 0u}, ox[4], oy[4];
    orc_philox(cx, key, ox);
    orc_philox(cy, key, oy);
    if (d * d == spp) {
        float nz = 1.0f / (float)d;
        *sx = ((float)(kx % d) + u24(ox[0])) * nz;
        *sy = ((float)(ky / d) + u24(oy[1])) * nz;
    } else {
        float nz = 1.0f / (float)spp;
        *sx = ((float)kx + u24(ox[0])) * nz;
        *sy = ((float)ky + u24(oy[1])) * nz;
    }
}

/* Pinhole::CastViewRay, src/Camera/pinhole.cpp:97-136 (constructor values :30-51); with
 * a focal distance (Pinhole::DepthOfField, :88-95) the origin is a point of the lens disk
 * drawn from the uniforms lu1 (radius) and lu2 (angle, PI a double literal) and the ray
 * aims at the pinhole ray's point on the focal plane.  _up and _right are the basis
 * applied to (0,1,0) and (1,0,0) with its translation column added, like _dir. */
static void camera_ray(const orc_camera *c, int W, int H, int w, int h, float sx, float sy, float lu1, float lu2,
                       V3 *o, V3 *d) {
    float fov = c->fov_deg > 0.0f ? c->fov_deg : 20.0f;
    float tanfov = (float)tan(PI_D / 180.f * fov * 0.5f);
    float hw = W * 0.5f, hh = H * 0.5f;
    float x = -(((float)w - hw) + sx) / hw * tanfov;
    float y = -(((float)h - hh) + sy) / hh * tanfov * c->y_ratio;
    V3 l = normalize(v3(x, y, 1.0f));
    const float *m = c->basis;
    *d = v3(m[0] * l.x + m[1] * l.y + m[2] * l.z + m[3], m[4] * l.x + m[5] * l.y + m[6] * l.z + m[7],
            m[8] * l.x + m[9] * l.y + m[10] * l.z + m[11]);
    *o = fv(c->position);
    if (c->focal_distance > 0.0f) {
        V3 p = fv(c->position);
        float t = c->focal_distance / l.z;
        V3 fp = v3(p.x + d->x * t, p.y + d->y * t, p.z + d->z * t);
        V3 up = v3(m[1] + m[3], m[5] + m[7], m[9] + m[11]);
        V3 right = v3(m[0] + m[3], m[4] + m[7], m[8] + m[11]);
        float r = sqrtf(lu1) * c->lens_radius;
        float theta = (float)((double)(lu2 * 2.0f) * PI_D);
        float sn = sinf(theta), cs = cosf(theta);
        V3 cp = v3(p.x + up.x * r * sn + right.x * r * cs, p.y + up.y * r * sn + right.y * r * cs,
                   p.z + up.z * r * sn + right.z * r * cs);
        *o = cp;
        *d = normalize(v3(fp.x - cp.x, fp.y - cp.y, fp.z - cp.z));
    }
}

/* The two lens uniforms of a camera ray: the path's Philox stream at bounce counter
 * 0x7FFFFFFF, which no vertex uses. */
static void lens_u(const orc_camera *c, uint64_t path, const uint32_t key[2], float *lu1, float *lu2) {
    float u[4] = {0, 0, 0, 0};
    if (c->focal_distance > 0.0f) path_u(path, 0x7FFFFFFFu, 0, key, u);
    *lu1 = u[0];
    *lu2 = u[1];
}

/* ------------------------------------------------------------------ path tracer
 * PathTracer::Trace(w, h, ...) (src/Integrator/pathtracer.cpp:117-354) in forward form:
 * L = sum_k beta_k direct_k, beta_{k+1} = beta_k vol_k fr_k cos_k / Average(pdf_wi_k pdf_path_k). */
/* Debug record of one path's extension rays (orc_path_rays): o, in_object, d, tmax;
 * the closest hit's t and primitive. */
/* The vertex normal a shape's Intersect writes at a hit: triangle.cpp:110-114
 * (interpolated, flipped on a back hit of an opaque material), rect.cpp:118,
 * sphere.cpp:117-128 (an emitter's normal faces the ray origin's side). */
static V3 hit_normal(const orc_scene_desc *s, const Hit *h, V3 o, V3 p) {
    const orc_material *m = prim_mat(s, h->id);
    if (h->id < s->n_triangles) {
        const float *q = s->tri_normals + 9 * (size_t)h->id;
        V3 n = add(add(mul(fv(q), 1.0f - h->u - h->v), mul(fv(q + 3), h->u)), mul(fv(q + 6), h->v));
        int opaque = m->type != DIELECTRIC && m->type != SUBSURFACE;
        return h->back && opaque ? neg(n) : n;
    }
    if (h->id < s->n_triangles + s->n_rects) {
        const float *q = s->rects + 9 * (size_t)(h->id - s->n_triangles);
        return normalize(cross(fv(q + 3), fv(q + 6)));
    }
    const float *c = s->spheres + 4 * (size_t)(h->id - s->n_triangles - s->n_rects);
    if (m->type == EMISSIVE)
        return length(sub(o, fv(c))) > c[3] ? normalize(sub(p, fv(c))) : normalize(sub(fv(c), p));
    return normalize(sub(p, fv(c)));
}

static float *g_dbg_rays, *g_dbg_t;
static int32_t *g_dbg_prim;
static int g_dbg_n;

static V3 trace_path(const orc_scene_desc *s, int max_depth, uint64_t path, const uint32_t key[2], V3 o, V3 d) {
    V3 beta = v3(1, 1, 1), L = v3(0, 0, 0);
    int le = 1, inobj = 0;
    const orc_volume *V = &s->volume;
    V3 vs_t = v3(V->sigma_s[0] + V->sigma_a[0], V->sigma_s[1] + V->sigma_a[1], V->sigma_s[2] + V->sigma_a[2]);
    float v_avg = average(vs_t);
    float v_abs = average(vdiv(fv(V->sigma_a), vs_t));
    for (int b = 0; b < max_depth; ++b) {
        int last = b + 1 >= max_depth;
        float U0[4], U1[4], U2[4];
        path_u(path, b, 0, key, U0);
        path_u(path, b, 1, key, U1);
        path_u(path, b, 2, key, U2);
        Ray ray = {o, d, 3.402823466e+38f, inobj};
        Hit h = closest(s, &ray, 0);
        int hit = h.t > 0.0f;
        if (g_dbg_rays) {
            float *q = g_dbg_rays + 8 * g_dbg_n;
            q[0] = o.x; q[1] = o.y; q[2] = o.z; q[3] = (float)inobj;
            q[4] = d.x; q[5] = d.y; q[6] = d.z; q[7] = 3.402823466e+38f;
            g_dbg_t[g_dbg_n] = h.t;
            g_dbg_prim[g_dbg_n] = hit ? h.id : -1;
            ++g_dbg_n;
        }
        int cont = 0;
        V3 nxo = o, nxd = d;
        int nle = 0, nin = 0;
        int done = 0;
        if (V->present && !inobj) {
            float tn, tf, thit = hit ? h.t : 0.0f;
            if (vol_isect(V, o, d, thit, &tn, &tf)) {
                float smax = vol_smax(thit, tn, tf), sd;
                V3 tau, pdf;
                int oc = dist_sample(vs_t, v_avg, v_abs, smax, U1[2], U1[3], &sd, &tau, &pdf);
                if (oc == 2) {
                    done = 1;
                } else if (oc == 1) {
                    V3 p = add(o, mul(d, tn < 0.0f ? sd : tn + sd));
                    V3 vol = vdiv(tau, pdf);
                    if (s->n_lights > 0) { /* HomogeneousVolume::DirectLighting */
                        /* the vertex normal is the one of the surface the ray hit beyond the
                         * scatter point (pathtracer.cpp:154-170 overwrites only _p), read by
                         * an image-based light; (0,1,0) when the ray left the scene */
                        V3 nb = hit ? hit_normal(s, &h, o, add(o, mul(d, h.t))) : v3(0.0f, 1.0f, 0.0f);
                        LSample ls = light_sample(s, U0[3], U1[0], U1[1], p, nb);
                        V3 wi;
                        float dist, G;
                        if (nee_geom(&ls, p, &wi, &dist, &G)) {
                            float tr = 1.0f, stn, stf;
                            if (vol_isect(V, p, wi, 0.0f, &stn, &stf)) {
                                float sm = vol_smax(dist, stn, stf);
                                if (U2[2] < 1.0f - expf(v_avg * -sm)) tr = 0.0f;
                            }
                            Ray sr = {p, wi, dist, 0};
                            if (tr > 0.0f && closest(s, &sr, 1).t == 0.0f) {
                                float fp = V->g == 0.0f ? (float)(1.0 / (4.0 * PI_D)) : hg_eval(dot(d, wi), V->g);
                                /* Li * tau * sigma_s * fp * g / lights_sampling_pdf */
                                V3 direct = mul(mul(mul(vmul(mul(ls.Li, tr), fv(V->sigma_s)), fp), G), 1.0f / ls.pdf);
                                L = add(L, vmul(vmul(beta, vol), direct));
                            }
                        }
                    }
                    float pdfp;
                    V3 w = V->g == 0.0f ? isotropic(d, U0[1], U0[2]) : hg_sample(d, V->g, U0[1], U0[2], &pdfp);
                    V3 fpp;
                    if (V->g == 0.0f) {
                        float fp = (float)(1.0 / (4.0 * PI_D));
                        fpp = mul(mul(fv(V->sigma_s), fp), 1.0f / average(v3(fp, fp, fp)));
                    } else {
                        fpp = fv(V->sigma_s);
                    }
                    beta = vmul(vmul(beta, vol), fpp);
                    nxo = p; nxd = w; nle = 0; nin = 0;
                    cont = 1;
                    done = 1;
                }
            }
        }
        if (!done && hit) {
            const orc_material *m = prim_mat(s, h.id);
            V3 p = add(o, mul(d, h.t)), n = hit_normal(s, &h, o, p), albedo = fv(m->rgb);
            if (h.id < s->n_triangles && s->tri_albedo) albedo = fv(s->tri_albedo + 3 * (size_t)h.id);
            if (m->type == EMISSIVE) {
                if (le && !inobj && -dot(d, n) > 0.0f) L = add(L, vmul(vmul(beta, mat_le(m)), tex_pattern(s, h.id, p)));
            } else {
                V3 wo = neg(d), vol_ratio = v3(1, 1, 1), volw = v3(1, 1, 1);
                Bsdf bs;
                int walk = 0, absorbed = 0;
                if (m->type == SUBSURFACE && inobj) { /* Subsurface::PhaseSampling */
                    V3 sst = v3(m->rgb[0] + m->rgb2[0], m->rgb[1] + m->rgb2[1], m->rgb[2] + m->rgb2[2]);
                    float dens = m->density > 0.0f ? m->density : 1.0f;
                    float savg = (sst.z + sst.y + sst.x) / 3.0f * dens;
                    float sabs = ((m->rgb2[2] / sst.z) + (m->rgb2[1] / sst.y) + (m->rgb2[0] / sst.x)) / 3.0f;
                    float sd;
                    V3 tau, pdf;
                    int oc = dist_sample(sst, savg, sabs, h.t, U2[0], U2[1], &sd, &tau, &pdf);
                    if (oc == 1) {
                        walk = 1;
                        p = add(o, mul(d, sd));
                        memset(&bs, 0, sizeof(bs));
                        bs.w = isotropic(neg(wo), U0[1], U0[2]);
                        bs.le = 1; bs.go_in = 1; bs.xi = 1.0f; bs.pdf_path = 1.0f; bs.cost = 1.0f;
                        bs.pdfw = (float)(1.0 / (4.0 * PI_D));
                        volw = vmul(vdiv(tau, pdf), mul(fv(m->rgb), (float)(1.0 / (4.0 * PI_D))));
                    } else if (oc == 2) {
                        absorbed = 1;
                    } else {
                        vol_ratio = vdiv(tau, pdf);
                        bs = mat_sample(m, wo, n, U0[0], U0[1], U0[2]);
                    }
                } else {
                    bs = mat_sample(m, wo, n, U0[0], U0[1], U0[2]);
                }
                /* Texture::Pattern scales what this vertex returns (pathtracer.cpp:343-344) */
                beta = vmul(beta, tex_pattern(s, h.id, p));
                if (!absorbed) {
                    float kd_pdf = m->type == GLOSSY ? m->kd / (m->kd + m->ks) : 1.0f;
                    int nee = s->n_lights > 0 && !walk &&
                              (m->type == MATTE || (m->type == GLOSSY && m->kd != 0.0f && bs.xi <= kd_pdf));
                    if (nee) { /* Matte::DirectLighting, matte.cpp:54-82 */
                        LSample ls = light_sample(s, U0[3], U1[0], U1[1], p, n);
                        V3 wi;
                        float dist, G;
                        if (nee_geom(&ls, p, &wi, &dist, &G)) {
                            V3 f = mul(mul(albedo, INV_PI_F), m->kd);
                            float c = dot(wi, n);
                            if (c < 0.0f) c = 0.0f;
                            V3 direct = mul(mul(mul(vmul(f, ls.Li), c), G), 1.0f / ls.pdf);
                            if (m->type == GLOSSY) direct = mul(direct, 1.0f / kd_pdf);
                            float tr = 1.0f, stn, stf;
                            if (V->present && vol_isect(V, p, wi, 0.0f, &stn, &stf)) {
                                float sm = vol_smax(dist, stn, stf);
                                if (U2[2] < 1.0f - expf(v_avg * -sm)) tr = 0.0f;
                            }
                            Ray sr = {p, wi, dist, 0};
                            if (tr > 0.0f && closest(s, &sr, 1).t == 0.0f) L = add(L, vmul(beta, direct));
                        }
                    }
                    V3 fr = walk ? v3(1, 1, 1)
                                 : mat_fr(m, albedo, n, bs.w, wo, inobj, bs.xi, bs.pdf_path, h.t, vol_ratio);
                    float pp = bs.pdfw * bs.pdf_path;
                    float pdf = average(v3(pp, pp, pp));
                    beta = mul(mul(vmul(vmul(beta, volw), fr), bs.cost), 1.0f / pdf);
                    nxo = p; nxd = bs.w; nle = bs.le; nin = bs.go_in;
                    cont = 1;
                }
            }
        }
        if (!cont || last) break;
        o = nxo; d = nxd; le = nle; inobj = nin;
    }
    return L;
}

/* ------------------------------------------------------------------ ray tracer
 * RayTracer::Trace(ray, depth, le, in_object) (src/Integrator/raytracer.cpp:37-72) in the
 * reference's recursive form: Specular::GlobalIllumination (specular.cpp:60-75) and
 * Dielectric::GlobalIllumination (dielectric.cpp:105-159) recurse, every other material
 * returns its DirectLighting (Matte next-event estimation matte.cpp:54-82; Glossy only
 * when Intersection::_rand = 1.0 lies on its diffuse lobe, glossy.cpp:92-102; Emissive
 * emissive.cpp:61-74; Subsurface none).  *t_hit: the traced ray's Ray::_tmin (0 when
 * nothing was traced or hit), which Dielectric's Beer-Lambert factor reads. */
static V3 whitted(const orc_scene_desc *s, int max_depth, uint64_t path, const uint32_t key[2], V3 o, V3 d, int depth,
                  int le, int inobj, float *t_hit) {
    *t_hit = 0.0f;
    if (depth > max_depth) return v3(0, 0, 0);
    Ray ray = {o, d, 3.402823466e+38f, inobj};
    Hit h = closest(s, &ray, 0);
    if (!(h.t > 0.0f)) return v3(0, 0, 0);
    *t_hit = h.t;
    const orc_material *m = prim_mat(s, h.id);
    V3 p = add(o, mul(d, h.t)), n = hit_normal(s, &h, o, p), albedo = fv(m->rgb);
    if (h.id < s->n_triangles && s->tri_albedo) albedo = fv(s->tri_albedo + 3 * (size_t)h.id);
    float U0[4], U1[4], U2[4];
    path_u(path, depth, 0, key, U0);
    V3 wo = neg(d);
    V3 pat = tex_pattern(s, h.id, p); /* lo *= Texture::Pattern (raytracer.cpp:69-70) */
    if (m->type == SPECULAR) {
        Bsdf b = mat_sample(m, wo, n, U0[0], U0[1], U0[2]);
        float tt;
        V3 Li = whitted(s, max_depth, path, key, p, b.w, depth + 1, 1, 0, &tt);
        V3 f = mul(albedo, m->kd);
        return vmul(mul(mul(vmul(f, Li), b.cost), 1.0f / b.pdfw), pat);
    }
    if (m->type == DIELECTRIC) {
        Bsdf b = mat_sample(m, wo, n, U0[0], U0[1], U0[2]);
        float tt, inv;
        V3 Li = whitted(s, max_depth, path, key, p, b.w, depth + 1, 1, b.go_in, &tt), lo;
        if (b.xi == 1.0f) {
            lo = mul(mul(Li, b.pdf_path), 1.0f / b.pdfw);
            inv = 1.0f / b.pdf_path;
        } else {
            float eta = inobj ? m->eta_in / m->eta_out : m->eta_out / m->eta_in;
            lo = mul(mul(Li, 1.0f / (eta * eta) * b.pdf_path), 1.0f / b.pdfw);
            inv = 1.0f / b.pdf_path;
        }
        if (b.go_in) lo = vmul(lo, v3(expf(-m->rgb[0] * tt), expf(-m->rgb[1] * tt), expf(-m->rgb[2] * tt)));
        return vmul(mul(lo, inv), pat);
    }
    if (m->type == EMISSIVE) {
        if (inobj || !le || -dot(d, n) <= 0.0f) return v3(0, 0, 0);
        return vmul(mat_le(m), pat);
    }
    float kd_pdf = m->type == GLOSSY ? m->kd / (m->kd + m->ks) : 1.0f;
    if (s->n_lights > 0 && (m->type == MATTE || (m->type == GLOSSY && m->kd != 0.0f && 1.0f <= kd_pdf))) {
        path_u(path, depth, 1, key, U1);
        path_u(path, depth, 2, key, U2);
        LSample ls = light_sample(s, U0[3], U1[0], U1[1], p, n);
        V3 wi;
        float dist, G;
        if (!nee_geom(&ls, p, &wi, &dist, &G)) return v3(0, 0, 0);
        V3 f = mul(mul(albedo, INV_PI_F), m->kd);
        float c = dot(wi, n);
        if (c < 0.0f) c = 0.0f;
        V3 direct = mul(mul(mul(vmul(f, ls.Li), c), G), 1.0f / ls.pdf);
        if (m->type == GLOSSY) direct = mul(direct, 1.0f / kd_pdf);
        const orc_volume *V = &s->volume;
        float tr = 1.0f, stn, stf;
        if (V->present && vol_isect(V, p, wi, 0.0f, &stn, &stf)) {
            V3 vs_t = v3(V->sigma_s[0] + V->sigma_a[0], V->sigma_s[1] + V->sigma_a[1], V->sigma_s[2] + V->sigma_a[2]);
            float sm = vol_smax(dist, stn, stf);
            if (U2[2] < 1.0f - expf(average(vs_t) * -sm)) tr = 0.0f;
        }
        Ray sr = {p, wi, dist, 0};
        if (tr > 0.0f && closest(s, &sr, 1).t == 0.0f) return vmul(direct, pat);
    }
    return v3(0, 0, 0);
}

/* RayTracer::Trace(w, h, camera, film) over rows [row0, row1), film as orc_render_pt. */
long long orc_render_whitted(const orc_scene_desc *s, int max_depth, int spp, uint64_t seed, int row0, int row1,
                             float *film) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x5851F42Du};
    long long nan = 0;
    int W = s->width, H = s->height;
    for (int h = row0; h < row1 && h < H; ++h) {
        for (int w = 0; w < W; ++w) {
            long long pixel = (long long)h * W + w;
            V3 acc = v3(0, 0, 0);
            for (int k = 0; k < spp; ++k) {
                float sx, sy, lu1, lu2, tt;
                V3 o, d;
                uint64_t path = (uint64_t)(pixel * spp + k);
                pixel_sample(k, spp, pixel, key, &sx, &sy);
                lens_u(&s->camera, path, key, &lu1, &lu2);
                camera_ray(&s->camera, W, H, w, h, sx, sy, lu1, lu2, &o, &d);
                V3 L = whitted(s, max_depth, path, key, o, d, 0, 1, 0, &tt);
                if (isnan3(L))
                    ++nan;
                else
                    acc = add(acc, L);
            }
            film[pixel * 3 + 0] = acc.z;
            film[pixel * 3 + 1] = acc.y;
            film[pixel * 3 + 2] = acc.x;
        }
    }
    return nan;
}

/* One path of orc_render_pt (pixel, sample k): its radiance (out_L[3], r g b) and its
 * extension rays, written to rays (max_depth * 8), t and prim; returns their count. */
int orc_path_rays(const orc_scene_desc *s, int max_depth, int spp, uint64_t seed, long long pixel, int k,
                  float *out_L, float *rays, float *t, int32_t *prim) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x5851F42Du};
    int W = s->width, H = s->height;
    int w = (int)(pixel % W), h = (int)(pixel / W);
    float sx, sy, lu1, lu2;
    V3 o, d;
    (void)H;
    pixel_sample(k, spp, pixel, key, &sx, &sy);
    lens_u(&s->camera, (uint64_t)(pixel * spp + k), key, &lu1, &lu2);
    camera_ray(&s->camera, W, s->height, w, h, sx, sy, lu1, lu2, &o, &d);
    g_dbg_rays = rays; g_dbg_t = t; g_dbg_prim = prim; g_dbg_n = 0;
    V3 L = trace_path(s, max_depth, (uint64_t)(pixel * spp + k), key, o, d);
    int n = g_dbg_n;
    g_dbg_rays = NULL; g_dbg_t = NULL; g_dbg_prim = NULL;
    out_L[0] = L.x; out_L[1] = L.y; out_L[2] = L.z;
    return n;
}

/* Renders rows [row0, row1): film receives B,G,R sums per pixel (Film::_pixel_buffer
 * layout, src/Camera/film.cpp:83-97); NaN samples dropped and counted like
 * Scene::Rendering (src/Scene/scene.cpp:229-241). */
long long orc_render_pt(const orc_scene_desc *s, int max_depth, int spp, uint64_t seed, int row0, int row1,
                        float *film) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x5851F42Du};
    long long nan = 0;
    int W = s->width, H = s->height;
    for (int h = row0; h < row1 && h < H; ++h) {
        for (int w = 0; w < W; ++w) {
            long long pixel = (long long)h * W + w;
            V3 acc = v3(0, 0, 0);
            for (int k = 0; k < spp; ++k) {
                float sx, sy;
                pixel_sample(k, spp, pixel, key, &sx, &sy);
                V3 o, d;
                float lu1, lu2;
                lens_u(&s->camera, (uint64_t)(pixel * spp + k), key, &lu1, &lu2);
                camera_ray(&s->camera, W, H, w, h, sx, sy, lu1, lu2, &o, &d);
                V3 L = trace_path(s, max_depth, (uint64_t)(pixel * spp + k), key, o, d);
                if (isnan3(L))
                    ++nan;
                else
                    acc = add(acc, L);
            }
            film[pixel * 3 + 0] = acc.z;
            film[pixel * 3 + 1] = acc.y;
            film[pixel * 3 + 2] = acc.x;
        }
    }
    return nan;
}

/* ------------------------------------------------------------------ unit entry points */
/* out[9]: wi.xyz, le, go_in, xi, pdf_path, cost, pdfw */
void orc_material_sample(const orc_material *m, const float *wo, const float *n, const float *u, float *out) {
    Bsdf b = mat_sample(m, fv(wo), fv(n), u[0], u[1], u[2]);
    out[0] = b.w.x; out[1] = b.w.y; out[2] = b.w.z;
    out[3] = (float)b.le; out[4] = (float)b.go_in; out[5] = b.xi; out[6] = b.pdf_path; out[7] = b.cost; out[8] = b.pdfw;
}

/* out[3]: r, g, b */
void orc_material_fr(const orc_material *m, const float *n, const float *wi, const float *wo, int in_object, float xi,
                     float pdf_path, float t_in, const float *vol_ratio, float *out) {
    V3 vr = vol_ratio ? fv(vol_ratio) : v3(1, 1, 1);
    V3 f = mat_fr(m, fv(m->rgb), fv(n), fv(wi), fv(wo), in_object, xi, pdf_path, t_in, vr);
    out[0] = f.x; out[1] = f.y; out[2] = f.z;
}

/* out[9]: outcome, s, tau rgb, pdf rgb, unused */
void orc_distance_sample(const float *sigma_s, const float *sigma_a, float smax, float xi, float xa, float *out) {
    V3 st = add(fv(sigma_s), fv(sigma_a));
    float avg = average(st), ab = average(vdiv(fv(sigma_a), st)), sd;
    V3 tau, pdf;
    int oc = dist_sample(st, avg, ab, smax, xi, xa, &sd, &tau, &pdf);
    out[0] = (float)oc; out[1] = sd;
    out[2] = tau.x; out[3] = tau.y; out[4] = tau.z; out[5] = pdf.x; out[6] = pdf.y; out[7] = pdf.z; out[8] = 0.0f;
}

/* out[4]: wi.xyz, pdf (phase about the incoming direction d) */
void orc_phase_sample(const float *d, float g, float u1, float u2, float *out) {
    float pdf = (float)(1.0 / (4.0 * PI_D));
    V3 w = g == 0.0f ? isotropic(fv(d), u1, u2) : hg_sample(fv(d), g, u1, u2, &pdf);
    out[0] = w.x; out[1] = w.y; out[2] = w.z; out[3] = pdf;
}

float orc_hg_eval(float cos_theta, float g) { return hg_eval(cos_theta, g); }

/* Batched forms of the three samplers above for the sample-versus-pdf histogram tests:
 * `count` draws, u holding 3 (material) or 2 (phase, distance) uniforms per draw, out the
 * per-draw records of the single-draw entry points. */
void orc_material_sample_n(const orc_material *m, const float *wo, const float *n, int64_t count, const float *u,
                           float *out) {
    for (int64_t i = 0; i < count; ++i) orc_material_sample(m, wo, n, u + 3 * i, out + 9 * i);
}
void orc_phase_sample_n(const float *d, float g, int64_t count, const float *u, float *out) {
    for (int64_t i = 0; i < count; ++i) orc_phase_sample(d, g, u[2 * i], u[2 * i + 1], out + 4 * i);
}
void orc_distance_sample_n(const float *sigma_s, const float *sigma_a, float smax, int64_t count, const float *u,
                           float *out) {
    for (int64_t i = 0; i < count; ++i) orc_distance_sample(sigma_s, sigma_a, smax, u[2 * i], u[2 * i + 1], out + 9 * i);
}

/* out[6]: o.xyz, d.xyz */
void orc_camera_ray(const orc_camera *c, int W, int H, int w, int h, float sx, float sy, float lu1, float lu2,
                    float *out) {
    V3 o, d;
    camera_ray(c, W, H, w, h, sx, sy, lu1, lu2, &o, &d);
    out[0] = o.x; out[1] = o.y; out[2] = o.z; out[3] = d.x; out[4] = d.y; out[5] = d.z;
}

/* out[2]: pixel sample */
void orc_pixel_sample(int s, int spp, long long pixel, uint64_t seed, float *out) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x5851F42Du};
    pixel_sample(s, spp, pixel, key, &out[0], &out[1]);
}

int orc_perm(int i, int n, uint32_t key) { return perm(i, n, key); }

/* Texture::Pattern of canonical primitives prim[n] at pts (n*3); out n*3 (r, g, b). */
void orc_texture_pattern(const orc_scene_desc *s, int64_t n, const int32_t *prim, const float *pts, float *out) {
    for (int64_t i = 0; i < n; ++i) {
        V3 c = tex_pattern(s, prim[i], fv(pts + 3 * i));
        out[3 * i] = c.x; out[3 * i + 1] = c.y; out[3 * i + 2] = c.z;
    }
}
