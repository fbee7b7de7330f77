// Harness around the reference renderer's own classes (compiled together with the
// reference sources into oracle/_ref/librumi_ref.so by oracle/build_ref.py).
// TEST INFRASTRUCTURE ONLY: the parity tests and the CPU-baseline leg of bench.py call
// it; the GPU product never links or loads it.
//
// It builds scenes exactly as a reference host program does in Scene::Build
// (src/Scene/scene.cpp:135-204): shapes + AddingMaterial, AreaLight over an emissive
// shape, HomogeneousVolume, Pinhole, Film, BVHAccel, then PathTracer or
// BidirectionalPathTracer.  Rendering repeats the per-pixel loop of Scene::Rendering
// (src/Scene/scene.cpp:219-241) over a row range, so several processes can share a
// frame.  Unit entry points call single reference routines with injected uniforms.
#include "Kernel/clibrary.h"
#include "Kernel/vector.h"
#include "Kernel/point.h"
#include "Kernel/color.h"
#include "Kernel/ray.h"
#include "Kernel/bbox.h"
#include "Kernel/matrix.h"
#include "Kernel/bsdf.h"
#include "Kernel/phase.h"
#include "Kernel/intersection.h"
#include "Shape/shape.h"
#include "Shape/triangle.h"
#include "Shape/rect.h"
#include "Shape/sphere.h"
#include "Shape/model.h"
#include "Material/material.h"
#include "Material/matte.h"
#include "Material/glossy.h"
#include "Material/specular.h"
#include "Material/emissive.h"
#include "Material/dielectric.h"
#include "Material/subsurface.h"
#include "Light/light.h"
#include "Light/arealight.h"
#include "Volume/homogeneousvolume.h"
#include "Acceleration/bvh.h"
#include "Camera/pinhole.h"
#include "Camera/film.h"
#include "Sample/sampler.h"
#include "Integrator/integrator.h"
#include "Integrator/path.h"
#include "Integrator/pathtracer.h"
#include "Integrator/bidirectionalpathtracer.h"
#include "Integrator/raytracer.h"
#include "Scene/scene.h"

// ---------------------------------------------------------------------------------
// Random numbers.  The shim maps rand()/srand() here.  Normal mode: splitmix64 with
// 31-bit outputs (RAND_MAX = 2^31-1).  Inject mode: pops caller-supplied uniforms u,
// returning k = u * 2^31 so RandomFloat() = (float)k / (float)RAND_MAX == u exactly for
// every u of the form m * 2^-24 (the form the GPU's Philox uniforms take).
static uint64_t g_rng_state = 0x9E3779B97F4A7C15ull;
static const float *g_inject = nullptr;
static int g_inject_n = 0, g_inject_pos = 0, g_inject_overrun = 0;

extern "C" int rumi_ref_rand(void) {
    if (g_inject) {
        if (g_inject_pos < g_inject_n) {
            double k = (double)g_inject[g_inject_pos++] * 2147483648.0;
            if (k > 2147483647.0) k = 2147483647.0;
            if (k < 0.0) k = 0.0;
            return (int)k;
        }
        ++g_inject_overrun;
        return 0;
    }
    uint64_t z = (g_rng_state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (int)(z >> 33);
}

// Scene::Scene seeds from time(0) (src/Scene/scene.cpp:88); the harness seeds
// explicitly instead, so the constructor's call is ignored.
extern "C" void rumi_ref_srand(unsigned int) {}

extern "C" void ref_seed(unsigned long long seed) {
    g_rng_state = seed * 0xD1B54A32D192ED03ull + 0x8CB92BA72F3D8DD7ull;
}
extern "C" void ref_inject(const float *u, int n) {
    g_inject = u;
    g_inject_n = n;
    g_inject_pos = 0;
    g_inject_overrun = 0;
}
extern "C" int ref_inject_consumed(void) { return g_inject_pos; }
extern "C" int ref_inject_overrun(void) { return g_inject_overrun; }
extern "C" void ref_inject_off(void) { g_inject = nullptr; }

// ---------------------------------------------------------------------------------
// Materials from a flat spec.  type: 0 Matte(kd, rgb) 1 Glossy(kd, ks, e, rgb)
// 2 Specular(kr, rgb) 3 Emissive(ls, rgb) 4 Dielectric(eta_in, eta_out, absorption rgb)
// 5 Subsurface(eta_in, eta_out, sigma_s rgb, sigma_a rgb, density).
// params layout (floats): [0..2] scalars a,b,c  [3..5] rgb  [6..8] rgb2  [9] density
enum { M_MATTE = 0, M_GLOSSY = 1, M_SPECULAR = 2, M_EMISSIVE = 3, M_DIELECTRIC = 4, M_SUBSURFACE = 5 };

static Material *make_material(int type, const float *p) {
    Color c1(p[3], p[4], p[5]);
    Color c2(p[6], p[7], p[8]);
    switch (type) {
    case M_MATTE: return new Matte(p[0], c1);
    case M_GLOSSY: return new Glossy(p[0], p[1], p[2], c1);
    case M_SPECULAR: return new Specular(p[0], c1);
    case M_EMISSIVE: return new Emissive(p[0], c1);
    case M_DIELECTRIC: return new Dielectric(p[0], p[1], c1);
    case M_SUBSURFACE: return new Subsurface(p[0], p[1], c1, c2, p[9] > 0.0f ? p[9] : 1.0f);
    default: return nullptr;
    }
}

struct RefScene {
    Scene *scene = nullptr;
    std::vector<Shape *> objects;            // top-level shapes (Scene::_objects)
    std::vector<Light *> lights;             // Scene::_lights
    std::unordered_map<const Shape *, int> prim_id;  // leaf shape -> global primitive id
    int next_prim = 0;
    int width = 0, height = 0, spp = 0;
    int integrator = 0;
};

static Point3 P3(const float *v) { return Point3(v[0], v[1], v[2]); }
static Vector3 V3(const float *v) { return Vector3(v[0], v[1], v[2]); }

extern "C" void *ref_scene_new(int width, int height, int spp, float gamma) {
    RefScene *rs = new RefScene();
    rs->scene = new Scene();
    rs->width = width;
    rs->height = height;
    rs->spp = spp;
    rs->scene->_image = new Film(width, height, 4, spp, gamma);
    return rs;
}

// Standalone Triangle shapes (each its own top-level object, own material instance).
// v: n*9 floats, nrm: n*9 floats or NULL (NULL -> face normal Normalize(Cross(v1-v0, v2-v0)),
// the rule Model::LoadObjectFile applies without vn, src/Shape/model.cpp:320-323).
// params: material params, advanced by params_stride floats per triangle (0 = shared).
extern "C" int ref_add_triangles(void *h, int n, const float *v, const float *nrm, int mat_type,
                                 const float *params, int params_stride) {
    RefScene *rs = (RefScene *)h;
    int first = (int)rs->objects.size();
    for (int i = 0; i < n; ++i) {
        const float *t = v + 9 * (size_t)i;
        Point3 a = P3(t), b = P3(t + 3), c = P3(t + 6);
        Triangle *tri = new Triangle(a, b, c);
        if (nrm) {
            const float *m = nrm + 9 * (size_t)i;
            tri->Normal(V3(m), V3(m + 3), V3(m + 6));
        } else {
            Vector3 fn = Normalize(Cross(b - a, c - a));
            tri->Normal(fn, fn, fn);
        }
        tri->AddingMaterial(make_material(mat_type, params + (size_t)params_stride * i));
        rs->prim_id[tri] = rs->next_prim++;
        rs->objects.push_back(tri);
    }
    return first;
}

// A Model: triangles inside their own BVH, one shared material (src/Shape/model.cpp:35-74,
// 345-354).  The triangle arrays replace LoadObjectFile's parse; the transform is identity.
extern "C" int ref_add_model(void *h, int n, const float *v, const float *nrm, int mat_type,
                             const float *params) {
    RefScene *rs = (RefScene *)h;
    Model *m = new Model();
    m->_n_triangles = n;
    m->_triangles = new Triangle *[n];
    for (int i = 0; i < n; ++i) {
        const float *t = v + 9 * (size_t)i;
        Point3 a = P3(t), b = P3(t + 3), c = P3(t + 6);
        Triangle *tri = new Triangle(a, b, c);
        if (nrm) {
            const float *q = nrm + 9 * (size_t)i;
            tri->Normal(V3(q), V3(q + 3), V3(q + 6));
        } else {
            Vector3 fn = Normalize(Cross(b - a, c - a));
            tri->Normal(fn, fn, fn);
        }
        m->_triangles[i] = tri;
        rs->prim_id[tri] = rs->next_prim++;
    }
    m->BuildAccel();
    m->AddingMaterial(make_material(mat_type, params));
    int idx = (int)rs->objects.size();
    rs->objects.push_back(m);
    return idx;
}

extern "C" int ref_add_rect(void *h, const float *p, const float *l, const float *w, int n_samples,
                            int mat_type, const float *params) {
    RefScene *rs = (RefScene *)h;
    Rect *r = n_samples > 0 ? new Rect(P3(p), V3(l), V3(w), n_samples) : new Rect(P3(p), V3(l), V3(w));
    r->AddingMaterial(make_material(mat_type, params));
    rs->prim_id[r] = rs->next_prim++;
    int idx = (int)rs->objects.size();
    rs->objects.push_back(r);
    return idx;
}

extern "C" int ref_add_sphere(void *h, const float *c, float radius, int n_samples, int mat_type,
                              const float *params) {
    RefScene *rs = (RefScene *)h;
    Sphere *s = n_samples > 0 ? new Sphere(P3(c), radius, n_samples) : new Sphere(P3(c), radius);
    s->AddingMaterial(make_material(mat_type, params));
    rs->prim_id[s] = rs->next_prim++;
    int idx = (int)rs->objects.size();
    rs->objects.push_back(s);
    return idx;
}

extern "C" int ref_add_area_light(void *h, int object_index) {
    RefScene *rs = (RefScene *)h;
    Shape *s = rs->objects.at(object_index);
    rs->lights.push_back(new AreaLight(s, s->MaterialPtr()));
    return (int)rs->lights.size() - 1;
}

extern "C" void ref_set_volume(void *h, const float *bmin, const float *bmax, const float *sigma_s,
                               const float *sigma_a) {
    RefScene *rs = (RefScene *)h;
    rs->scene->_volume_ptr = new HomogeneousVolume(BBox(P3(bmin), P3(bmax)),
                                                   Color(sigma_s[0], sigma_s[1], sigma_s[2]),
                                                   Color(sigma_a[0], sigma_a[1], sigma_a[2]));
}

// basis16: row-major Mat4x4 (Pinhole::_basis_transform); fov_deg > 0 overrides the
// constructor's fixed 20 degrees with the constructor's own formulas
// (src/Camera/pinhole.cpp:36-47).
extern "C" void ref_set_camera(void *h, const float *pos, const float *basis16, float y_ratio, float fov_deg) {
    RefScene *rs = (RefScene *)h;
    Mat4x4 m;
    for (int i = 0; i < 16; ++i) m._m[i] = basis16[i];
    Pinhole *cam = new Pinhole(P3(pos), m, y_ratio);
    if (fov_deg > 0.0f) {
        cam->_fov = fov_deg;
        cam->_tanfov = tan(PI / 180.f * cam->_fov * 0.5f);
        cam->_film_area = (2.0f * cam->_tanfov) * (2.0f * cam->_tanfov * cam->_y_ratio);
    }
    rs->scene->_camera = cam;
}

// Pinhole::DepthOfField on the scene's camera (the BDPT constructor turns it off again).
extern "C" void ref_set_camera_dof(void *h, float focal_distance, float lens_radius) {
    ((RefScene *)h)->scene->_camera->DepthOfField(focal_distance, lens_radius);
}

// integrator: 0 PathTracer(max_depth=a), 1 BidirectionalPathTracer(nL=a, nE=b),
// 2 RayTracer(max_depth=a).
// Sample sets are generated after seeding, as Scene::Build does once per frame.
extern "C" int ref_finalize(void *h, int integrator, int a, int b, unsigned long long seed) {
    RefScene *rs = (RefScene *)h;
    Scene *sc = rs->scene;
    ref_seed(seed);
    sc->_image->PixelSampler()->GenerateSamples();
    for (Shape *s : rs->objects) s->GenerateSamples();
    sc->_n_objects = (int)rs->objects.size();
    sc->_objects = new Shape *[sc->_n_objects];
    for (int i = 0; i < sc->_n_objects; ++i) sc->_objects[i] = rs->objects[i];
    sc->_n_lights = (int)rs->lights.size();
    sc->_lights = new Light *[sc->_n_lights > 0 ? sc->_n_lights : 1];
    for (int i = 0; i < sc->_n_lights; ++i) sc->_lights[i] = rs->lights[i];
    sc->_bvh_ptr = new BVHAccel(sc->_objects, sc->_n_objects);
    rs->integrator = integrator;
    if (integrator == 0)
        sc->_tracer_ptr = new PathTracer(sc, a);
    else if (integrator == 2)
        sc->_tracer_ptr = new RayTracer(sc, a);
    else
        sc->_tracer_ptr = new BidirectionalPathTracer(sc, a, b);
    return 0;
}

// Renders rows [row0, row1) exactly as Scene::Rendering's loop does
// (src/Scene/scene.cpp:219-241): Trace per pixel sample, NaN samples dropped, the
// per-pixel sum added to Film::_pixel_buffer.  film_out (H*W*3, B,G,R like the
// reference buffer) receives the pixel sums of those rows; light_out (may be NULL)
// receives the BDPT light-tracing splats un-flipped into pixel layout, as
// Film::CombineBuffer would add them (src/Camera/film.cpp:123-150).
extern "C" long long ref_render_rows(void *h, unsigned long long seed, int row0, int row1, float *film_out,
                                     float *light_out) {
    RefScene *rs = (RefScene *)h;
    Scene *sc = rs->scene;
    Film *film = sc->_image;
    ref_seed(seed);
    const int W = film->Width(), H = film->Height();
    const int n_samples = film->PixelSampler()->SampleCount();
    long long nan_count = 0;
    memset(film->_pixel_buffer, 0, sizeof(float) * W * H * 3);
    if (film->_light_buffer) memset(film->_light_buffer, 0, sizeof(float) * W * H * 3);
    Color Lo, lo;
    for (int hh = row0; hh < row1 && hh < H; ++hh) {
        for (int ww = 0; ww < W; ++ww) {
            for (int s = 0; s < n_samples; ++s) {
                lo = sc->_tracer_ptr->Trace(ww, hh, sc->_camera, film);
                if (lo.IsNaN() == true)
                    ++nan_count;
                else
                    Lo += lo;
            }
            film->Pixel(ww, hh, Lo);
            Lo._r = Lo._g = Lo._b = 0.0f;
        }
    }
    if (film_out) memcpy(film_out, film->_pixel_buffer, sizeof(float) * W * H * 3);
    if (light_out) {
        if (film->_light_buffer) {
            for (int hh = 0; hh < H; ++hh)
                for (int ww = 0; ww < W; ++ww)
                    for (int c = 0; c < 3; ++c)
                        light_out[(hh * W + ww) * 3 + c] = film->_light_buffer[((H - (hh + 1)) * W + ww) * 3 + c];
        } else {
            memset(light_out, 0, sizeof(float) * W * H * 3);
        }
    }
    return nan_count;
}

extern "C" int ref_sample_count(void *h) {
    return ((RefScene *)h)->scene->_image->PixelSampler()->SampleCount();
}

// Closest-hit (anyhit=0) or shadow/any-hit (anyhit=1) queries through BVHAccel::Travel
// (src/Acceleration/bvh.cpp:150-213) on the scene's top-level BVH.
// rays: n*7 floats (o.xyz, d.xyz, tmax).  t_out: Ray::_tmin after traversal (0 = miss);
// id_out: global primitive id of isect->_object_ptr (-1 = miss; any-hit: 1 blocked / 0);
// n_out (closest-hit, may be NULL): the Vertex normal the shape wrote (3 floats).
extern "C" void ref_trace(void *h, int n, const float *rays, int anyhit, float *t_out, int *id_out,
                          float *n_out) {
    RefScene *rs = (RefScene *)h;
    Scene *sc = rs->scene;
    for (int i = 0; i < n; ++i) {
        const float *r = rays + 7 * (size_t)i;
        Ray ray(P3(r), V3(r + 3));
        ray._tmax = r[6];
        if (anyhit) {
            sc->_bvh_ptr->Travel(&ray, nullptr);
            t_out[i] = ray._tmin;
            id_out[i] = ray._tmin > 0.0f ? 1 : 0;
        } else {
            Vertex v;
            Intersection info(&ray, sc);
            info._vertex_ptr = &v;
            sc->_bvh_ptr->Travel(&ray, &info);
            t_out[i] = ray._tmin;
            int id = -1;
            if (info._object_ptr) {
                auto it = rs->prim_id.find(info._object_ptr);
                id = it == rs->prim_id.end() ? -2 : it->second;
            }
            id_out[i] = id;
            if (n_out) {
                n_out[3 * i + 0] = v._n._x;
                n_out[3 * i + 1] = v._n._y;
                n_out[3 * i + 2] = v._n._z;
            }
        }
    }
}

extern "C" void ref_scene_free(void *h) {
    RefScene *rs = (RefScene *)h;
    if (!rs) return;
    delete rs->scene;  // owns objects, lights, volume, camera, film, BVH, integrator
    delete rs;
}

// ---------------------------------------------------------------------------------
// Unit entry points: one reference routine per call, uniforms injected by the caller.

// Material::BSDFSampling (src/Material/*.cpp).  out[12]: wi.xyz, Le, go_into_object, xi,
// pdf_path, costheta, pdf_w.
extern "C" void ref_material_sample(int mat_type, const float *params, const float *wo, const float *n,
                                    float *out) {
    Material *m = make_material(mat_type, params);
    bool le = false, goin = false;
    float xi = 1.0f, pdf_path = 1.0f, cost = 1.0f, pdfw = 1.0f;
    Vector3 wi = m->BSDFSampling(V3(wo), V3(n), &le, &goin, &xi, &pdf_path, &cost, &pdfw);
    out[0] = wi._x; out[1] = wi._y; out[2] = wi._z;
    out[3] = le ? 1.0f : 0.0f; out[4] = goin ? 1.0f : 0.0f;
    out[5] = xi; out[6] = pdf_path; out[7] = cost; out[8] = pdfw;
    delete m;
}

// Material::Fr with the Intersection state it reads: _in_object, _rand (lobe xi),
// vertex _pdf_path, ray _tmin (Beer-Lambert distance), volumetric tau / pdf.
// out[3]: r, g, b.
extern "C" void ref_material_fr(int mat_type, const float *params, const float *n, const float *wi,
                                const float *wo, int in_object, float xi, float pdf_path, float tmin,
                                const float *vol_tau, const float *vol_pdf, float *out) {
    Material *m = make_material(mat_type, params);
    Ray ray;
    ray._tmin = tmin;
    Vertex v;
    v._pdf_path = pdf_path;
    Intersection info(&ray, nullptr);
    info._vertex_ptr = &v;
    info._in_object = in_object != 0;
    info._rand = xi;
    if (vol_tau) info._volumetric_tau = Color(vol_tau[0], vol_tau[1], vol_tau[2]);
    if (vol_pdf) info._volumetric_pdf = Color(vol_pdf[0], vol_pdf[1], vol_pdf[2]);
    Color f = m->Fr(info, V3(n), V3(wi), V3(wo));
    out[0] = f._r; out[1] = f._g; out[2] = f._b;
    delete m;
}

// Material::Pdfw (Glossy reads the lobe choice from info._rand).
extern "C" float ref_material_pdfw(int mat_type, const float *params, const float *n, const float *w,
                                   const float *w_pdf, float xi) {
    Material *m = make_material(mat_type, params);
    Intersection info;
    info._rand = xi;
    float r = m->Pdfw(info, V3(n), V3(w), V3(w_pdf));
    delete m;
    return r;
}

// FresnelReflection::Fresnel (src/Kernel/bsdf.cpp:256-283).
extern "C" float ref_fresnel(const float *d, const float *n, float eta_in, float eta_out) {
    FresnelReflection fr(Color(1.0f, 1.0f, 1.0f));
    return fr.Fresnel(V3(d), V3(n), eta_in, eta_out);
}

// Isotropic::PhaseSampling (src/Kernel/phase.cpp:34-71).  out[4]: wi.xyz, pdf.
extern "C" void ref_isotropic_sample(const float *direction, float *out) {
    Isotropic iso;
    float pdf = 0.0f;
    Vector3 w = iso.PhaseSampling(V3(direction), &pdf);
    out[0] = w._x; out[1] = w._y; out[2] = w._z; out[3] = pdf;
}

// OrthonormalBasis (src/Kernel/vector.h:70-95).  out[6]: v1.xyz, v2.xyz.
extern "C" void ref_onb(const float *v0, float *out) {
    Vector3 a, b;
    OrthonormalBasis(V3(v0), &a, &b);
    out[0] = a._x; out[1] = a._y; out[2] = a._z; out[3] = b._x; out[4] = b._y; out[5] = b._z;
}

// HomogeneousVolume pieces (src/Volume/homogeneousvolume.cpp:46-215).
// out[10]: returned bool, s, absorb, tau rgb, pdf rgb, (unused).
extern "C" void ref_volume_distance_sampling(const float *sigma_s, const float *sigma_a, float max_distance,
                                             float *out) {
    HomogeneousVolume vol(BBox(Point3(0, 0, 0), Point3(1, 1, 1)), Color(sigma_s[0], sigma_s[1], sigma_s[2]),
                          Color(sigma_a[0], sigma_a[1], sigma_a[2]));
    float s = 0.0f;
    bool absorb = false;
    Color tau(1.0f), pdf(1.0f);
    bool r = vol.DistanceSampling(max_distance, &s, &absorb, &tau, &pdf);
    out[0] = r; out[1] = s; out[2] = absorb;
    out[3] = tau._r; out[4] = tau._g; out[5] = tau._b;
    out[6] = pdf._r; out[7] = pdf._g; out[8] = pdf._b;
}

// HomogeneousVolume::Intersect + MaxDistance for a ray with hit distance thit
// (Ray::_tmin after Travel).  out[4]: hit flag, tnear, tfar, max_distance.
extern "C" void ref_volume_segment(const float *bmin, const float *bmax, const float *o, const float *d,
                                   float thit, float *out) {
    HomogeneousVolume vol(BBox(P3(bmin), P3(bmax)), Color(0.1f), Color(0.1f));
    Ray ray(P3(o), V3(d));
    ray._tmin = thit;
    float tn = 0.0f, tf = 0.0f;
    bool hit = vol.Intersect(ray, &tn, &tf);
    out[0] = hit; out[1] = tn; out[2] = tf;
    out[3] = hit ? vol.MaxDistance(thit, tn, tf) : 0.0f;
}

// HomogeneousVolume::ShadowRayTr (binary transmittance).  out[3]: rgb.
extern "C" void ref_volume_shadow_tr(const float *bmin, const float *bmax, const float *sigma_s,
                                     const float *sigma_a, const float *o, const float *d, float tmax,
                                     float *out) {
    HomogeneousVolume vol(BBox(P3(bmin), P3(bmax)), Color(sigma_s[0], sigma_s[1], sigma_s[2]),
                          Color(sigma_a[0], sigma_a[1], sigma_a[2]));
    Ray ray(P3(o), V3(d));
    ray._tmax = tmax;
    Color c = vol.ShadowRayTr(ray);
    out[0] = c._r; out[1] = c._g; out[2] = c._b;
}

// Subsurface::DistanceSampling (src/Material/subsurface.cpp:49-98).  out[10] as the volume.
extern "C" void ref_subsurface_distance_sampling(const float *params, float tfar, float *out) {
    Material *m = make_material(M_SUBSURFACE, params);
    Subsurface *ss = (Subsurface *)m;
    float s = 0.0f, smax = 0.0f;
    bool absorb = false;
    Color tau(1.0f), pdf(1.0f);
    bool r = ss->DistanceSampling(0.0f, tfar, &absorb, &s, &smax, &tau, &pdf);
    out[0] = r; out[1] = s; out[2] = absorb;
    out[3] = tau._r; out[4] = tau._g; out[5] = tau._b;
    out[6] = pdf._r; out[7] = pdf._g; out[8] = pdf._b; out[9] = smax;
    delete m;
}

// Pinhole::CastViewRay (src/Camera/pinhole.cpp:97-136) for one pixel and sub-pixel
// sample.  out[8]: o.xyz, d.xyz, costheta, pdf_w.
extern "C" void ref_camera_cast(const float *pos, const float *basis16, float y_ratio, float fov_deg, int W,
                                int H, int w, int h, float sx, float sy, float *out) {
    Mat4x4 m;
    for (int i = 0; i < 16; ++i) m._m[i] = basis16[i];
    Pinhole cam(P3(pos), m, y_ratio);
    if (fov_deg > 0.0f) {
        cam._fov = fov_deg;
        cam._tanfov = tan(PI / 180.f * cam._fov * 0.5f);
        cam._film_area = (2.0f * cam._tanfov) * (2.0f * cam._tanfov * cam._y_ratio);
    }
    Point3 o;
    Vector3 d;
    float cost = 0.0f, pdf = 0.0f;
    cam.CastViewRay(W, H, w, h, Point2(sx, sy), &o, &d, &cost, &pdf);
    out[0] = o._x; out[1] = o._y; out[2] = o._z; out[3] = d._x; out[4] = d._y; out[5] = d._z;
    out[6] = cost; out[7] = pdf;
}

// Pinhole::CastViewRay with depth of field: the harness generator is seeded with
// `seed` before the call (and restored after it), and the two RandomFloat() values the call draws (lens radius, then angle) are
// drawn again from the same seed and reported.  out[10]: o.xyz, d.xyz, costheta, pdf_w,
// u1, u2.
extern "C" void ref_camera_cast_dof(const float *pos, const float *basis16, float y_ratio, float fov_deg,
                                    float focal_distance, float lens_radius, int W, int H, int w, int h, float sx,
                                    float sy, unsigned seed, float *out) {
    Mat4x4 m;
    for (int i = 0; i < 16; ++i) m._m[i] = basis16[i];
    Pinhole cam(P3(pos), m, y_ratio);
    if (fov_deg > 0.0f) {
        cam._fov = fov_deg;
        cam._tanfov = tan(PI / 180.f * cam._fov * 0.5f);
        cam._film_area = (2.0f * cam._tanfov) * (2.0f * cam._tanfov * cam._y_ratio);
    }
    cam.DepthOfField(focal_distance, lens_radius);
    const uint64_t saved = g_rng_state;
    ref_seed(seed);
    const float u1 = RandomFloat();
    const float u2 = RandomFloat();
    ref_seed(seed);
    Point3 o;
    Vector3 d;
    float cost = 0.0f, pdf = 0.0f;
    cam.CastViewRay(W, H, w, h, Point2(sx, sy), &o, &d, &cost, &pdf);
    out[0] = o._x; out[1] = o._y; out[2] = o._z; out[3] = d._x; out[4] = d._y; out[5] = d._z;
    g_rng_state = saved;
    out[6] = cost; out[7] = pdf; out[8] = u1; out[9] = u2;
}

// Reads back Pinhole::_tanfov / _film_area of a scene's camera.  out[2].
extern "C" void ref_camera_params(void *h, float *out) {
    RefScene *rs = (RefScene *)h;
    out[0] = rs->scene->_camera->_tanfov;
    out[1] = rs->scene->_camera->_film_area;
}

#include <fcntl.h>
#include <unistd.h>

// Model(file, transform) (src/Shape/model.cpp:35-43, 76-343): the triangles the reference
// loads from an OBJ file.  m16: row-major Mat4x4 (NULL = identity).  Writes up to cap
// triangles (9 vertex floats and 9 normal floats each) and returns the model's count.
extern "C" int ref_load_obj(const char *path, const float *m16, int cap, float *v_out, float *n_out) {
    Mat4x4 m;
    if (m16)
        for (int k = 0; k < 16; ++k) m._m[k] = m16[k];
    int devnull = open("/dev/null", O_WRONLY), saved = dup(1);
    fflush(stdout);
    dup2(devnull, 1);  // the loader prints progress
    Model *model = new Model(path, m);
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
    close(devnull);
    const int n = model->_n_triangles;
    for (int i = 0; i < n && i < cap; ++i) {
        const Triangle *t = model->_triangles[i];
        const Point3 *v[3] = {&t->_v0, &t->_v1, &t->_v2};
        const Vector3 *nn[3] = {&t->_n0, &t->_n1, &t->_n2};
        for (int k = 0; k < 3; ++k) {
            v_out[9 * i + 3 * k + 0] = v[k]->_x;
            v_out[9 * i + 3 * k + 1] = v[k]->_y;
            v_out[9 * i + 3 * k + 2] = v[k]->_z;
            n_out[9 * i + 3 * k + 0] = nn[k]->_x;
            n_out[9 * i + 3 * k + 1] = nn[k]->_y;
            n_out[9 * i + 3 * k + 2] = nn[k]->_z;
        }
    }
    delete model;
    return n;
}

// Film::Save (src/Camera/film.cpp:152-203) and FirefliesFiltering (src/Scene/scene.cpp:
// 261-432) on a caller's pixel sums: writes the reference's BMP into `dir`, reads it back
// with the reference's LoadBmp (tonemapped bytes, W*H*bpp), runs the fireflies filter on
// that file and reads its output (filtered bytes).
#include "Kernel/bmp.h"
extern "C" int ref_film_save_filter(const char *dir, int width, int height, int bpp, int spp, float gamma,
                                    const float *film, unsigned char *tonemapped, unsigned char *filtered) {
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd)) || chdir(dir) != 0) return -1;
    int devnull = open("/dev/null", O_WRONLY), saved = dup(1);
    fflush(stdout);
    dup2(devnull, 1);
    Film *f = new Film(width, height, bpp, spp, gamma);
    memcpy(f->_pixel_buffer, film, sizeof(float) * width * height * 3);
    f->Save(0.0f);  // "0.000s.bmp"
    unsigned int w = 0, h = 0, b = 0;
    char name[] = "0.000s.bmp";
    unsigned char *t = LoadBmp(name, &w, &h, &b);
    memcpy(tonemapped, t, (size_t)width * height * bpp);
    free(t);
    FirefliesFiltering(name);
    char out_name[] = "FirefliesFiltering.bmp";
    unsigned char *g = LoadBmp(out_name, &w, &h, &b);
    memcpy(filtered, g, (size_t)width * height * bpp);
    free(g);
    delete f;
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
    close(devnull);
    return chdir(cwd) == 0 ? 0 : -1;
}

// ---------------------------------------------------------------------------------
// Textures and image-based lights.
#include "Texture/texture.h"
#include "Texture/checker.h"
#include "Texture/imagetexture.h"
#include "Texture/hdrtexture.h"
#include "Light/imagebasedlight.h"
#include "Kernel/hdr.h"

// Shape::AddingTexture (Model::AddingTexture hands it to every triangle) of top-level
// object `object_index`: kind 0 Checker(w, h, c1, c2); 1 ImageTexture(path, gamma);
// 2 HDRTexture(path).  Colours are (r, g, b).
extern "C" int ref_add_texture(void *h, int object_index, int kind, float w, float hh, const float *c1,
                               const float *c2, const char *path, float gamma) {
    RefScene *rs = (RefScene *)h;
    Shape *s = rs->objects.at(object_index);
    Texture *t = nullptr;
    if (kind == 0)
        t = new Checker(w, hh, Color(c1[0], c1[1], c1[2]), Color(c2[0], c2[1], c2[2]));
    else if (kind == 1)
        t = new ImageTexture((char *)path, gamma);
    else
        t = new HDRTexture((char *)path);
    s->AddingTexture(t);
    return 0;
}

// Shape::_transform (public; Sphere::TextureMapping reads its upper 3x3 rows).
extern "C" void ref_set_shape_transform(void *h, int object_index, const float *m16) {
    RefScene *rs = (RefScene *)h;
    Shape *s = rs->objects.at(object_index);
    for (int i = 0; i < 16; ++i) s->_transform._m[i] = m16[i];
}

extern "C" int ref_add_ibl_light(void *h, int object_index) {
    RefScene *rs = (RefScene *)h;
    Shape *s = rs->objects.at(object_index);
    rs->lights.push_back(new ImageBasedLight(s, s->MaterialPtr(), s->TexturePtr()));
    return (int)rs->lights.size() - 1;
}

// Texture::Pattern(shape, p) of a top-level object's texture at n points (n*3 floats);
// out n*3 (r, g, b).
extern "C" void ref_texture_pattern(void *h, int object_index, int n, const float *pts, float *out) {
    RefScene *rs = (RefScene *)h;
    Shape *s = rs->objects.at(object_index);
    Texture *t = s->TexturePtr();
    for (int i = 0; i < n; ++i) {
        Color c = t ? t->Pattern(s, P3(pts + 3 * (size_t)i)) : Color(1.0f);
        out[3 * i] = c._r; out[3 * i + 1] = c._g; out[3 * i + 2] = c._b;
    }
}

// LoadHDR into a caller buffer of `cap` floats; returns width * height (0 on failure),
// dims in wh[2].
extern "C" int ref_load_hdr(const char *path, int cap, float *out, int *wh) {
    float *buf = nullptr;
    int w = 0, hgt = 0;
    LoadHDR((char *)path, &buf, &w, &hgt);
    wh[0] = w;
    wh[1] = hgt;
    if (!buf) return 0;
    const long long n = (long long)w * hgt;
    if (n * 3 <= cap) memcpy(out, buf, sizeof(float) * 3 * (size_t)n);
    free(buf);
    return (int)n;
}

// LoadBmp into a caller buffer of `cap` bytes; returns the byte count, dims in whb[3].
extern "C" int ref_load_bmp(const char *path, int cap, unsigned char *out, unsigned int *whb) {
    unsigned char *buf = LoadBmp((char *)path, &whb[0], &whb[1], &whb[2]);
    const long long n = (long long)whb[0] * whb[1] * whb[2];
    if (buf && n <= cap) memcpy(out, buf, (size_t)n);
    free(buf);
    return (int)n;
}

// The reference Scene a harness handle wraps (the GPU-integrator host library,
// oracle/ref_gpu_host.cpp, installs its integrators on it).
extern "C" void *ref_scene_ptr(void *h) { return ((RefScene *)h)->scene; }
