// Reference-side adapter: GPU integrators behind the reference's Integrator interface
// (declarations and usage in rumi_gpu_integrators.h).
//
// RumiFlattenScene restates, in the other direction, what the reference's constructors
// store (each cited below), so that the descriptor carries the same numbers the
// reference's own routines read during rendering.
#include "rumi_gpu_integrators.h"

#include <cstdio>
#include <cstring>
#include <map>
#include <utility>

#include "Camera/film.h"
#include "Camera/pinhole.h"
#include "Kernel/bbox.h"
#include "Kernel/bsdf.h"
#include "Kernel/color.h"
#include "Kernel/matrix.h"
#include "Kernel/point.h"
#include "Kernel/vector.h"
#include "Light/arealight.h"
#include "Light/imagebasedlight.h"
#include "Light/light.h"
#include "Material/dielectric.h"
#include "Material/emissive.h"
#include "Material/glossy.h"
#include "Material/material.h"
#include "Material/matte.h"
#include "Material/specular.h"
#include "Material/subsurface.h"
#include "Sample/sampler.h"
#include "Scene/scene.h"
#include "Shape/model.h"
#include "Shape/rect.h"
#include "Shape/shape.h"
#include "Shape/sphere.h"
#include "Shape/triangle.h"
#include "Texture/checker.h"
#include "Texture/hdrtexture.h"
#include "Texture/imagetexture.h"
#include "Texture/texture.h"
#include "Volume/homogeneousvolume.h"

// Reads the private members the flattening needs.  Classes that must declare
// `friend struct RumiSceneAccess;`: Triangle, Rect, Sphere, Model, Matte, Glossy,
// Specular, Emissive, Dielectric, Subsurface, Lambertian, Phong, PerfectReflection,
// AreaLight, ImageBasedLight, HomogeneousVolume, Checker, ImageTexture, HDRTexture.
struct RumiSceneAccess {
    static void put3(float *o, const Point3 &p) { o[0] = p._x; o[1] = p._y; o[2] = p._z; }
    static void put3(float *o, const Vector3 &v) { o[0] = v._x; o[1] = v._y; o[2] = v._z; }
    static void rgb(float *o, const Color &c) { o[0] = c._r; o[1] = c._g; o[2] = c._b; }

    static void triangle(const Triangle *t, float *v9, float *n9) {
        put3(v9, t->_v0); put3(v9 + 3, t->_v1); put3(v9 + 6, t->_v2);
        put3(n9, t->_n0); put3(n9 + 3, t->_n1); put3(n9 + 6, t->_n2);
    }
    static int model_count(const Model *m) { return m->_n_triangles; }
    static const Triangle *model_triangle(const Model *m, int i) { return m->_triangles[i]; }
    // Rect(p, l, w) (src/Shape/rect.cpp:12-20) keeps p, l, w as given
    static void rect(const Rect *r, float *o9) { put3(o9, r->_p); put3(o9 + 3, r->_vect_l); put3(o9 + 6, r->_vect_w); }
    static void sphere(const Sphere *s, float *o4) { put3(o4, s->_c); o4[3] = s->_r; }

    // Material constructors: Matte(kd, rgb) -> _kd, Lambertian(rgb) (matte.cpp:26-31);
    // Glossy(kd, ks, e, rgb) -> Matte(kd, rgb), _ks, Phong(e, rgb) (glossy.cpp:27-33);
    // Specular(kr, rgb) -> _kr, PerfectReflection(rgb) (specular.cpp:24-29);
    // Emissive(ls, ce) -> _ls, _ce (emissive.cpp:19-25); Dielectric(eta_in, eta_out, a) ->
    // FresnelTransparency(eta_in, eta_out, a) (dielectric.cpp:26-31); Subsurface(eta_in,
    // eta_out, s, a, density) -> _sigma_s, _sigma_a, _avg_sigmat = avg(s + a) * density
    // (subsurface.cpp:34-47).
    static bool material(const Material *m, rumi_material *o) {
        memset(o, 0, sizeof(*o));
        o->eta_in = o->eta_out = 1.0f;  // the fields a kind does not use keep neutral values
        o->density = 1.0f;
        if (const Glossy *g = dynamic_cast<const Glossy *>(m)) {
            o->type = RUMI_MAT_GLOSSY;
            o->kd = g->_kd;
            o->ks = g->_ks;
            o->exponent = g->_phong_brdf ? static_cast<const Phong *>(g->_phong_brdf)->_e : 0.0f;
            rgb(o->rgb, static_cast<const Lambertian *>(g->_diffuse_brdf)->_cd);
        } else if (const Matte *mt = dynamic_cast<const Matte *>(m)) {
            o->type = RUMI_MAT_MATTE;
            o->kd = mt->_kd;
            rgb(o->rgb, static_cast<const Lambertian *>(mt->_diffuse_brdf)->_cd);
        } else if (const Specular *sp = dynamic_cast<const Specular *>(m)) {
            o->type = RUMI_MAT_SPECULAR;
            o->kd = sp->_kr;
            rgb(o->rgb, static_cast<const PerfectReflection *>(sp->_specular_brdf)->_cr);
        } else if (const Emissive *e = dynamic_cast<const Emissive *>(m)) {
            o->type = RUMI_MAT_EMISSIVE;
            o->kd = e->_ls;
            rgb(o->rgb, e->_ce);
        } else if (const Dielectric *d = dynamic_cast<const Dielectric *>(m)) {
            o->type = RUMI_MAT_DIELECTRIC;
            o->eta_in = d->_fresnel_btdf->_eta_in;
            o->eta_out = d->_fresnel_btdf->_eta_out;
            rgb(o->rgb, d->_fresnel_btdf->_absorption);
        } else if (const Subsurface *s = dynamic_cast<const Subsurface *>(m)) {
            o->type = RUMI_MAT_SUBSURFACE;
            o->eta_in = s->_fresnel_btdf->_eta_in;
            o->eta_out = s->_fresnel_btdf->_eta_out;
            rgb(o->rgb, s->_sigma_s);
            rgb(o->rgb2, s->_sigma_a);
            const float avg = (s->_sigma_t._b + s->_sigma_t._g + s->_sigma_t._r) / 3.0f;
            o->density = avg > 0.0f ? s->_avg_sigmat / avg : 1.0f;
        } else {
            return false;
        }
        return true;
    }
    static const Shape *area_light_shape(const AreaLight *l) { return l->_object; }
    static const Shape *ibl_shape(const ImageBasedLight *l) { return l->_object; }

    static void volume(const HomogeneousVolume *v, rumi_volume *o) {
        memset(o, 0, sizeof(*o));
        o->present = 1;
        put3(o->pmin, v->_extents._pmin);
        put3(o->pmax, v->_extents._pmax);
        rgb(o->sigma_s, v->_sigma_s);
        rgb(o->sigma_a, v->_sigma_a);
        o->g = 0.0f;  // the reference's medium has the Isotropic phase
    }

    // Checker(w, h, c1, c2) (checker.cpp:17-22); ImageTexture keeps LoadBmp's bytes
    // (imagetexture.cpp:20-30); HDRTexture keeps LoadHDR's floats (hdrtexture.cpp:19-28)
    static bool texture(const Texture *t, rumi_texture *o) {
        memset(o, 0, sizeof(*o));
        o->gamma = 1.0f;
        if (const Checker *c = dynamic_cast<const Checker *>(t)) {
            o->type = RUMI_TEX_CHECKER;
            o->repeat_u = c->_w;
            o->repeat_v = c->_h;
            rgb(o->color1, c->_c1);
            rgb(o->color2, c->_c2);
        } else if (const ImageTexture *it = dynamic_cast<const ImageTexture *>(t)) {
            o->type = RUMI_TEX_IMAGE;
            o->gamma = it->_gamma;
            o->img_width = (int32_t)it->_width;
            o->img_height = (int32_t)it->_height;
            o->bytes_per_pixel = (int32_t)it->_byte_per_pixel;
            o->pixels = it->_buffer;
        } else if (const HDRTexture *h = dynamic_cast<const HDRTexture *>(t)) {
            o->type = RUMI_TEX_HDR;
            o->img_width = h->_width;
            o->img_height = h->_height;
            o->bytes_per_pixel = 12;
            o->pixels = h->_buffer;
        } else {
            return false;
        }
        return true;
    }
};

namespace {

// Material table: one entry per distinct Material object, except that Matte materials of
// triangles are keyed by kd alone -- their colour travels per triangle in tri_albedo, so
// a mesh whose triangles each own a Matte (per-triangle albedo) needs one table entry.
struct MaterialTable {
    std::vector<rumi_material> *out;
    std::map<const Material *, int> by_ptr;
    std::map<float, int> matte_by_kd;
    int add(const Material *m, bool triangle, float *albedo, std::string *error) {
        rumi_material rm;
        if (!RumiSceneAccess::material(m, &rm)) {
            *error = "unsupported Material subclass";
            return -1;
        }
        if (albedo) memcpy(albedo, rm.rgb, sizeof(rm.rgb));
        if (triangle && rm.type == RUMI_MAT_MATTE) {
            auto it = matte_by_kd.find(rm.kd);
            if (it != matte_by_kd.end()) return it->second;
            rm.rgb[0] = rm.rgb[1] = rm.rgb[2] = 1.0f;
            out->push_back(rm);
            return matte_by_kd[rm.kd] = (int)out->size() - 1;
        }
        auto it = by_ptr.find(m);
        if (it != by_ptr.end()) return it->second;
        out->push_back(rm);
        return by_ptr[m] = (int)out->size() - 1;
    }
};

}  // namespace

bool RumiFlattenScene(const Scene *scene, RumiFlatScene *out, std::string *error) {
    RumiFlatScene &f = *out;
    f = RumiFlatScene();
    if (!scene || !scene->_image || !scene->_camera) {
        *error = "scene without film or camera";
        return false;
    }
    MaterialTable mats{&f.materials, {}, {}};
    std::map<const Texture *, int> tex_index;
    bool any_texture = false;
    auto tex_of = [&](const Shape *s) -> int {
        const Texture *t = s->TexturePtr();
        if (!t) return -1;
        auto it = tex_index.find(t);
        if (it != tex_index.end()) return it->second;
        rumi_texture rt;
        if (!RumiSceneAccess::texture(t, &rt)) return -2;
        f.textures.push_back(rt);
        any_texture = true;
        return tex_index[t] = (int)f.textures.size() - 1;
    };
    std::map<const Shape *, std::pair<int, int>> where;  // shape -> (kind, index)

    auto add_triangle = [&](const Triangle *t) -> bool {
        float v[9], n[9], alb[3];
        RumiSceneAccess::triangle(t, v, n);
        const Material *m = t->MaterialPtr();
        if (!m) { *error = "triangle without a material"; return false; }
        const int mi = mats.add(m, true, alb, error);
        const int ti = tex_of(t);
        if (mi < 0) return false;
        if (ti == -2) { *error = "unsupported Texture subclass"; return false; }
        f.tri_vertices.insert(f.tri_vertices.end(), v, v + 9);
        f.tri_normals.insert(f.tri_normals.end(), n, n + 9);
        f.tri_albedo.insert(f.tri_albedo.end(), alb, alb + 3);
        f.tri_material.push_back(mi);
        f.tri_texture.push_back(ti);
        return true;
    };

    // primitive order inside each array follows _objects (canonical ids: triangles,
    // rects, spheres)
    const int n_obj = scene->ObjectCount();
    for (int i = 0; i < n_obj; ++i) {
        const Shape *s = scene->_objects[i];
        if (const Triangle *t = dynamic_cast<const Triangle *>(s)) {
            where[s] = {RUMI_SHAPE_TRIANGLE, (int)f.tri_material.size()};
            if (!add_triangle(t)) return false;
        } else if (const Model *m = dynamic_cast<const Model *>(s)) {
            where[s] = {RUMI_SHAPE_TRIANGLE, (int)f.tri_material.size()};
            for (int k = 0; k < RumiSceneAccess::model_count(m); ++k)
                if (!add_triangle(RumiSceneAccess::model_triangle(m, k))) return false;
        } else if (const Rect *r = dynamic_cast<const Rect *>(s)) {
            where[s] = {RUMI_SHAPE_RECT, (int)f.rect_material.size()};
            float o[9];
            RumiSceneAccess::rect(r, o);
            if (!s->MaterialPtr()) { *error = "rect without a material"; return false; }
            const int mi = mats.add(s->MaterialPtr(), false, nullptr, error);
            const int ti = tex_of(s);
            if (mi < 0) return false;
            if (ti == -2) { *error = "unsupported Texture subclass"; return false; }
            f.rects.insert(f.rects.end(), o, o + 9);
            f.rect_material.push_back(mi);
            f.rect_texture.push_back(ti);
        } else if (const Sphere *sp = dynamic_cast<const Sphere *>(s)) {
            where[s] = {RUMI_SHAPE_SPHERE, (int)f.sphere_material.size()};
            float o[4];
            RumiSceneAccess::sphere(sp, o);
            if (!s->MaterialPtr()) { *error = "sphere without a material"; return false; }
            const int mi = mats.add(s->MaterialPtr(), false, nullptr, error);
            const int ti = tex_of(s);
            if (mi < 0) return false;
            if (ti == -2) { *error = "unsupported Texture subclass"; return false; }
            f.spheres.insert(f.spheres.end(), o, o + 4);
            f.sphere_material.push_back(mi);
            f.sphere_texture.push_back(ti);
            // rows 0-2 of the upper 3x3 of Shape::_transform orient a sphere's texture
            const float *tm = s->_transform._m;
            const float fr[9] = {tm[0], tm[1], tm[2], tm[4], tm[5], tm[6], tm[8], tm[9], tm[10]};
            f.sphere_frame.insert(f.sphere_frame.end(), fr, fr + 9);
        } else {
            *error = "unsupported Shape subclass in Scene::_objects";
            return false;
        }
    }

    const int n_lights = scene->LightCount();
    for (int i = 0; i < n_lights; ++i) {
        const Light *l = scene->_lights[i];
        rumi_light rl;
        memset(&rl, 0, sizeof(rl));
        const Shape *shape = nullptr;
        if (const AreaLight *al = dynamic_cast<const AreaLight *>(l)) {
            rl.type = RUMI_LIGHT_AREA;
            shape = RumiSceneAccess::area_light_shape(al);
        } else if (const ImageBasedLight *il = dynamic_cast<const ImageBasedLight *>(l)) {
            rl.type = RUMI_LIGHT_IBL;
            shape = RumiSceneAccess::ibl_shape(il);
        } else {
            *error = "unsupported Light subclass in Scene::_lights (area and image-based lights only)";
            return false;
        }
        auto it = where.find(shape);
        if (it == where.end() || it->second.first == RUMI_SHAPE_TRIANGLE) {
            *error = "light over a shape that is not a Rect or Sphere of Scene::_objects";
            return false;
        }
        rl.shape_type = it->second.first;
        rl.shape_index = it->second.second;
        f.lights.push_back(rl);
    }

    rumi_scene_desc &d = f.desc;
    memset(&d, 0, sizeof(d));
    d.width = scene->_image->Width();
    d.height = scene->_image->Height();
    d.n_triangles = (int32_t)f.tri_material.size();
    d.tri_vertices = f.tri_vertices.data();
    d.tri_normals = f.tri_normals.data();
    d.tri_material = f.tri_material.data();
    d.tri_albedo = f.tri_albedo.data();
    d.n_rects = (int32_t)f.rect_material.size();
    d.rects = f.rects.data();
    d.rect_material = f.rect_material.data();
    d.n_spheres = (int32_t)f.sphere_material.size();
    d.spheres = f.spheres.data();
    d.sphere_material = f.sphere_material.data();
    d.n_materials = (int32_t)f.materials.size();
    d.materials = f.materials.data();
    d.n_lights = (int32_t)f.lights.size();
    d.lights = f.lights.data();
    if (scene->_volume_ptr) RumiSceneAccess::volume(scene->_volume_ptr, &d.volume);
    const Pinhole *cam = scene->_camera;
    RumiSceneAccess::put3(d.camera.position, cam->_p);
    memcpy(d.camera.basis, cam->_basis_transform._m, sizeof(d.camera.basis));
    d.camera.y_ratio = cam->_y_ratio;
    d.camera.fov_deg = cam->_fov;
    d.camera.focal_distance = cam->_focal_distance;
    d.camera.lens_radius = cam->_lens_radius;
    if (any_texture) {
        d.n_textures = (int32_t)f.textures.size();
        d.textures = f.textures.data();
        d.tri_texture = f.tri_texture.data();
        d.rect_texture = f.rect_texture.data();
        d.sphere_texture = f.sphere_texture.data();
        d.sphere_frame = f.sphere_frame.data();
    }
    return true;
}

// ------------------------------------------------------------------ frames
RumiGpuFrame::~RumiGpuFrame() {
    if (_gpu) rumi_scene_destroy(_gpu);
}

bool RumiGpuFrame::Render(Scene *scene, rumi_render_params params, Film *film) {
    if (!_gpu) {
        RumiFlatScene flat;
        std::string err;
        if (!RumiFlattenScene(scene, &flat, &err)) {
            _error = "RumiFlattenScene: " + err;
            return false;
        }
        if (rumi_scene_create(&flat.desc, &_gpu) != RUMI_OK) {
            _error = std::string("rumi_scene_create: ") + rumi_last_error_string();
            _gpu = nullptr;
            return false;
        }
    }
    _width = (unsigned int)film->Width();
    _height = (unsigned int)film->Height();
    _spp = film->PixelSampler() ? film->PixelSampler()->SampleCount() : 0;
    if (_spp == 0) {
        _error = "film without a pixel sampler";
        return false;
    }
    params.spp = (int32_t)_spp;
    params.seed = next_seed++;
    _frame.assign((size_t)_width * _height * 3, 0.0f);
    if (rumi_render(_gpu, &params, _frame.data(), 0, nullptr) != RUMI_OK) {
        _error = std::string("rumi_render: ") + rumi_last_error_string();
        return false;
    }
    _calls_left = (unsigned long long)_width * _height * _spp;
    return true;
}

Color RumiGpuFrame::Sample(Scene *scene, const rumi_render_params &params, unsigned int w, unsigned int h,
                           Film *film) {
    if (!_error.empty()) return Color(0.0f);
    if (_calls_left == 0 && !Render(scene, params, film)) {
        if (!_reported) {
            fprintf(stderr, "GPU integrator: %s\n", _error.c_str());
            _reported = true;
        }
        return Color(0.0f);
    }
    --_calls_left;
    if (w >= _width || h >= _height) return Color(0.0f);
    const float *p = &_frame[((size_t)h * _width + w) * 3];  // B, G, R sums
    const float inv = 1.0f / (float)_spp;
    return Color(p[2] * inv, p[1] * inv, p[0] * inv);  // Color(r, g, b)
}

GpuPathTracer::GpuPathTracer(Scene *scene_ptr, int max_depth) : Integrator(scene_ptr), _max_depth(max_depth) {}
GpuPathTracer::~GpuPathTracer() {}

Color GpuPathTracer::Trace(const unsigned int &width_idx, const unsigned int &height_idx, Pinhole *, Film *image_ptr) {
    rumi_render_params p;
    memset(&p, 0, sizeof(p));
    p.integrator = RUMI_PATH_TRACER;
    p.max_depth = _max_depth;
    return frame.Sample(_scene_ptr, p, width_idx, height_idx, image_ptr);
}

GpuRayTracer::GpuRayTracer(Scene *scene_ptr, int max_depth) : Integrator(scene_ptr), _max_depth(max_depth) {}
GpuRayTracer::~GpuRayTracer() {}

Color GpuRayTracer::Trace(const unsigned int &width_idx, const unsigned int &height_idx, Pinhole *, Film *image_ptr) {
    rumi_render_params p;
    memset(&p, 0, sizeof(p));
    p.integrator = RUMI_RAY_TRACER;
    p.max_depth = _max_depth;
    return frame.Sample(_scene_ptr, p, width_idx, height_idx, image_ptr);
}

GpuBDPT::GpuBDPT(Scene *scene_ptr, int nL, int nE) : Integrator(scene_ptr), _nL(nL), _nE(nE) {
    if (scene_ptr && scene_ptr->_camera) scene_ptr->_camera->DepthOfField(0.0f, 0.0f);
}
GpuBDPT::~GpuBDPT() {}

Color GpuBDPT::Trace(const unsigned int &width_idx, const unsigned int &height_idx, Pinhole *, Film *image_ptr) {
    rumi_render_params p;
    memset(&p, 0, sizeof(p));
    p.integrator = RUMI_BDPT;
    p.n_light = _nL;
    p.n_eye = _nE;
    p.max_depth = _nL + _nE;
    return frame.Sample(_scene_ptr, p, width_idx, height_idx, image_ptr);
}
