// rumi_gpu_integrators.h -- reference-side adapter: GPU integrators behind the
// reference's own Integrator interface.
//
// A Rumi-Renderer host program builds its Scene exactly as it does today
// (Scene::Build, src/Scene/scene.cpp:135-204) and installs one of these classes as
// Scene::_tracer_ptr instead of PathTracer / BidirectionalPathTracer.  Its own
// Scene::Rendering loop (src/Scene/scene.cpp:206-258) then renders on the GPU through the
// C-ABI of rumi_b200.h:
//
//   GpuPathTracer(Scene*, int max_depth)  replaces  PathTracer(Scene*, int max_depth)
//                                                    (src/Integrator/pathtracer.h:17)
//   GpuBDPT(Scene*, int nL, int nE)        replaces  BidirectionalPathTracer(Scene*, int nL, int nE)
//                                                    (src/Integrator/bidirectionalpathtracer.h:35)
//
// Both override Integrator::Trace(w, h, camera, film) (src/Integrator/integrator.h:15-28).
// The first call of a frame flattens the Scene (RumiFlattenScene) into a rumi_scene_desc,
// creates the GPU scene and renders the whole frame; every call then returns its pixel's
// sample sum divided by the sample count, so Rendering's own per-pixel accumulation and
// Film::Pixel reproduce the GPU frame in Film::_pixel_buffer.  After width * height *
// SampleCount() calls the frame is used up and the next call renders a new one (the
// Philox seed advances by one per frame).  BDPT light-tracing splats are already folded
// into the GPU film, so Film::LightPixel receives nothing.
//
// Compile this file with the reference's sources (their src/ directory on the include
// path, as the reference's own files include each other) and link it with
// -lrumi_b200 -lcudart.  The flattening reads members the reference keeps private
// (Triangle::_v0 ..., Rect::_p ..., the materials' BSDF parameters, Pinhole, Film,
// HomogeneousVolume, textures); it reaches them through RumiSceneAccess, so each of
// those classes needs the line `friend struct RumiSceneAccess;` (the list of classes is
// in RumiSceneAccess's definition in rumi_gpu_integrators.cpp).
#ifndef RUMI_GPU_INTEGRATORS_H
#define RUMI_GPU_INTEGRATORS_H

#include <string>
#include <vector>

#include "Integrator/integrator.h"
#include "Kernel/color.h"
#include "rumi_b200.h"

class Scene;
class Pinhole;
class Film;

// The arrays a rumi_scene_desc points into, owned together with the descriptor.
struct RumiFlatScene {
    std::vector<float> tri_vertices, tri_normals, tri_albedo;
    std::vector<int32_t> tri_material, tri_texture;
    std::vector<float> rects, spheres, sphere_frame;
    std::vector<int32_t> rect_material, sphere_material, rect_texture, sphere_texture;
    std::vector<rumi_material> materials;
    std::vector<rumi_light> lights;
    std::vector<rumi_texture> textures;
    rumi_scene_desc desc;  // points into the vectors above; valid while this object lives
};

// Walks scene->_objects (Triangle, Rect, Sphere, Model), scene->_lights (AreaLight,
// ImageBasedLight), _volume_ptr, _camera and _image into *out.  Materials are Matte,
// Glossy, Specular, Emissive, Dielectric and Subsurface; textures Checker, ImageTexture
// and HDRTexture.  Returns false with *error set for anything the GPU path does not
// render (another Shape or Light subclass, a shape without a material, a light whose
// shape is not in _objects).
bool RumiFlattenScene(const Scene *scene, RumiFlatScene *out, std::string *error);

// Shared frame logic of the two integrators.
class RumiGpuFrame {
  public:
    ~RumiGpuFrame();
    // The pixel's sum of the current frame / sample count, rendering a new frame first
    // when the previous one is used up.  On an error the message is printed once and
    // black is returned (the reference's Integrator interface has no error channel;
    // Ok() / LastError() report it).
    Color Sample(Scene *scene, const rumi_render_params &params, unsigned int w, unsigned int h, Film *film);
    bool Ok() const { return _error.empty(); }
    const std::string &LastError() const { return _error; }
    uint64_t next_seed = 1;  // Philox seed of the next frame

  private:
    bool Render(Scene *scene, rumi_render_params params, Film *film);
    rumi_scene *_gpu = nullptr;
    std::vector<float> _frame;  // B,G,R sums, Film::_pixel_buffer layout
    unsigned int _width = 0, _height = 0, _spp = 0;
    unsigned long long _calls_left = 0;
    std::string _error;
    bool _reported = false;
};

// Drop-in for PathTracer(Scene *scene_ptr, int max_depth).
class GpuPathTracer : public Integrator {
  public:
    GpuPathTracer(Scene *scene_ptr, int max_depth);
    ~GpuPathTracer();
    using Integrator::Trace;  // the per-ray overload stays the base class's
    Color Trace(const unsigned int &width_idx, const unsigned int &height_idx, Pinhole *camera_ptr,
                Film *image_ptr);
    RumiGpuFrame frame;

  private:
    int _max_depth;
};

// Drop-in for RayTracer(Scene *scene_ptr, int max_depth) (src/Integrator/raytracer.h:14):
// the Whitted integrator, trace depths 0..max_depth.
class GpuRayTracer : public Integrator {
  public:
    GpuRayTracer(Scene *scene_ptr, int max_depth);
    ~GpuRayTracer();
    using Integrator::Trace;
    Color Trace(const unsigned int &width_idx, const unsigned int &height_idx, Pinhole *camera_ptr,
                Film *image_ptr);
    RumiGpuFrame frame;

  private:
    int _max_depth;
};

// Drop-in for BidirectionalPathTracer(Scene *scene_ptr, int nL, int nE).  Like the
// reference's constructor it turns the camera's thin lens off (BDPT renders through the
// pinhole, src/Integrator/bidirectionalpathtracer.cpp:56).
class GpuBDPT : public Integrator {
  public:
    GpuBDPT(Scene *scene_ptr, int nL, int nE);
    ~GpuBDPT();
    using Integrator::Trace;
    Color Trace(const unsigned int &width_idx, const unsigned int &height_idx, Pinhole *camera_ptr,
                Film *image_ptr);
    RumiGpuFrame frame;

  private:
    int _nL, _nE;
};

#endif
