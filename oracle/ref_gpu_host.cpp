// Test host for the reference-side adapter (rumi-renderer_b200/adapter/): runs the
// reference's own frame loop, Scene::Rendering (src/Scene/scene.cpp:206-258), on a Scene
// built through the reference's classes by ref_harness.cpp, with GpuPathTracer or GpuBDPT
// installed as Scene::_tracer_ptr in place of the CPU integrator.
// TEST INFRASTRUCTURE ONLY: built by oracle/build_ref.py into
// oracle/_ref/librumi_ref_gpuhost.so, linked with the reference build and librumi_b200.so.
#include <cstring>
#include <string>

#include "Camera/film.h"
#include "Integrator/integrator.h"
#include "Scene/scene.h"
#include "rumi_gpu_integrators.h"

// integrator 0: GpuPathTracer(scene, a); 1: GpuBDPT(scene, a, b); 2: GpuRayTracer(scene, a).  `frames` calls of
// Scene::Rendering in a row (each renders into a cleared film; the adapter advances its
// seed per frame, starting at `seed`).  film_out (frames*H*W*3, B,G,R) receives each
// frame's Film::_pixel_buffer.  Returns 0, or -1 with the adapter's error in err.
// Scene::Rendering ends with Film::Save, which writes "<seconds>s.bmp" into the working
// directory.
extern "C" int ref_gpu_rendering(void *scene_ptr, int integrator, int a, int b, unsigned long long seed, int frames,
                                 float *film_out, char *err, int err_len) {
    Scene *sc = (Scene *)scene_ptr;
    Film *film = sc->_image;
    Integrator *cpu = sc->_tracer_ptr;
    RumiGpuFrame *state = nullptr;
    Integrator *gpu = nullptr;
    if (integrator == 0) {
        GpuPathTracer *t = new GpuPathTracer(sc, a);
        state = &t->frame;
        gpu = t;
    } else if (integrator == 2) {
        GpuRayTracer *t = new GpuRayTracer(sc, a);
        state = &t->frame;
        gpu = t;
    } else {
        GpuBDPT *t = new GpuBDPT(sc, a, b);
        state = &t->frame;
        gpu = t;
    }
    state->next_seed = seed;
    sc->_tracer_ptr = gpu;
    const size_t n = (size_t)film->Width() * film->Height() * 3;
    for (int f = 0; f < frames; ++f) {
        memset(film->_pixel_buffer, 0, sizeof(float) * n);
        if (film->_light_buffer) memset(film->_light_buffer, 0, sizeof(float) * n);
        float seconds = 0.0f;
        sc->Rendering(&seconds);
        memcpy(film_out + n * (size_t)f, film->_pixel_buffer, sizeof(float) * n);
    }
    const bool ok = state->Ok();
    if (!ok && err && err_len > 0) {
        strncpy(err, state->LastError().c_str(), (size_t)err_len - 1);
        err[err_len - 1] = 0;
    }
    sc->_tracer_ptr = cpu;
    delete gpu;
    return ok ? 0 : -1;
}

// RumiFlattenScene on the reference Scene.  counts[0..4] receive the numbers of
// triangles, rects, spheres, materials and lights; every non-NULL buffer receives the
// matching descriptor array (sizes from a first call with NULL buffers).  camera and
// volume receive the rumi_camera / rumi_volume.  Returns 0, or -1 with the error in err.
extern "C" int ref_gpu_flatten(void *scene_ptr, int *counts, float *tri_v, float *tri_n, float *tri_alb, int *tri_mat,
                               float *rects, int *rect_mat, float *spheres, int *sphere_mat, rumi_material *mats,
                               rumi_light *lights, rumi_camera *camera, rumi_volume *volume, char *err,
                               int err_len) {
    RumiFlatScene f;
    std::string e;
    if (!RumiFlattenScene((const Scene *)scene_ptr, &f, &e)) {
        if (err && err_len > 0) {
            strncpy(err, e.c_str(), (size_t)err_len - 1);
            err[err_len - 1] = 0;
        }
        return -1;
    }
    const rumi_scene_desc &d = f.desc;
    counts[0] = d.n_triangles;
    counts[1] = d.n_rects;
    counts[2] = d.n_spheres;
    counts[3] = d.n_materials;
    counts[4] = d.n_lights;
    auto cp = [](void *dst, const void *src, size_t bytes) {
        if (dst && bytes) memcpy(dst, src, bytes);
    };
    cp(tri_v, d.tri_vertices, sizeof(float) * 9 * d.n_triangles);
    cp(tri_n, d.tri_normals, sizeof(float) * 9 * d.n_triangles);
    cp(tri_alb, d.tri_albedo, sizeof(float) * 3 * d.n_triangles);
    cp(tri_mat, d.tri_material, sizeof(int) * d.n_triangles);
    cp(rects, d.rects, sizeof(float) * 9 * d.n_rects);
    cp(rect_mat, d.rect_material, sizeof(int) * d.n_rects);
    cp(spheres, d.spheres, sizeof(float) * 4 * d.n_spheres);
    cp(sphere_mat, d.sphere_material, sizeof(int) * d.n_spheres);
    cp(mats, d.materials, sizeof(rumi_material) * d.n_materials);
    cp(lights, d.lights, sizeof(rumi_light) * d.n_lights);
    cp(camera, &d.camera, sizeof(rumi_camera));
    cp(volume, &d.volume, sizeof(rumi_volume));
    return 0;
}
