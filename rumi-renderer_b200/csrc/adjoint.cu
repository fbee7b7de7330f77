// Path-replay adjoint of the path tracer (rumi_forward / rumi_backward in
// include/rumi_b200.h) and the parameter updates an optimiser needs between steps
// (rumi_scene_set_albedo, rumi_scene_set_volume).  The kernels live in pt.cu
// (pt_shade<true>, pt_shadow<0, true>, pt_backward).
#include "renderer.h"

using namespace rumi;

extern "C" {

rumi_status rumi_forward(rumi_scene *sc, const rumi_render_params *p, float *film, int32_t film_on_device,
                         rumi_render_stats *stats) {
    if (p && p->integrator != RUMI_PATH_TRACER) {
        set_error("rumi_forward: the adjoint covers the path tracer only");
        return RUMI_ERR_INVALID_ARG;
    }
    if (!sc || !p || !(p->flags & RUMI_FLAG_KEEP_RADIANCE)) {
        if (sc) sc->kept_valid = false;
        return rumi_render(sc, p, film, film_on_device, stats);
    }
    // RUMI_FLAG_KEEP_RADIANCE: the frame's per-path radiance stays on the device for
    // rumi_backward (16 bytes per path)
    sc->kept_valid = false;
    if (!film || p->spp <= 0 || p->max_depth <= 0) return rumi_render(sc, p, film, film_on_device, stats);
    cudaStream_t s = p->stream ? (cudaStream_t)p->stream : sc->stream;
    const long long n = (long long)sc->dev.width * sc->dev.height * p->spp;
    if (sc->kept_cap < n) {
        dfree(sc->kept_L, s);
        sc->kept_L = nullptr;
        sc->kept_cap = 0;
        cudaError_t e = dalloc((void **)&sc->kept_L, sizeof(float4) * (size_t)n, s);
        if (e != cudaSuccess) return cuda_status(e, "rumi_forward: kept radiance");
        sc->kept_cap = n;
    }
    const size_t film_bytes = sizeof(float) * 3 * (size_t)sc->dev.width * sc->dev.height;
    float *film_dev = film, *tmp = nullptr;
    if (!film_on_device) {
        cudaError_t e = dalloc((void **)&tmp, film_bytes, s);
        if (e != cudaSuccess) return cuda_status(e, "device allocation (film)");
        film_dev = tmp;
    }
    rumi_status st = pt_render(sc, p, film_dev, stats, s, sc->kept_L);
    if (st == RUMI_OK && !film_on_device) {
        cudaError_t e = cudaMemcpyAsync(film, film_dev, film_bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_status(e, "film copy");
    }
    dfree(tmp, s);
    if (st == RUMI_OK) {
        sc->kept_valid = true;
        sc->kept_seed = p->seed;
        sc->kept_spp = p->spp;
        sc->kept_depth = p->max_depth;
    }
    return st;
}

rumi_status rumi_backward(rumi_scene *sc, const rumi_render_params *p, const float *d_film, float *grad_albedo,
                          float *grad_volume, int32_t on_device, rumi_render_stats *stats) {
    if (!sc || !p || !d_film) {
        set_error("rumi_backward: NULL argument");
        return RUMI_ERR_INVALID_ARG;
    }
    if (p->integrator != RUMI_PATH_TRACER) {
        set_error("rumi_backward: the adjoint covers the path tracer only");
        return RUMI_ERR_INVALID_ARG;
    }
    if (p->spp <= 0 || p->max_depth <= 0) {
        set_error("rumi_backward: spp and max_depth must be positive");
        return RUMI_ERR_INVALID_ARG;
    }
    if (grad_albedo && !sc->tri_albedo) {
        set_error("rumi_backward: the scene has no per-triangle albedo to differentiate");
        return RUMI_ERR_INVALID_ARG;
    }
    if (grad_volume && !sc->dev.volume.present) {
        set_error("rumi_backward: the scene has no medium to differentiate");
        return RUMI_ERR_INVALID_ARG;
    }
    cudaStream_t s = p->stream ? (cudaStream_t)p->stream : sc->stream;
    const size_t film_bytes = sizeof(float) * 3 * (size_t)sc->dev.width * sc->dev.height;
    const size_t alb_bytes = sizeof(float) * 3 * (size_t)sc->dev.n_tris;
    const size_t vol_bytes = sizeof(float) * 7;
    const float *df = d_film;
    float *ga = grad_albedo, *gv = grad_volume;
    float *t_df = nullptr, *t_ga = nullptr, *t_gv = nullptr;
    cudaError_t e = cudaSuccess;
    if (!on_device) {
        e = dalloc((void **)&t_df, film_bytes, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(t_df, d_film, film_bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && grad_albedo) e = dalloc((void **)&t_ga, alb_bytes, s);
        if (e == cudaSuccess && grad_volume) e = dalloc((void **)&t_gv, vol_bytes, s);
        df = t_df;
        ga = t_ga;
        gv = t_gv;
    }
    rumi_status st = e == cudaSuccess ? RUMI_OK : cuda_status(e, "rumi_backward buffers");
    if (st == RUMI_OK) st = pt_backward(sc, p, df, ga, gv, stats, s);
    if (st == RUMI_OK && !on_device) {
        if (grad_albedo) e = cudaMemcpyAsync(grad_albedo, t_ga, alb_bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && grad_volume) e = cudaMemcpyAsync(grad_volume, t_gv, vol_bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_status(e, "rumi_backward copy");
    }
    dfree(t_df, s);
    dfree(t_ga, s);
    dfree(t_gv, s);
    return st;
}

rumi_status rumi_scene_set_albedo(rumi_scene *sc, const float *albedo, int32_t on_device) {
    if (!sc || !albedo) {
        set_error("rumi_scene_set_albedo: NULL argument");
        return RUMI_ERR_INVALID_ARG;
    }
    sc->kept_valid = false;  // a kept forward radiance no longer describes the scene
    if (!sc->tri_albedo) {
        set_error("rumi_scene_set_albedo: the scene was created without per-triangle albedo");
        return RUMI_ERR_INVALID_ARG;
    }
    const int n = sc->dev.n_tris;
    const size_t bytes = sizeof(float) * 3 * (size_t)n;
    cudaStream_t s = sc->stream;
    const float *src = albedo;
    float *tmp = nullptr;
    cudaError_t e = cudaSuccess;
    if (!on_device) {
        e = dalloc((void **)&tmp, bytes, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(tmp, albedo, bytes, cudaMemcpyHostToDevice, s);
        src = tmp;
    }
    if (e == cudaSuccess) pack_albedo(src, n, sc->tri_albedo, s);
    if (e == cudaSuccess) e = cudaGetLastError();
    dfree(tmp, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? RUMI_OK : cuda_status(e, "rumi_scene_set_albedo");
}

rumi_status rumi_scene_set_volume(rumi_scene *sc, const rumi_volume *v) {
    if (sc) sc->kept_valid = false;  // a kept forward radiance no longer describes the scene
    if (!sc || !v) {
        set_error("rumi_scene_set_volume: NULL argument");
        return RUMI_ERR_INVALID_ARG;
    }
    if (v->present) {
        for (int c = 0; c < 3; ++c) {
            if (!(v->sigma_s[c] >= 0.0f) || !(v->sigma_a[c] >= 0.0f) || !(v->sigma_s[c] + v->sigma_a[c] > 0.0f)) {
                set_error("rumi_scene_set_volume: coefficients must be >= 0 with positive extinction");
                return RUMI_ERR_INVALID_ARG;
            }
        }
        if (!(v->g > -1.0f && v->g < 1.0f)) {
            set_error("rumi_scene_set_volume: g must lie in (-1, 1)");
            return RUMI_ERR_INVALID_ARG;
        }
    }
    DevVolume dv{};
    if (v->present) fill_dev_volume(dv, *v);
    sc->dev.volume = dv;
    return RUMI_OK;
}

}  // extern "C"
