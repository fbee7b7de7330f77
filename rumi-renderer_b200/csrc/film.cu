// Film output: the reference's tonemapping of pixel sums into 8-bit pixels (Film::Save,
// src/Camera/film.cpp:152-203) and its fireflies post-filter (FirefliesFiltering,
// src/Scene/scene.cpp:261-432), as one thread per pixel each.
#include "renderer.h"

namespace {

// Film::Save: sum / n -> powf(., 1 / gamma) * 255 -> clamp to [0, 255] -> truncation.
__global__ void tonemap_kernel(const float *__restrict__ film, int W, int H, int bpp, float inv_n, float gamma_c,
                               unsigned char *__restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)W * H) return;
    unsigned char *o = out + i * bpp;
    for (int c = 0; c < 3; ++c) {
        float v = powf(film[3 * i + c] * inv_n, gamma_c) * 255.0f;
        v = v > 255.0f ? 255.0f : (v < 0.0f ? 0.0f : v);
        o[c] = (unsigned char)(unsigned int)v;  // NaN stays NaN through the clamp and converts to 0
    }
    for (int c = 3; c < bpp; ++c) o[c] = 0;
}

// FirefliesFiltering: a pixel with a channel at 255 is replaced by the mean of its
// neighbours unless one of them is white (all three channels at 255).  The reference walks the BMP rows
// bottom-up (row h of its loop is buffer row H - 1 - h), gathers neighbours under its own
// border conditions into a list and averages the first n_copy of them; this kernel takes
// the same steps per pixel.  Where the reference's border conditions reach outside the
// image it reads outside its buffer; here such reads give 0.
__global__ void fireflies_kernel(const unsigned char *__restrict__ src, int W, int H, int bpp,
                                 unsigned char *__restrict__ dst) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)W * H) return;
    const int h_idx = (int)(q / W), w_idx = (int)(q % W);
    const long long total = (long long)W * H * bpp;
    auto rd = [&](long long idx) -> float { return (idx >= 0 && idx < total) ? (float)src[idx] : 0.0f; };
    int n_copy = 8;
    if (w_idx == 0 || h_idx == 0 || w_idx == W - 1 || h_idx == H - 1) {
        n_copy -= 3;
        if (w_idx == 0 && h_idx == 0) n_copy -= 2;
        if (w_idx == 0 && h_idx == H - 1) n_copy -= 2;
        if (w_idx == W - 1 && h_idx == 0) n_copy -= 2;
        if (w_idx == W - 1 && h_idx == H - 1) n_copy -= 2;
    }
    const long long ph = (long long)(H - (h_idx + 1)) * W * bpp, pw = (long long)w_idx * bpp, row = (long long)W * bpp;
    const long long p0 = ph + pw;
    const float tb = rd(p0), tg = rd(p0 + 1), tr = rd(p0 + 2);
    if (tb < 255.0f && tg < 255.0f && tr < 255.0f) {
        dst[p0] = (unsigned char)(int)tb;
        dst[p0 + 1] = (unsigned char)(int)tg;
        dst[p0 + 2] = (unsigned char)(int)tr;
        return;
    }
    float fb[8], fg[8], fr[8];
    int k = 0;
    auto take = [&](long long idx) {
        if (k < 8) {
            fb[k] = rd(idx);
            fg[k] = rd(idx + 1);
            fr[k] = rd(idx + 2);
        }
        ++k;
    };
    if (w_idx != 0) take(p0 - bpp);
    if (w_idx != W - 1) take(p0 + bpp);
    if (h_idx != 0 || w_idx != 0) take(p0 - row - bpp);
    if (h_idx != 0) take(p0 - row);
    if (h_idx != 0 || w_idx != W - 1) take(p0 - row + bpp);
    if (h_idx != H - 1 || w_idx != 0) take(p0 + row - bpp);
    if (h_idx != H - 1) take(p0 + row);
    if (h_idx != H - 1 || w_idx != W - 1) take(p0 + row + bpp);
    bool fireflies = true;
    for (int c = 0; c < n_copy && c < k && c < 8; ++c)
        if (fb[c] == 255.0f && fg[c] == 255.0f && fr[c] == 255.0f) fireflies = false;
    if (!fireflies) {
        dst[p0] = (unsigned char)(int)tb;
        dst[p0 + 1] = (unsigned char)(int)tg;
        dst[p0 + 2] = (unsigned char)(int)tr;
        return;
    }
    float sb = 0.0f, sg = 0.0f, sr = 0.0f;
    for (int c = 0; c < n_copy && c < k && c < 8; ++c) {
        sr = __fadd_rn(sr, fr[c]);
        sg = __fadd_rn(sg, fg[c]);
        sb = __fadd_rn(sb, fb[c]);
    }
    const float s = __fdiv_rn(1.0f, (float)n_copy);
    sr = __fmul_rn(sr, s);
    sg = __fmul_rn(sg, s);
    sb = __fmul_rn(sb, s);
    sr = sr > 255.0f ? 255.0f : (sr < 0.0f ? 0.0f : sr);
    sg = sg > 255.0f ? 255.0f : (sg < 0.0f ? 0.0f : sg);
    sb = sb > 255.0f ? 255.0f : (sb < 0.0f ? 0.0f : sb);
    dst[p0] = (unsigned char)(int)sb;
    dst[p0 + 1] = (unsigned char)(int)sg;
    dst[p0 + 2] = (unsigned char)(int)sr;
}

}  // namespace

using namespace rumi;

extern "C" {

rumi_status rumi_film_tonemap(const float *film, int32_t width, int32_t height, int32_t n_samples, float gamma,
                              int32_t bytes_per_pixel, uint8_t *out, int32_t on_device, void *stream) {
    if (!film || !out || width <= 0 || height <= 0 || n_samples <= 0 || !(gamma > 0.0f) ||
        (bytes_per_pixel != 3 && bytes_per_pixel != 4)) {
        set_error("rumi_film_tonemap: bad argument");
        return RUMI_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t npix = (size_t)width * height;
    const float *f = film;
    uint8_t *o = out;
    float *tf = nullptr;
    uint8_t *to = nullptr;
    cudaError_t e = cudaSuccess;
    if (!on_device) {
        e = dalloc((void **)&tf, npix * 3 * sizeof(float), s);
        if (e == cudaSuccess) e = dalloc((void **)&to, npix * bytes_per_pixel, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(tf, film, npix * 3 * sizeof(float), cudaMemcpyHostToDevice, s);
        f = tf;
        o = to;
    }
    // Film's sampling depth is (int)sqrt((float)n_samples) and Save divides by its square
    const int depth = (int)std::sqrt((float)n_samples);
    const float inv_n = 1.0f / (float)(depth * depth);
    if (e == cudaSuccess) {
        tonemap_kernel<<<(unsigned)((npix + 255) / 256), 256, 0, s>>>(f, width, height, bytes_per_pixel, inv_n,
                                                                     1.0f / gamma, o);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && !on_device) e = cudaMemcpyAsync(out, to, npix * bytes_per_pixel, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dfree(tf, s);
    dfree(to, s);
    return e == cudaSuccess ? RUMI_OK : cuda_status(e, "rumi_film_tonemap");
}

rumi_status rumi_film_fireflies(const uint8_t *in, int32_t width, int32_t height, int32_t bytes_per_pixel,
                                uint8_t *out, int32_t on_device, void *stream) {
    if (!in || !out || in == out || width <= 0 || height <= 0 || (bytes_per_pixel != 3 && bytes_per_pixel != 4)) {
        set_error("rumi_film_fireflies: bad argument (in and out must be distinct buffers)");
        return RUMI_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = (size_t)width * height * bytes_per_pixel;
    const uint8_t *i8 = in;
    uint8_t *o8 = out;
    uint8_t *ti = nullptr, *to = nullptr;
    cudaError_t e = cudaSuccess;
    if (!on_device) {
        e = dalloc((void **)&ti, bytes, s);
        if (e == cudaSuccess) e = dalloc((void **)&to, bytes, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ti, in, bytes, cudaMemcpyHostToDevice, s);
        i8 = ti;
        o8 = to;
    }
    // bytes the filter does not write (a fourth channel) keep the input's value
    if (e == cudaSuccess) e = cudaMemcpyAsync(o8, i8, bytes, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) {
        const size_t npix = (size_t)width * height;
        fireflies_kernel<<<(unsigned)((npix + 255) / 256), 256, 0, s>>>(i8, width, height, bytes_per_pixel, o8);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && !on_device) e = cudaMemcpyAsync(out, to, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dfree(ti, s);
    dfree(to, s);
    return e == cudaSuccess ? RUMI_OK : cuda_status(e, "rumi_film_fireflies");
}

}  // extern "C"
