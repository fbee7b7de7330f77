// Camera rays and the per-pixel sample positions of the renderer.
#pragma once
#include "scene.cuh"

namespace rumi {

// ------------------------------------------------------------- pixel samples
// Keyed bijection on [0, n): balanced Feistel network on the next even bit width with
// cycle walking.
RUMI_D uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return x;
}

RUMI_HD int perm_index(int i, int n, uint32_t key) {
    if (n <= 1) return 0;
    int bits = 0;
    while ((1 << bits) < n) ++bits;
    if (bits & 1) ++bits;
    if (bits < 2) bits = 2;
    const int half = bits >> 1;
    const uint32_t mask = (1u << half) - 1u;
    uint32_t x = (uint32_t)i;
    for (int walk = 0; walk < 4096; ++walk) {
        uint32_t Lh = x >> half, R = x & mask;
        for (int r = 0; r < 4; ++r) {
#ifdef __CUDA_ARCH__
            const uint32_t F = mix32(R ^ (key + 0x9E3779B9u * (uint32_t)(r + 1))) & mask;
#else
            uint32_t y = R ^ (key + 0x9E3779B9u * (uint32_t)(r + 1));
            y ^= y >> 16; y *= 0x7FEB352Du; y ^= y >> 15; y *= 0x846CA68Bu; y ^= y >> 16;
            const uint32_t F = y & mask;
#endif
            const uint32_t nl = R;
            R = Lh ^ F;
            Lh = nl;
        }
        x = (Lh << half) | R;
        if ((int)x < n) return (int)x;
    }
    return i;  // unreachable for a permutation; keeps the loop bounded
}

// The reference's pixel sampler (src/Sample/uniformsample.cpp:32-58, sampler.cpp:17-38):
// one jittered sqrt(n) x sqrt(n) grid per frame shared by all pixels; each pixel draws
// its n samples' x and y coordinates independently without replacement.  Here the two
// draws are keyed permutations of the grid per pixel.  Non-square counts use n strata
// per axis.
RUMI_D float2 pixel_sample(int s, int spp, int grid_d, bool square, long long pixel, uint32_t k0, uint32_t k1) {
    const uint32_t pk = (uint32_t)pixel * 0x9E3779B1u ^ (uint32_t)(pixel >> 32);
    const int kx = perm_index(s, spp, mix32(pk ^ k0) ^ 0x68E31DA4u);
    const int ky = perm_index(s, spp, mix32(pk ^ k1) ^ 0xB5297A4Du);
    const Philox4 jx = philox4x32_10((uint32_t)kx, 0u, 0xFFFFFFFFu, 0u, k0, k1);
    const Philox4 jy = philox4x32_10((uint32_t)ky, 0u, 0xFFFFFFFFu, 0u, k0, k1);
    // correctly rounded operations in source order: no contraction into the caller's
    // arithmetic, so every inlined copy yields the same bits
    float2 r;
    if (square) {
        const float normalize = __fdiv_rn(1.0f, (float)grid_d);
        r.x = __fmul_rn(__fadd_rn((float)(kx % grid_d), u01(jx.v[0])), normalize);
        r.y = __fmul_rn(__fadd_rn((float)(ky / grid_d), u01(jy.v[1])), normalize);
    } else {
        const float normalize = __fdiv_rn(1.0f, (float)spp);
        r.x = __fmul_rn(__fadd_rn((float)kx, u01(jx.v[0])), normalize);
        r.y = __fmul_rn(__fadd_rn((float)ky, u01(jy.v[1])), normalize);
    }
    return r;
}

// Pinhole::CastViewRay (src/Camera/pinhole.cpp:97-136).  With a focal distance set
// (Pinhole::DepthOfField, pinhole.cpp:88-95) the origin moves to a point of the lens disk,
// radius sqrt(lu1) * lens_radius and angle lu2 * 2 * PI (the product taken in double as
// the reference's PI is a double literal), and the ray aims at the point of the focal
// plane that the pinhole ray reaches.
RUMI_D void camera_ray(const DevCamera &c, int W, int H, int w, int h, float sx, float sy, float lu1, float lu2,
                       float3 &o, float3 &d) {
    // correctly rounded operations in the reference's order (no FMA contraction)
    const float half_w = __fmul_rn((float)W, 0.5f), half_h = __fmul_rn((float)H, 0.5f);
    const float x = -__fmul_rn(__fdiv_rn(__fadd_rn(__fsub_rn((float)w, half_w), sx), half_w), c.tanfov);
    const float y = -__fmul_rn(__fmul_rn(__fdiv_rn(__fadd_rn(__fsub_rn((float)h, half_h), sy), half_h), c.tanfov),
                               c.y_ratio);
    const float3 l = normalize_ref(mk3(x, y, c.plane_dist));
    auto row = [&](int r) {
        return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(c.m[4 * r], l.x), __fmul_rn(c.m[4 * r + 1], l.y)),
                                   __fmul_rn(c.m[4 * r + 2], l.z)),
                         c.m[4 * r + 3]);
    };
    d = mk3(row(0), row(1), row(2));
    o = c.p;
    if (c.focal_distance > 0.0f) {
        const float t = __fdiv_rn(c.focal_distance, l.z);
        const float3 fp = mk3(__fadd_rn(c.p.x, __fmul_rn(d.x, t)), __fadd_rn(c.p.y, __fmul_rn(d.y, t)),
                              __fadd_rn(c.p.z, __fmul_rn(d.z, t)));
        const float r = __fmul_rn(__fsqrt_rn(lu1), c.lens_radius);
        const float theta = (float)__dmul_rn((double)__fmul_rn(lu2, 2.0f), 3.14159265358979323846);
        const float sn = sinf(theta), cs = cosf(theta);
        const float3 a = mk3(__fmul_rn(__fmul_rn(c.up.x, r), sn), __fmul_rn(__fmul_rn(c.up.y, r), sn),
                             __fmul_rn(__fmul_rn(c.up.z, r), sn));
        const float3 b = mk3(__fmul_rn(__fmul_rn(c.right.x, r), cs), __fmul_rn(__fmul_rn(c.right.y, r), cs),
                             __fmul_rn(__fmul_rn(c.right.z, r), cs));
        o = mk3(__fadd_rn(__fadd_rn(c.p.x, a.x), b.x), __fadd_rn(__fadd_rn(c.p.y, a.y), b.y),
                __fadd_rn(__fadd_rn(c.p.z, a.z), b.z));
        d = normalize_ref(mk3(__fsub_rn(fp.x, o.x), __fsub_rn(fp.y, o.y), __fsub_rn(fp.z, o.z)));
    }
}

// The two lens uniforms of a camera ray: their own Philox stream of the path (bounce
// counter 0x7FFFFFFF, which no vertex of a path or subpath uses).
RUMI_D float2 lens_uniforms(uint64_t path, uint32_t k0, uint32_t k1) {
    const Uniform4 u = path_uniforms(path, 0x7FFFFFFFu, 0u, k0, k1);
    return make_float2(u.u[0], u.u[1]);
}

}  // namespace rumi
