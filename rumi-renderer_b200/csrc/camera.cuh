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

// Pinhole::CastViewRay (src/Camera/pinhole.cpp:97-136) without depth of field.
RUMI_D void camera_ray(const DevCamera &c, int W, int H, int w, int h, float sx, float sy, float3 &o, float3 &d) {
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
}

}  // namespace rumi
