// Device-side basics shared by every kernel of the renderer: float3 helpers, the
// counter-based Philox4x32-10 generator, ordered-int float atomics and constants.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <cfloat>

#define RUMI_HD __host__ __device__ __forceinline__
#define RUMI_D __device__ __forceinline__
#ifdef __CUDACC__
#define RUMI_NOINLINE __noinline__
#else  // a host compiler building device code as plain C++
#define RUMI_NOINLINE __attribute__((noinline))
#endif

// The reference's epsilon for self-intersection and the light end of shadow rays
// (src/Kernel/ray.cpp:4).
#define RUMI_EPS 1e-4f
#define RUMI_PI_F 3.14159265358979323846f
#define RUMI_INV_PI_F 0.3183098865475128f

// ------------------------------------------------------------------------- float3
RUMI_HD float3 mk3(float x, float y, float z) { return make_float3(x, y, z); }
RUMI_HD float3 operator+(float3 a, float3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
RUMI_HD float3 operator-(float3 a, float3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
RUMI_HD float3 operator-(float3 a) { return mk3(-a.x, -a.y, -a.z); }
RUMI_HD float3 operator*(float3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
RUMI_HD float3 operator*(float3 a, float3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
RUMI_HD float3 operator/(float3 a, float3 b) { return mk3(a.x / b.x, a.y / b.y, a.z / b.z); }
RUMI_HD float3 operator/(float3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
RUMI_HD float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RUMI_HD float3 cross3(float3 u, float3 v) {
    return mk3(u.y * v.z - v.y * u.z, u.z * v.x - v.z * u.x, u.x * v.y - v.x * u.y);
}
// Average(Color) of the reference: (b + g + r) * 0.33333333333f (src/Kernel/color.h).  A
// float3 colour holds (r, g, b) in (x, y, z).
RUMI_HD float avg3(float3 c) { return (c.z + c.y + c.x) * 0.33333333333f; }
RUMI_HD float3 f4xyz(float4 a) { return mk3(a.x, a.y, a.z); }
RUMI_HD bool any_nan3(float3 c) { return c.x != c.x || c.y != c.y || c.z != c.z; }

// Normalize as the reference does: 1 / sqrtf(len2), then three products
// (src/Kernel/vector.h:43-55).
RUMI_D float3 normalize_ref(float3 v) {
    float inv = __frcp_rn(__fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y)),
                                                __fmul_rn(v.z, v.z))));
    return mk3(__fmul_rn(v.x, inv), __fmul_rn(v.y, inv), __fmul_rn(v.z, inv));
}

// ------------------------------------------------------- correctly rounded helpers
// Used where results must match the reference's x86 float arithmetic bit for bit
// (primitive intersection): no FMA contraction, IEEE rounding on every operation.
RUMI_D float rn_dot(float3 a, float3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
RUMI_D float3 rn_cross(float3 u, float3 v) {
    return mk3(__fsub_rn(__fmul_rn(u.y, v.z), __fmul_rn(v.y, u.z)),
               __fsub_rn(__fmul_rn(u.z, v.x), __fmul_rn(v.z, u.x)),
               __fsub_rn(__fmul_rn(u.x, v.y), __fmul_rn(v.x, u.y)));
}
RUMI_D float3 rn_sub(float3 a, float3 b) {
    return mk3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}
RUMI_D float3 rn_madd(float3 o, float3 d, float t) {  // o + d * t, two roundings per lane
    return mk3(__fadd_rn(o.x, __fmul_rn(d.x, t)), __fadd_rn(o.y, __fmul_rn(d.y, t)),
               __fadd_rn(o.z, __fmul_rn(d.z, t)));
}

// n0 (1 - u - v) + n1 u + n2 v, one rounding per operation in that order (the shading
// normal of Triangle::Intersect, triangle.cpp:111).  The last bit matters: the
// reference's tangent frame takes a special branch only for normals of exactly
// (0, +-1, 0), and the two branches mirror the sampled directions about the frame.
RUMI_D float3 bary_ref(float3 n0, float3 n1, float3 n2, float u, float v) {
    const float w = __fsub_rn(__fsub_rn(1.0f, u), v);
    return mk3(__fadd_rn(__fadd_rn(__fmul_rn(n0.x, w), __fmul_rn(n1.x, u)), __fmul_rn(n2.x, v)),
               __fadd_rn(__fadd_rn(__fmul_rn(n0.y, w), __fmul_rn(n1.y, u)), __fmul_rn(n2.y, v)),
               __fadd_rn(__fadd_rn(__fmul_rn(n0.z, w), __fmul_rn(n1.z, u)), __fmul_rn(n2.z, v)));
}

// ------------------------------------------------------------- Philox4x32-10
// Counter-based generator of Salmon, Moraes, Dror and Shaw, "Parallel random numbers:
// as easy as 1, 2, 3" (SC 2011): 10 rounds of two 32x32->64 multiplies with a Weyl key
// schedule.  One call maps (counter, key) to four independent 32-bit words.
struct Philox4 {
    uint32_t v[4];
};

RUMI_HD void philox_round(uint32_t &c0, uint32_t &c1, uint32_t &c2, uint32_t &c3, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    uint64_t p0 = (uint64_t)M0 * c0;
    uint64_t p1 = (uint64_t)M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    uint32_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
}

RUMI_HD Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        philox_round(c0, c1, c2, c3, k0, k1);
        k0 += W0;
        k1 += W1;
    }
    Philox4 o;
    o.v[0] = c0; o.v[1] = c1; o.v[2] = c2; o.v[3] = c3;
    return o;
}

// 24-bit uniform in [0, 1): m * 2^-24.
RUMI_HD float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

struct Uniform4 {
    float u[4];
};

// Stream layout of one path: counter = (path index lo, path index hi, bounce, group).
RUMI_HD Uniform4 path_uniforms(uint64_t path, uint32_t bounce, uint32_t group, uint32_t k0, uint32_t k1) {
    Philox4 r = philox4x32_10((uint32_t)path, (uint32_t)(path >> 32), bounce, group, k0, k1);
    Uniform4 o;
    o.u[0] = u01(r.v[0]); o.u[1] = u01(r.v[1]); o.u[2] = u01(r.v[2]); o.u[3] = u01(r.v[3]);
    return o;
}

// ------------------------------------------------------- ordered-int float atomics
// Monotone map float -> int so integer atomicMin/atomicMax order floats correctly.
RUMI_HD int f2o(float f) {
#ifdef __CUDA_ARCH__
    int i = __float_as_int(f);
#else
    union { float f; int i; } u; u.f = f; int i = u.i;
#endif
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
RUMI_HD float o2f(int i) {
    int b = i >= 0 ? i : i ^ 0x7FFFFFFF;
#ifdef __CUDA_ARCH__
    return __int_as_float(b);
#else
    union { float f; int i; } u; u.i = b; return u.f;
#endif
}

// Warp-aggregated queue push: every active lane with want=true gets a unique slot.
RUMI_D int warp_push(int *counter, bool want) {
    unsigned mask = __activemask();
    unsigned ballot = __ballot_sync(mask, want);
    int leader = __ffs(mask) - 1;
    int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == leader && ballot) base = atomicAdd(counter, __popc(ballot));
    base = __shfl_sync(mask, base, leader);
    return want ? base + __popc(ballot & ((1u << lane) - 1u)) : -1;
}
