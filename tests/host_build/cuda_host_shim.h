// Host definitions of the CUDA device intrinsics that the BDPT kernel's sources use, so
// that a host compiler (g++) can build the kernel body as plain C++ and run it one sample
// at a time under AddressSanitizer / UndefinedBehaviorSanitizer with every automatic
// variable initialised to a pattern.  Test infrastructure only: results follow the host's
// libm, so the values are not the device's bit for bit; what the build checks is that
// every array access stays in range and nothing reads an uninitialised index.
//
// Single-thread semantics: one emulated thread is one lane of its own warp.
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>
#include <cstring>

#define RUMI_HOST_BUILD 1
// plain inline functions: forcing every device routine inline makes the sanitized build
// take minutes to compile
#undef __forceinline__
#define __forceinline__ inline
#ifndef __launch_bounds__
#define __launch_bounds__(...)
#endif

// Built-in variables of the emulated launch (set by the driver loop before each sample).
struct HostDim {
    unsigned x, y, z;
};
inline HostDim threadIdx = {0, 0, 0}, blockIdx = {0, 0, 0}, blockDim = {1, 1, 1}, gridDim = {1, 1, 1};

template <typename T>
inline T __ldg(const T *p) {
    return *p;
}

inline int __float_as_int(float f) {
    int i;
    memcpy(&i, &f, 4);
    return i;
}
inline float __int_as_float(int i) {
    float f;
    memcpy(&f, &i, 4);
    return f;
}
inline unsigned __float_as_uint(float f) {
    unsigned i;
    memcpy(&i, &f, 4);
    return i;
}
inline float __uint_as_float(unsigned i) {
    float f;
    memcpy(&f, &i, 4);
    return f;
}

// Correctly rounded float and double operations (SSE arithmetic; the build turns FMA
// contraction off).
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fsub_rn(float a, float b) { return a - b; }
inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fdiv_rn(float a, float b) { return a / b; }
inline float __frcp_rn(float a) { return 1.0f / a; }
inline float __fsqrt_rn(float a) { return std::sqrt(a); }
inline double __dadd_rn(double a, double b) { return a + b; }
inline double __dsub_rn(double a, double b) { return a - b; }
inline double __dmul_rn(double a, double b) { return a * b; }
inline double __ddiv_rn(double a, double b) { return a / b; }

inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline int __ffs(int x) { return __builtin_ffs(x); }
inline unsigned __umulhi(unsigned a, unsigned b) { return (unsigned)(((uint64_t)a * b) >> 32); }

// Per-byte inequality: byte k of the result is 0xff when byte k of a and b differ.
inline unsigned __vcmpne4(unsigned a, unsigned b) {
    unsigned r = 0;
    for (int k = 0; k < 4; ++k)
        if (((a >> (8 * k)) & 0xffu) != ((b >> (8 * k)) & 0xffu)) r |= 0xffu << (8 * k);
    return r;
}
// Byte k of the result is byte (s >> 4k) & 7 of the eight bytes {x (0-3), y (4-7)}.
inline unsigned __byte_perm(unsigned x, unsigned y, unsigned s) {
    const uint64_t v = ((uint64_t)y << 32) | x;
    unsigned r = 0;
    for (int k = 0; k < 4; ++k) r |= (unsigned)((v >> (8 * ((s >> (4 * k)) & 7u))) & 0xffu) << (8 * k);
    return r;
}

// Warp operations of a warp with one active lane.
inline unsigned __activemask() { return 1u; }
inline unsigned __ballot_sync(unsigned, int p) { return p ? 1u : 0u; }
inline int __any_sync(unsigned, int p) { return p != 0; }
template <typename T>
inline T __shfl_sync(unsigned, T v, int, int = 32) {
    return v;
}
template <typename T>
inline T __shfl_up_sync(unsigned, T v, unsigned, int = 32) {
    return v;
}
// A butterfly exchange with no other lane: the lane's own value, which keeps min / max
// reductions right; the warp sums of the adjoint kernels would come out scaled, and the host
// builds do not run those kernels.
template <typename T>
inline T __shfl_xor_sync(unsigned, T v, int, int = 32) {
    return v;
}
template <typename T>
inline unsigned __match_any_sync(unsigned, T) {
    return 1u;
}
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline void __syncthreads() {}
inline void __syncwarp(unsigned = 0xffffffffu) {}

// Atomics of a single thread.
template <typename T>
inline T atomicAdd(T *p, T v) {
    const T old = *p;
    *p = old + v;
    return old;
}
inline int atomicCAS(int *p, int cmp, int v) {
    const int old = *p;
    if (old == cmp) *p = v;
    return old;
}
inline int atomicMin(int *p, int v) {
    const int old = *p;
    if (v < old) *p = v;
    return old;
}
inline int atomicMax(int *p, int v) {
    const int old = *p;
    if (v > old) *p = v;
    return old;
}
