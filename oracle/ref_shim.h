/* Force-included into every translation unit of the reference build
 * (oracle/_ref/librumi_ref.so, made by oracle/build_ref.py).  Test infrastructure only.
 *
 * - MSVC-only names the reference uses: _finite, __min, __max, __int16.
 * - rand()/srand() are routed to a generator owned by oracle/ref_harness.cpp so a CPU
 *   render is reproducible for a given seed and unit checks can inject exact uniforms.
 *   RAND_MAX stays glibc's 2^31-1, so RandomFloat() (src/Kernel/clibrary.h:50-53) and
 *   rand() % n keep their meaning.
 * - private/protected are opened so the harness can read members (Scene::_objects,
 *   Pinhole::_fov, Model::_triangles ...) without touching the reference's headers.
 *   Every system header the build needs is included first, so only reference code
 *   sees the redefinition.
 */
#ifndef RUMI_REF_SHIM_H
#define RUMI_REF_SHIM_H

#include <stdio.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <math.h>
#include <time.h>
#include <typeinfo>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <unordered_map>
#include <algorithm>
#include <new>

#define _finite(x) std::isfinite(x)
#define __min(a, b) (((a) < (b)) ? (a) : (b))
#define __max(a, b) (((a) > (b)) ? (a) : (b))
#define __int16 short

extern "C" int rumi_ref_rand(void);
extern "C" void rumi_ref_srand(unsigned int seed);
#define rand() rumi_ref_rand()
#define srand(x) rumi_ref_srand(x)

#define private public
#define protected public

#endif
