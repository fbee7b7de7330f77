// Host build of the BDPT kernel (rumi-renderer_b200/csrc/bdpt.cu): the kernel body
// compiled by g++ as plain C++ and run one camera sample after another, so that the CPU
// tests can run it under AddressSanitizer and UndefinedBehaviorSanitizer with every
// automatic variable set to a non-zero pattern (an index read before it is written then
// leaves its range and is caught).  Test infrastructure, not part of the library.
//
// The scene is laid out by host_scene.h.
#include "cuda_host_shim.h"
#include "../../rumi-renderer_b200/csrc/bdpt.cu"

using namespace rumi;

#include "host_scene.h"

using namespace host_build;

extern "C" {

// Renders camera samples [pix0 * spp, (pix0 + n_pix) * spp) of a BDPT frame, one after
// another, with the kernel's launch parameters set as bdpt_render sets them.
//   L_out      : n_pix * spp * 4 floats (each sample's value, as the kernel writes it)
//   light_film : width * height * 3 floats (B, G, R light-tracing splats), zeroed here
//   chk        : 4 ints, the kernel's index-check record (0 in chk[0]: no check fired)
// Returns 0, -1 for a description this build does not cover, -2 for bad arguments.
int rumi_host_bdpt(const rumi_scene_desc *d, int n_light, int n_eye, int spp, uint64_t seed, int pix0, int n_pix,
                   float *L_out, float *light_film, int *chk) {
    if (!d || !L_out || !light_film || !chk || spp < 1 || n_pix < 0 || pix0 < 0) return -2;
    if (n_light < 2 || n_eye < 2 || n_light > BD_MAXV || n_eye > BD_MAXV) return -2;
    if ((long long)pix0 + n_pix > (long long)d->width * d->height || d->n_lights <= 0) return -2;
    HostScene H;
    if (build_scene(*d, H) != 0 || H.has_ibl) return -1;  // bdpt_render rejects image-based lights
    BdLaunch B;
    memset(&B, 0, sizeof(B));
    B.s = H.dev;
    B.nL = n_light;
    B.nE = n_eye;
    B.spp = spp;
    B.k0 = (uint32_t)seed;
    B.k1 = (uint32_t)(seed >> 32) ^ 0x5851F42Du;
    int g = 0;
    while ((g + 1) * (g + 1) <= spp) ++g;
    B.grid_d = g;
    B.square = g * g == spp;
    B.L = reinterpret_cast<float4 *>(L_out);
    B.light_film = light_film;
    memset(light_film, 0, sizeof(float) * 3 * (size_t)d->width * d->height);
    const DevCamera &c = B.s.camera;
    B.right = mk3(c.m[0] + c.m[3], c.m[4] + c.m[7], c.m[8] + c.m[11]);
    B.up = mk3(c.m[1] + c.m[3], c.m[5] + c.m[7], c.m[9] + c.m[11]);
    B.pix0 = pix0;
    B.n_paths = n_pix * spp;
    B.path0 = (long long)pix0 * spp;
    memset(g_bd_range, 0, sizeof(g_bd_range));
    blockDim = {(unsigned)BD_THREADS, 1, 1};
    gridDim = {(unsigned)((B.n_paths + BD_THREADS - 1) / BD_THREADS), 1, 1};
    for (int j = 0; j < B.n_paths; ++j) {
        blockIdx.x = (unsigned)(j / BD_THREADS);
        threadIdx.x = (unsigned)(j % BD_THREADS);
        if (n_light <= 8 && n_eye <= 8)
            bdpt_kernel<8>(B);
        else
            bdpt_kernel<BD_MAXV>(B);
    }
    memcpy(chk, g_bd_range, sizeof(g_bd_range));
    return 0;
}

}  // extern "C"
