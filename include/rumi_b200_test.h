/* rumi_b200_test.h -- verification entry points of librumi_b200.so.
 *
 * Each runs ONE device routine of the renderer over a batch of caller-supplied inputs
 * (host pointers; the call copies to the GPU, launches, and copies back), so that tests
 * can compare the GPU arithmetic with the reference's routines on identical inputs and
 * uniforms.  They are not part of the rendering interface and have no counterpart in the
 * reference beyond the routine each one evaluates (cited per function).
 */
#ifndef RUMI_B200_TEST_H
#define RUMI_B200_TEST_H

#include "rumi_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Philox4x32-10: ctr n*4 words, key 2 words -> out n*4 words. */
rumi_status rumi_test_philox(int64_t n, const uint32_t *ctr, const uint32_t *key, uint32_t *out);

/* Material::BSDFSampling (src/Material/, one file per material).  wo, nrm: n*3; u: n*3 (lobe, u1, u2).
 * out n*9: wi.xyz, Le, go_into_object, xi, pdf_path, costheta, pdf_w. */
rumi_status rumi_test_material_sample(const rumi_material *m, int64_t n, const float *wo, const float *nrm,
                                      const float *u, float *out);

/* Material::Fr.  nrm, wi, wo, vol_ratio: n*3; in_object, xi, pdf_path, t_in: n.  out n*3 (r, g, b). */
rumi_status rumi_test_material_fr(const rumi_material *m, int64_t n, const float *nrm, const float *wi,
                                  const float *wo, const int32_t *in_object, const float *xi, const float *pdf_path,
                                  const float *t_in, const float *vol_ratio, float *out);

/* HomogeneousVolume::DistanceSampling (src/Volume/homogeneousvolume.cpp:168-215).
 * smax, xi, xi_absorb: n.  out n*9: outcome (0 pass, 1 scatter, 2 absorbed), s, tau rgb, pdf rgb, 0. */
rumi_status rumi_test_distance_sample(const float *sigma_s, const float *sigma_a, int64_t n, const float *smax,
                                      const float *xi, const float *xi_absorb, float *out);

/* Phase sampling about the propagation direction d (Isotropic::PhaseSampling at g = 0,
 * Henyey-Greenstein otherwise).  d: n*3, u: n*2.  out n*4: wi.xyz, pdf. */
rumi_status rumi_test_phase_sample(int64_t n, const float *d, float g, const float *u, float *out);

/* Pinhole::CastViewRay (src/Camera/pinhole.cpp:97-136).  pix: n*2 (w, h), smp: n*2,
 * lens_u: n*2 lens uniforms (radius, angle) used when cam->focal_distance > 0, or NULL
 * for zeros.  out n*6: o.xyz, d.xyz. */
rumi_status rumi_test_camera_rays(const rumi_camera *cam, int32_t width, int32_t height, int64_t n, const int32_t *pix,
                                  const float *smp, const float *lens_u, float *out);

/* The pixel sampler: sample index s of `spp` in pixel `pixel` for `seed`.  out n*2. */
rumi_status rumi_test_pixel_samples(int64_t n, const int32_t *s, int32_t spp, const int64_t *pixel, uint64_t seed,
                                    float *out);

/* Device time (ms, CUDA events on `stream`) of one launch that reads the device buffer
 * `passes` times (float4 loads, cached in L2 only).  A buffer smaller than L2 measures L2
 * read bandwidth: bytes * passes / ms. */
rumi_status rumi_test_read_bandwidth(const void *buf_dev, int64_t bytes, int32_t passes, void *stream, double *ms);

/* Texture::Pattern(shape, p) (src/Texture/texture.cpp:17-23) of a scene's primitives:
 * prim n canonical primitive ids (triangles, rects, spheres), pts n*3; out n*3 (r, g, b),
 * 1 where the primitive has no texture. */
rumi_status rumi_test_texture_pattern(rumi_scene *scene, int64_t n, const int32_t *prim, const float *pts,
                                      float *out);

/* rumi_trace_rays (host arrays, n rays of 8 floats: o, in_object, d, tmax) through the
 * traversal scheme trace_mode selects (as rumi_render_params.trace_mode: 1-4 the binary
 * tree's walks, 5 the eight-wide tree's; 0 = the default), so every scheme's hits can be
 * compared on the same rays.  t: n distances (0 = miss); prim: n canonical primitive ids
 * (-1 = miss; any-hit: 1 = occluded, 0 = not). */
rumi_status rumi_test_trace_scheme(rumi_scene *scene, int64_t n, const float *rays, int32_t anyhit,
                                   int32_t trace_mode, float *t, int32_t *prim);

#ifdef __cplusplus
}
#endif

#endif /* RUMI_B200_TEST_H */
