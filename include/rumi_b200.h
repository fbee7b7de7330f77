/* rumi_b200.h -- C-ABI of the B200 rendering path for Rumi-Renderer scenes.
 *
 * The reference renders with Scene::Rendering (src/Scene/scene.cpp:206-258), which calls
 * Integrator::Trace(w, h, camera, film) (src/Integrator/integrator.h:15-28) once per pixel
 * sample and sums the results into Film's float buffer (src/Camera/film.cpp:83-97).  This
 * library replaces that loop and the integrators beneath it with GPU kernels:
 *
 *   rumi_scene_create   <- Scene::Build's objects + BVHAccel::BuildBVH
 *                          (src/Scene/scene.cpp:135-204, src/Acceleration/bvh.cpp:129-148)
 *   rumi_render         <- Scene::Rendering + PathTracer::Trace / BidirectionalPathTracer::Trace
 *                          (src/Integrator/pathtracer.cpp:117-354,
 *                           src/Integrator/bidirectionalpathtracer.cpp:121-394)
 *   rumi_render_batch   <- many Scene::Rendering calls, one frame from shared queues
 *   rumi_forward / rumi_backward  <- path-replay adjoint of PathTracer::Trace (new)
 *   rumi_trace_rays     <- BVHAccel::Travel (src/Acceleration/bvh.cpp:150-213), closest-hit
 *                          (isect != NULL) and shadow (isect == NULL) forms
 *
 * Conventions
 *   - Every entry point returns rumi_status; nothing throws across the ABI.  The text of
 *     the last error of the calling thread is available from rumi_last_error_string().
 *   - Colours are given as (r, g, b) like the reference's Color(r, g, b) constructor.
 *     Film buffers are H*W*3 floats in the reference's B,G,R storage order
 *     (src/Kernel/color.h:7-9), row h, column w at ((h * W) + w) * 3 -- the same layout as
 *     Film::_pixel_buffer -- and hold the SUM of the samples of each pixel.
 *   - rumi_scene_create copies everything it is given; the caller's arrays may be freed
 *     on return.  Output buffers belong to the caller.
 *   - A rumi_scene may be used by one host thread at a time.  Calls are synchronous
 *     unless noted: they return once results are in the caller's buffer.
 *   - The library allocates device memory with cudaMalloc on the current CUDA device.
 */
#ifndef RUMI_B200_H
#define RUMI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* RUMI_ERR_INTERNAL: a device-side consistency check failed (the BVH builder's, the four-
 * and eight-wide collapses' and the BDPT kernel's index range checks, which record the
 * violation instead of reading or writing out of range; rumi_last_error_string names it).
 * RUMI_ERR_QUEUE_OVERFLOW and RUMI_ERR_TIMEOUT are reserved and returned by no entry
 * point: every ray queue is sized to its wave before launch, so no push can overflow,
 * and no kernel waits on another kernel or on a flag. */
typedef enum {
    RUMI_OK = 0,
    RUMI_ERR_INVALID_ARG = 1,
    RUMI_ERR_OOM = 2,
    RUMI_ERR_CUDA = 3,
    RUMI_ERR_QUEUE_OVERFLOW = 4,
    RUMI_ERR_TIMEOUT = 5,
    RUMI_ERR_INTERNAL = 6
} rumi_status;

/* material kinds (the reference's Material subclasses, src/Material/) */
enum {
    RUMI_MAT_MATTE = 0,      /* Matte(kd, rgb)                                 matte.cpp:27-31   */
    RUMI_MAT_GLOSSY = 1,     /* Glossy(kd, ks, e, rgb)                         glossy.cpp:19-25  */
    RUMI_MAT_SPECULAR = 2,   /* Specular(kr, rgb)                              specular.cpp:18-23 */
    RUMI_MAT_EMISSIVE = 3,   /* Emissive(ls, rgb)                              emissive.cpp:17-23 */
    RUMI_MAT_DIELECTRIC = 4, /* Dielectric(eta_in, eta_out, absorption)        dielectric.cpp:18-23 */
    RUMI_MAT_SUBSURFACE = 5  /* Subsurface(eta_in, eta_out, sigma_s, sigma_a, density) subsurface.cpp:21-40 */
};

typedef struct {
    int32_t type;
    float kd;        /* Matte kd, Glossy kd, Specular kr, Emissive ls */
    float ks;        /* Glossy ks */
    float exponent;  /* Glossy Phong exponent e */
    float rgb[3];    /* colour; Dielectric absorption; Subsurface sigma_s */
    float eta_in, eta_out;
    float rgb2[3];   /* Subsurface sigma_a */
    float density;   /* Subsurface density (1 = none) */
} rumi_material;

enum { RUMI_SHAPE_TRIANGLE = 0, RUMI_SHAPE_RECT = 1, RUMI_SHAPE_SPHERE = 2 };
enum { RUMI_LIGHT_AREA = 0, RUMI_LIGHT_SPOT = 1, RUMI_LIGHT_IBL = 2 };

/* texture kinds (src/Texture/): Texture::Pattern(shape, p) = Pixel(TextureMapping(p)) */
enum {
    RUMI_TEX_CHECKER = 0, /* Checker(width, height, c1, c2)                checker.cpp:17-32 */
    RUMI_TEX_IMAGE = 1,   /* ImageTexture(bmp, gamma): the pixels LoadBmp returns (rows in file
                             order, bottom row first, B,G,R[,A] bytes, no row padding)
                                                                    imagetexture.cpp:32-61 */
    RUMI_TEX_HDR = 2      /* HDRTexture(hdr): the floats LoadHDR returns (top scanline first,
                             R,G,B)                                 hdrtexture.cpp:30-44 */
};

typedef struct {
    int32_t type;
    float repeat_u, repeat_v;   /* Checker _w, _h */
    float color1[3], color2[3]; /* Checker _c1, _c2 (r, g, b) */
    float gamma;                /* ImageTexture _gamma (1 = linear bytes) */
    int32_t img_width, img_height, bytes_per_pixel;
    const void *pixels;         /* IMAGE: uint8 img_height*img_width*bytes_per_pixel;
                                   HDR: float img_height*img_width*3 */
} rumi_texture;

typedef struct {
    int32_t type;         /* RUMI_LIGHT_AREA: AreaLight(shape) (src/Light/arealight.cpp);
                             RUMI_LIGHT_SPOT: point emitter with a cone (no reference
                             counterpart);
                             RUMI_LIGHT_IBL: ImageBasedLight(sphere, material, texture)
                             (src/Light/imagebasedlight.cpp): an emissive, textured sphere
                             around the scene, sampled by cosine-weighted directions about
                             the shading normal */
    int32_t shape_type;   /* area light: RUMI_SHAPE_RECT or RUMI_SHAPE_SPHERE; IBL: RUMI_SHAPE_SPHERE */
    int32_t shape_index;  /* area light / IBL: index within that shape array */
    float position[3];    /* spot */
    float direction[3];   /* spot, unit */
    float cone_deg;       /* spot half-angle */
    float intensity[3];   /* spot */
} rumi_light;

typedef struct {
    int32_t present;
    float pmin[3], pmax[3];   /* HomogeneousVolume(BBox(pmin, pmax), sigma_s, sigma_a) */
    float sigma_s[3], sigma_a[3];
    float g;                  /* Henyey-Greenstein asymmetry; 0 = the reference's Isotropic */
} rumi_volume;

typedef struct {
    float position[3];
    float basis[16];      /* Pinhole::_basis_transform, row-major */
    float y_ratio;        /* Pinhole y_ratio (1 / Film aspect in the reference presets) */
    float fov_deg;        /* Pinhole::_fov (the reference constructor fixes 20) */
    float focal_distance; /* Pinhole::DepthOfField (pinhole.cpp:88-94): > 0 turns on the thin lens */
    float lens_radius;
} rumi_camera;

typedef struct {
    int32_t width, height;

    int32_t n_triangles;
    const float *tri_vertices;    /* n*9: v0, v1, v2 */
    const float *tri_normals;     /* n*9: n0, n1, n2 (Triangle::Normal); NULL = face normal */
    const int32_t *tri_material;  /* n material indices */
    const float *tri_albedo;      /* n*3 per-triangle colour overriding the material's rgb; may be NULL */

    int32_t n_rects;
    const float *rects;           /* n*9: p, l, w  (Rect(p, l, w)) */
    const int32_t *rect_material;

    int32_t n_spheres;
    const float *spheres;         /* n*4: centre, radius */
    const int32_t *sphere_material;

    int32_t n_materials;
    const rumi_material *materials;

    int32_t n_lights;
    const rumi_light *lights;

    rumi_volume volume;
    rumi_camera camera;

    /* textures (Shape::AddingTexture, src/Shape/shape.cpp:71-84); all may be 0 / NULL */
    int32_t n_textures;
    const rumi_texture *textures;
    const int32_t *tri_texture;    /* n_triangles texture indices, -1 = none (a triangle maps
                                      every point to (u, v) = (0, 0): Shape::TextureMapping) */
    const int32_t *rect_texture;   /* n_rects, -1 = none (Rect::TextureMapping, rect.cpp:183-196) */
    const int32_t *sphere_texture; /* n_spheres, -1 = none (Sphere::TextureMapping, sphere.cpp:172-192) */
    const float *sphere_frame;     /* n_spheres*9: rows 0-2 of Shape::_transform's upper 3x3, which
                                      orient a sphere's texture; NULL = identity */
} rumi_scene_desc;

typedef struct rumi_scene rumi_scene;

/* RUMI_RAY_TRACER: RayTracer(scene, max_depth), the Whitted integrator
 * (src/Integrator/raytracer.cpp:30-86): mirror and glass chains up to trace depth
 * max_depth (>= 0), direct lighting at the first other surface. */
enum { RUMI_PATH_TRACER = 0, RUMI_BDPT = 1, RUMI_RAY_TRACER = 2 };
enum {
    RUMI_FLAG_TIMING = 1,  /* per-kernel CUDA-event timing into rumi_render_stats */
    RUMI_FLAG_STATS = 2,   /* count BVH node fetches and primitive tests of closest-hit rays */
    RUMI_FLAG_SERIAL = 4,  /* path tracer: every launch in order on the one stream (by default a
                              bounce's shadow rays are traced on a second stream of the scene
                              beside the next bounce's closest-hit rays); with TIMING, each
                              kernel's time is then its time alone on the GPU */
    RUMI_FLAG_KEEP_RADIANCE = 8 /* rumi_forward: keep every path's radiance in a device array of the
                              scene (16 bytes per path, W*H*spp paths); the next rumi_backward with
                              the same seed, spp and max_depth, and no rumi_scene_set_albedo /
                              _set_volume in between, takes the radiance from there instead of
                              tracing its first pass */
};

typedef struct {
    int32_t integrator;    /* RUMI_PATH_TRACER (PathTracer(scene, max_depth)), RUMI_BDPT or RUMI_RAY_TRACER */
    int32_t max_depth;     /* path tracer: vertices per path; ray tracer: largest trace depth */
    int32_t n_light;       /* BDPT nL (light subpath vertices) */
    int32_t n_eye;         /* BDPT nE (eye subpath vertices) */
    int32_t spp;           /* samples per pixel, rendered exactly */
    uint64_t seed;         /* Philox key: same seed -> same image */
    int32_t wave_paths;    /* paths in flight per wave; 0 = library default (2^25) */
    int32_t flags;         /* RUMI_FLAG_* */
    void *stream;          /* cudaStream_t, NULL = the library's own stream */
    /* launch tuning (0 = library default; chosen by rumi_b200.autotune) */
    int32_t trace_mode;    /* traversal scheme.  Binary tree -- 1: a warp traces 32 rays to
                              completion; 2: per-lane ray refill; 3: per-lane refill with
                              leaves intersected warp-wide; 4: speculative while-while walk
                              with per-lane refill.  5: the same walk over the compressed
                              eight-wide tree, collapsed from the binary tree by the scene's
                              first call that asks for it (rumi_render_noalloc cannot: it
                              rejects 5 until then).  0: the library default (4).  Every
                              scheme gives the same hits and films */
    int32_t blocks_per_sm; /* persistent traversal blocks (128 threads) per SM, capped by occupancy */
    int32_t refill_min;    /* idle lanes that trigger a refill (modes 2-5) */
    int32_t stack_depth;   /* traversal stack entries per thread kept in shared memory: 8, 16
                              or 32 (0 = 16; modes 4 and 5 take all three, the others 32);
                              deeper entries spill to local memory, and a smaller stack leaves
                              more of the SM's unified L1 / shared storage to L1 */
} rumi_render_params;

typedef struct {
    int64_t paths;               /* camera paths traced */
    int64_t nan_samples;         /* samples dropped for NaN (counted, as the reference does) */
    int64_t extend_launches;     /* closest-hit launches */
    double extend_ms;            /* summed device time of closest-hit launches (TIMING) */
    int64_t shade_launches;
    double shade_ms;
    int64_t shadow_launches;
    double shadow_ms;
    double total_ms;             /* device time of the whole render (TIMING) */
    int64_t rays_extend;         /* closest-hit rays traced */
    int64_t rays_shadow;         /* shadow rays traced */
    int64_t extend_node_fetches; /* node bytes fetched by closest-hit rays / 32 (STATS): a binary
                                    node counts 1, a compressed eight-wide node 2.5 */
    int64_t extend_prim_tests;   /* primitives tested by closest-hit rays (STATS) */
} rumi_render_stats;

typedef struct {
    int32_t large_levels;
    int32_t small_tasks;
    int32_t n_nodes;             /* node slots reserved */
    double build_ms;
} rumi_bvh_info;

/* Creates a scene on the current device: copies the description, builds the BVH on the
 * GPU.  *out receives the scene or NULL on error. */
rumi_status rumi_scene_create(const rumi_scene_desc *desc, rumi_scene **out);

/* Releases every device allocation of the scene. */
rumi_status rumi_scene_destroy(rumi_scene *scene);

/* Information about the scene's BVH build. */
rumi_status rumi_scene_bvh_info(const rumi_scene *scene, rumi_bvh_info *info);

/* Renders one frame: film receives H*W*3 floats (B,G,R sums of `spp` samples per pixel).
 * film_on_device != 0: film is a device pointer (no host copy).  stats may be NULL. */
rumi_status rumi_render(rumi_scene *scene, const rumi_render_params *params, float *film, int32_t film_on_device,
                        rumi_render_stats *stats);

/* Renders one path-traced frame like rumi_render, but allocates no device memory: the
 * wave state lives in a fixed 16 MiB device array inside the library (held on every GPU
 * that loads it until exit), so frames render in waves of about 95k paths (176 bytes per
 * path).  For callers that may not allocate once running -- an application that owns a
 * fixed device-memory budget, or a real-time loop that cannot take cudaMalloc's
 * device-wide synchronisation.  The scene is created beforehand with rumi_scene_create.
 * film: device pointer, H*W*3 floats.  Path tracer only; spp or wave_paths beyond the
 * array's capacity and RUMI_FLAG_TIMING are rejected with RUMI_ERR_INVALID_ARG.  The
 * first call on a device looks up the array's device address and caches it (make that
 * call before any stream capture; the cache does not survive cudaDeviceReset).  All calls
 * share the array: calls that overlap on the GPU race and must be serialised by the
 * caller.  No counterpart in the reference. */
rumi_status rumi_render_noalloc(rumi_scene *scene, const rumi_render_params *params, float *film,
                                rumi_render_stats *stats);

/* Multi-scene batches: many scenes of uneven size and sample count rendered as one frame
 * from shared ray queues (no counterpart in the reference, which renders one scene per
 * process).  The batch references its scenes (which must outlive it and live on the
 * current device); films are the scenes' films concatenated in scene order
 * (rumi_batch_film_floats floats in total).  Scene i uses seeds[i] and its own path
 * numbering, so its image equals rumi_render's for that scene and seed. */
typedef struct rumi_batch rumi_batch;

enum { RUMI_BATCH_GRAPH = 4 };  /* capture the frame as a CUDA graph on first use, then replay */

typedef struct {
    int32_t max_depth;       /* path tracer depth shared by the batch */
    const int32_t *spp;      /* samples per pixel of each scene */
    const uint64_t *seeds;   /* Philox seed of each scene */
    int32_t wave_paths;      /* paths in flight per wave (queue capacity); 0 = default (2^25) */
    int32_t flags;           /* RUMI_FLAG_TIMING, RUMI_BATCH_GRAPH */
    int32_t blocks_per_sm;   /* persistent traversal blocks per SM; 0 = occupancy limit */
    void *stream;            /* cudaStream_t; NULL = the batch's own stream */
} rumi_batch_params;

rumi_status rumi_batch_create(rumi_scene *const *scenes, int32_t n, rumi_batch **out);
rumi_status rumi_batch_destroy(rumi_batch *batch);
int64_t rumi_batch_film_floats(const rumi_batch *batch);
rumi_status rumi_render_batch(rumi_batch *batch, const rumi_batch_params *params, float *films,
                              int32_t films_on_device, rumi_render_stats *stats);

/* Path-replay adjoint of the path tracer (no counterpart in the reference).
 *
 * rumi_forward renders exactly what rumi_render renders (integrator RUMI_PATH_TRACER).
 * rumi_backward, given d_film = dLoss/dfilm (H*W*3 floats, the film's B,G,R layout) and
 * the same params (seed, spp, depth, wave_paths), writes the gradient of
 * sum(d_film * film) with respect to
 *   grad_albedo: the per-triangle albedo (n_triangles * 3 floats, r,g,b, the layout of
 *                rumi_scene_desc.tri_albedo); only Lambertian (Matte) triangles receive
 *                gradient; NULL = not wanted;
 *   grad_volume: the medium (7 floats: sigma_s r,g,b, sigma_a r,g,b, g); NULL = not wanted.
 * Paths are replayed from their Philox streams (no per-vertex tape): each wave is traced
 * once to record every path's radiance and once more to weight each event's score with
 * the radiance that follows it.  Albedo gradients are exact for the estimator (albedo
 * drives no sampling decision); medium gradients are score-function estimates of the
 * derivative of the expected image (free-flight, absorption and shadow-transmittance
 * decisions and the phase direction depend on the coefficients).  NaN samples, which
 * the film drops, receive no gradient.  on_device: all buffers are device pointers.
 * With the forward's seed the result is the exact derivative of that frame's
 * <d_film, film>; for a loss that is nonlinear in the film (L2) give the backward a
 * different seed, so that the residual and the derivative come from independent paths
 * and the gradient is unbiased. */
rumi_status rumi_forward(rumi_scene *scene, const rumi_render_params *params, float *film,
                         int32_t film_on_device, rumi_render_stats *stats);
rumi_status rumi_backward(rumi_scene *scene, const rumi_render_params *params, const float *d_film,
                          float *grad_albedo, float *grad_volume, int32_t on_device,
                          rumi_render_stats *stats);

/* Parameter updates between optimisation steps (the BVH is kept).  albedo: n_triangles*3
 * floats (r,g,b); the scene must have been created with tri_albedo.  volume: replaces the
 * medium (box and coefficients; present = 0 removes it). */
rumi_status rumi_scene_set_albedo(rumi_scene *scene, const float *albedo, int32_t on_device);
rumi_status rumi_scene_set_volume(rumi_scene *scene, const rumi_volume *volume);

/* Ray queries against the scene's BVH.  rays: n*8 floats (o.xyz, in_object flag as
 * 0/1, d.xyz, tmax).  anyhit = 0: closest hit -> t (0 = miss, the reference's
 * Ray::_tmin after Travel) and prim (canonical primitive id, -1 = miss).  anyhit = 1:
 * occlusion -> prim 1 when something lies in [1e-4, tmax - 1e-4], else 0.
 * on_device != 0: all pointers are device pointers.  node_visits / prim_tests (may be
 * NULL): summed node bytes fetched / 32 and primitive tests over the batch. */
rumi_status rumi_trace_rays(rumi_scene *scene, int64_t n, const float *rays, int32_t anyhit, float *t,
                            int32_t *prim, int32_t on_device, int64_t *node_visits, int64_t *prim_tests,
                            void *stream);

/* Film output.  rumi_film_tonemap restates Film::Save's conversion
 * (src/Camera/film.cpp:152-203): each of the film's B,G,R pixel sums is divided by the
 * square of the film's sampling depth ((int)sqrt(n_samples)), raised to 1 / gamma, scaled
 * by 255, clamped to [0, 255] and truncated; out holds width*height*bytes_per_pixel bytes
 * (3 or 4; a fourth byte is 0) in the film's row order.  rumi_film_fireflies restates
 * FirefliesFiltering (src/Scene/scene.cpp:261-432) on such a buffer: a pixel with a
 * channel at 255 none of whose neighbours is white (all three channels at 255) becomes the
 * mean of its neighbours, with the reference's border rules (where those rules reach outside the
 * image, the reference reads outside its buffer; here such reads give 0).  in and out
 * must be distinct.  on_device: buffers are device pointers; stream may be NULL. */
rumi_status rumi_film_tonemap(const float *film, int32_t width, int32_t height, int32_t n_samples, float gamma,
                              int32_t bytes_per_pixel, uint8_t *out, int32_t on_device, void *stream);
rumi_status rumi_film_fireflies(const uint8_t *in, int32_t width, int32_t height, int32_t bytes_per_pixel,
                                uint8_t *out, int32_t on_device, void *stream);

/* Text of the calling thread's last error ("" if none). */
const char *rumi_last_error_string(void);

/* Library version string. */
const char *rumi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RUMI_B200_H */
