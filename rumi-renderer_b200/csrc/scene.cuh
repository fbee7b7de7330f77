// Device-resident scene layout (one struct of pointers, passed by value to kernels).
//
// HBM layout (all arrays cudaMalloc'd by rumi_scene_create, 256-byte aligned):
//   nodes      : BvhNode[n_nodes]        32 B each; siblings adjacent, pairs 64-B aligned
//   nodes4     : Bvh4Node[n_nodes4]      128 B each, collapsed from `nodes`; siblings adjacent
//   leaf_prims : float4[3 * n_prims]     48 B per primitive, in BVH leaf order
//   tri_shade  : float4[3 * n_tris]      shading normals n0,n1,n2 (canonical order);
//                                        .w of the first holds the material index
//   tri_albedo : float4[n_tris]          optional per-triangle Matte colour (rgb)
//   rects      : float4[3 * n_rects]     p, l, w (.w of p = material index)
//   spheres    : float4[n_spheres]       centre xyz, radius
//   sphere_mat : int[n_spheres]
//   materials  : DevMaterial[n_materials]
//   lights     : DevLight[n_lights]
//   textures   : DevTexture[n_textures] (+ one pixel array each), prim_tex : int[n_prims]
//                (canonical order, -1 = none), sphere_frame : float4[3 * n_spheres]
//                (present only when the scene has textures)
#pragma once
#include "common.cuh"

// Primitive kinds stored in leaf_prims[3i+1].w (as int bits).
enum { PRIM_TRI = 0, PRIM_RECT = 1, PRIM_SPHERE = 2 };
#define PRIM_FLAG_EMISSIVE 0x100
// an emissive, textured sphere (an image-based light's sphere): a ray that starts inside
// it takes the far root (Sphere::Intersect, sphere.cpp:85-92)
#define PRIM_FLAG_IBL 0x200

enum { MAT_MATTE = 0, MAT_GLOSSY = 1, MAT_SPECULAR = 2, MAT_EMISSIVE = 3, MAT_DIELECTRIC = 4, MAT_SUBSURFACE = 5 };
enum { LIGHT_AREA = 0, LIGHT_SPOT = 1, LIGHT_IBL = 2 };
enum { TEX_CHECKER = 0, TEX_IMAGE = 1, TEX_HDR = 2 };
enum { SHAPE_TRI = 0, SHAPE_RECT = 1, SHAPE_SPHERE = 2 };

// 32-byte BVH node.  count > 0: leaf over leaf_prims[first .. first+count).
// count == 0: interior; its two children are nodes[first] and nodes[first + 1].
struct __align__(16) BvhNode {
    float lo_x, lo_y, lo_z, hi_x;
    float hi_y, hi_z;
    int first;
    int count;
};

// 128-byte four-wide node, collapsed from the binary tree (bvh4.cu): child boxes in SoA
// order so a node is eight float4 loads (one 128-byte line).  count[i] > 0: leaf over
// leaf_prims[child[i] .. child[i]+count[i]); count[i] == 0: interior child node
// nodes4[child[i]]; count[i] < 0: empty slot (its box is empty).
struct __align__(128) Bvh4Node {
    float lo_x[4], hi_x[4];
    float lo_y[4], hi_y[4];
    float lo_z[4], hi_z[4];
    int child[4];
    int count[4];
};

// The four-wide tree halves the node steps per ray (34.6 vs 47.7 node units of 32 bytes per
// camera ray on the 1M-triangle mesh, fewer primitive tests), but each step costs more issue
// slots (four slabs, a sorting network, classification).  Measured per 1024x1024x64 frame on
// B200: warp-batch walk, binary 143 / four-wide 178 ms of closest-hit; speculative while-while
// walk (the default scheme), binary 100 / four-wide 130 ms (any-hit 83.5 / 87.8 ms).  So the
// binary tree is the default and the four-wide tree is built and walked only when this is 1
// (both walks pass the same hit and image parity tests).
#ifndef RUMI_BVH_WIDE
#define RUMI_BVH_WIDE 0  // 1: walk the four-wide tree (nodes4), 0: the binary tree
#endif

struct DevMaterial {
    int type;
    float kd, ks, e;          // Matte kd; Glossy kd, ks, Phong exponent; Specular kr; Emissive ls
    float3 rgb;               // albedo / emission colour / Dielectric absorption / Subsurface sigma_s
    float eta_in, eta_out;
    float3 rgb2;              // Subsurface sigma_a
    float3 sigma_t;           // Subsurface sigma_s + sigma_a
    float avg_sigma_t;        // Subsurface mean sigma_t * density
    float absorb;             // Subsurface mean sigma_a / sigma_t
    float kd_pdf;             // Glossy kd / (kd + ks)
    float phong_norm;         // Glossy (e + 1) / (2 pi)
    float3 le;                // Emissive rgb * ls
};

struct DevTexture {
    int type;                   // TEX_CHECKER / TEX_IMAGE / TEX_HDR
    float rep_u, rep_v;         // Checker _w, _h
    float3 c1, c2;              // Checker colours
    float gamma;                // ImageTexture gamma
    int iw, ih, bpp;            // image width, height, bytes per pixel
    const unsigned char *img;   // ImageTexture: LoadBmp's buffer
    const float *hdr;           // HDRTexture: LoadHDR's buffer
};

struct DevLight {
    int type;                 // LIGHT_AREA / LIGHT_SPOT
    int shape_type;           // SHAPE_RECT / SHAPE_SPHERE / SHAPE_TRI
    int shape_index;          // index within its shape array
    float inv_area;           // Shape::Pdf()
    float3 le;                // Emissive::Le()
    // spot light
    float3 position, direction;
    float cos_cone;
    float3 intensity;
};

struct DevVolume {
    int present;
    float3 bmin, bmax;
    float3 sigma_s, sigma_a, sigma_t;
    float avg_sigma_t;        // Average(sigma_t)
    float absorb;             // Average(sigma_a / sigma_t)
    float g;                  // Henyey-Greenstein asymmetry (0 = isotropic)
};

struct DevCamera {
    float3 p;
    float m[12];              // first three rows of Pinhole::_basis_transform
    float tanfov, y_ratio, film_area, plane_dist;
    float3 dir;               // _basis_transform * (0,0,1)
    float3 up, right;         // _basis_transform * (0,1,0), * (1,0,0) (translation column added)
    float focal_distance, lens_radius;  // Pinhole::DepthOfField; focal_distance > 0: thin lens
};

struct DevScene {
    const BvhNode *nodes;
    const float4 *leaf_prims;
    const float4 *tri_shade;
    const float4 *tri_albedo;   // may be null
    const float4 *rects;
    const float4 *spheres;
    const int *sphere_mat;
    const DevMaterial *materials;
    const DevLight *lights;
    int n_tris, n_rects, n_spheres, n_prims;
    int n_materials, n_lights;
    int n_nodes;
    const Bvh4Node *nodes4;     // the four-wide tree the traversal kernels walk
    int n_nodes4;
    DevVolume volume;
    DevCamera camera;
    int width, height;
    // textures (null when the scene has none)
    const DevTexture *textures;
    const int *prim_tex;
    const float4 *sphere_frame;
    int n_textures;
};

// Canonical primitive id -> material index.
RUMI_D int prim_material(const DevScene &s, int id) {
    if (id < s.n_tris) return __float_as_int(__ldg(&s.tri_shade[3 * id].w));
    id -= s.n_tris;
    if (id < s.n_rects) return __float_as_int(__ldg(&s.rects[3 * id].w));
    id -= s.n_rects;
    return __ldg(&s.sphere_mat[id]);
}
