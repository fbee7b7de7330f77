// Device-resident scene layout (one struct of pointers, passed by value to kernels).
//
// HBM layout (all arrays cudaMalloc'd by rumi_scene_create, 256-byte aligned):
//   nodes      : BvhNode[n_nodes]        32 B each; siblings adjacent, pairs 64-B aligned
//   nodes4     : Bvh4Node[n_nodes4]      128 B each, collapsed from `nodes`; siblings adjacent
//   nodes8     : Bvh8Node[n_nodes8]      80 B each, compressed eight-wide tree collapsed from
//                                        `nodes`; a node's interior children are adjacent
//   prims8     : float4[3 * n_prims]     the leaf primitives re-laid out for nodes8: the leaf
//                                        children of one node are adjacent, in slot order
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

// 80-byte compressed eight-wide node (five float4 loads), collapsed from the binary tree by
// bvh8.cu.  Child boxes are stored as 8-bit multiples of a per-axis power-of-two quantum
// 2^e relative to the origin (ox, oy, oz), rounded strictly outward by at least one
// quantum, so every child box contains its exact box: culling stays conservative and hit
// results equal the binary tree's.  Slot k of a node:
//   - interior child when bit k of imask is set: node child_base + popc(imask & ((1<<k)-1));
//   - leaf child when its count byte c_k (cnt_lo / cnt_hi) is > 0: primitives
//     prims8[prim_base + c_0 + ... + c_{k-1} .. + c_k);
//   - empty otherwise.
// Children are assigned to slots by octant: slot k holds the child that comes first along
// the diagonal direction (-1)^(k&1), (-1)^(k>>1&1), (-1)^(k>>2&1), so a ray whose direction
// signs form octant code q (bit a set when component a is negative) visits slots in the
// order k ^ q for k = 0, 1, ... -- near children first without sorting.
struct __align__(16) Bvh8Node {
    // first float4: what taking a child from a node needs
    unsigned int meta;        // bytes 0-2: e_x, e_y, e_z biased by 127 (the float exponent
                              // field of the quantum); byte 3: imask
    int child_base;           // first interior child
    int prim_base;            // first primitive of the leaf children
    float ox;                 // quantisation origin (x)
    // second float4
    float oy, oz;             // quantisation origin (y, z)
    unsigned int cnt_lo;      // leaf primitive counts of slots 0-3, one byte each
    unsigned int cnt_hi;      // slots 4-7
    // three float4 of child bounds
    unsigned int qlo_x[2], qlo_y[2], qlo_z[2];  // byte k: child k's low bound in quanta
    unsigned int qhi_x[2], qhi_y[2], qhi_z[2];  // byte k: high bound
};
static_assert(sizeof(Bvh8Node) == 80, "Bvh8Node is five float4");

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
    const Bvh8Node *nodes8;     // the compressed eight-wide tree (0 nodes: empty scene)
    const float4 *prims8;       // leaf primitives in nodes8 order
    int n_nodes8;
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
