// Collapse of the binary SAH tree into the compressed eight-wide tree (Bvh8Node, scene.cuh).
//
// Each eight-wide node is made from one binary interior node: start from its two children
// and, while fewer than eight, open the interior candidate of largest surface area (its two
// children take its place).  Leaves keep their primitives, which are copied into prims8 so
// that the leaf children of one node are adjacent (prim_base + the counts of the slots
// before).  Children are placed in slots by octant: greedily, the (child, slot) pair of
// smallest cost dot(centroid(child) - centroid(node), diagonal(slot)) is taken first, so
// slot k holds a child that comes early along diagonal k (the ordering idea of compressed
// wide BVHs: Ylitie, Karras & Laine, "Efficient Incoherent Ray Traversal on GPUs Through
// Compressed Wide BVHs", HPG 2017).
//
// Child boxes are quantised per node and axis to 8 bits: quantum 2^e with 253 * 2^e >= the
// node's extent, and never below 2^-21 of the coordinates' magnitude (eight float ulps);
// origin = node low - one quantum; a child's low bound is the largest grid value strictly
// below its exact low bound and its high bound the smallest strictly above, so the stored
// box contains the exact one with at least a quantum to spare on every side.  The
// collapse runs breadth first, one launch per level: a thread per frontier node.  Every
// index and quantised value is range-checked; a violation sets an error flag instead of
// writing.
#include "renderer.h"
#include <cfloat>

namespace rumi {

namespace {

struct Frontier8 {
    int b2;  // binary node
    int b8;  // eight-wide node to fill
};

__device__ __forceinline__ float half_area8(const BvhNode &n) {
    const float dx = n.hi_x - n.lo_x, dy = n.hi_y - n.lo_y, dz = n.hi_z - n.lo_z;
    return dx * dy + dy * dz + dz * dx;
}

// 1: leaf, 2: interior with a usable child pair and a non-empty box, 0: nothing to keep
// (an empty side of a degenerate split is a count-0 node with an empty box and no children).
__device__ __forceinline__ int node_kind8(const BvhNode &c, int n_nodes2) {
    if (c.count > 0) return 1;
    if (c.count == 0 && c.first >= 2 && c.first + 1 < n_nodes2 && c.lo_x <= c.hi_x && c.lo_y <= c.hi_y &&
        c.lo_z <= c.hi_z)
        return 2;
    return 0;
}

// Quantum exponent for an axis spanning [lo, hi].
__device__ int quant_exp(double lo, double hi) {
    int e = -126;
    const double ext = hi - lo;
    if (ext > 0.0) {
        int ex;
        const double m = frexp(ext / 253.0, &ex);  // ext / 253 = m * 2^ex, m in [0.5, 1)
        const int need = m == 0.5 ? ex - 1 : ex;   // smallest e with 2^e >= ext / 253
        e = need > e ? need : e;
    }
    const double mag = fmax(fabs(lo), fabs(hi));
    if (mag > 0.0) {
        int em;
        frexp(mag, &em);  // mag in [2^(em-1), 2^em): a float ulp there is 2^(em-24)
        e = em - 21 > e ? em - 21 : e;
    }
    return e > 127 ? 127 : e;
}

__device__ __forceinline__ unsigned int put_byte(unsigned int w, int k, unsigned int b) {
    return w | (b << (8 * k));
}

__global__ void collapse8_level(const BvhNode *__restrict__ nodes2, int n_nodes2, const float4 *__restrict__ prims2,
                                int n_prims, const Frontier8 *__restrict__ in, const int *__restrict__ n_in,
                                Frontier8 *__restrict__ out, int *__restrict__ n_out, Bvh8Node *__restrict__ nodes8,
                                int *__restrict__ n8, int cap8, float4 *__restrict__ prims8, int *__restrict__ n_p8,
                                int *__restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *n_in) return;
    const Frontier8 f = in[i];
    if (f.b2 < 0 || f.b2 >= n_nodes2 || f.b8 < 0 || f.b8 >= cap8) {
        atomicExch(err, 1);
        return;
    }
    int cand[8], kind[8];
    int nc = 0;
    const BvhNode root = nodes2[f.b2];
    const int rk = node_kind8(root, n_nodes2);
    if (rk == 1) {
        cand[0] = f.b2;  // a leaf root: one leaf child
        kind[0] = 1;
        nc = 1;
    } else if (rk == 2) {
        for (int s = 0; s < 2; ++s) {
            const int k = node_kind8(nodes2[root.first + s], n_nodes2);
            if (k) {
                cand[nc] = root.first + s;
                kind[nc] = k;
                ++nc;
            }
        }
        // open the interior candidate of largest surface area while there is room
        while (nc < 8) {
            int best = -1;
            float best_a = -1.0f;
            for (int k = 0; k < nc; ++k) {
                if (kind[k] != 2) continue;
                const float a = half_area8(nodes2[cand[k]]);
                if (a > best_a) {
                    best_a = a;
                    best = k;
                }
            }
            if (best < 0) break;
            const int first = nodes2[cand[best]].first;
            for (int k = best; k + 1 < nc; ++k) {
                cand[k] = cand[k + 1];
                kind[k] = kind[k + 1];
            }
            --nc;
            for (int s = 0; s < 2; ++s) {
                const int k = node_kind8(nodes2[first + s], n_nodes2);
                if (k) {
                    cand[nc] = first + s;
                    kind[nc] = k;
                    ++nc;
                }
            }
        }
    }
    // node box = union of the children's boxes
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int k = 0; k < nc; ++k) {
        const BvhNode c = nodes2[cand[k]];
        lo[0] = fminf(lo[0], c.lo_x); hi[0] = fmaxf(hi[0], c.hi_x);
        lo[1] = fminf(lo[1], c.lo_y); hi[1] = fmaxf(hi[1], c.hi_y);
        lo[2] = fminf(lo[2], c.lo_z); hi[2] = fmaxf(hi[2], c.hi_z);
    }
    // slots by octant: greedy assignment of the cheapest (child, slot) pair first
    int slot_of[8];
    for (int k = 0; k < 8; ++k) slot_of[k] = -1;
    {
        float pc[3];
        for (int a = 0; a < 3; ++a) pc[a] = nc > 0 ? 0.5f * (lo[a] + hi[a]) : 0.0f;
        float cost[8][8];
        for (int k = 0; k < nc; ++k) {
            const BvhNode c = nodes2[cand[k]];
            const float cx = 0.5f * (c.lo_x + c.hi_x) - pc[0];
            const float cy = 0.5f * (c.lo_y + c.hi_y) - pc[1];
            const float cz = 0.5f * (c.lo_z + c.hi_z) - pc[2];
            for (int s = 0; s < 8; ++s)
                cost[k][s] = ((s & 1) ? -cx : cx) + ((s & 2) ? -cy : cy) + ((s & 4) ? -cz : cz);
        }
        unsigned int used = 0;
        for (int it = 0; it < nc; ++it) {
            float bc = FLT_MAX;
            int bk = -1, bs = -1;
            for (int k = 0; k < nc; ++k) {
                if (slot_of[k] >= 0) continue;
                for (int s = 0; s < 8; ++s) {
                    if (used & (1u << s)) continue;
                    if (bk < 0 || cost[k][s] < bc) {
                        bc = cost[k][s];
                        bk = k;
                        bs = s;
                    }
                }
            }
            slot_of[bk] = bs;
            used |= 1u << bs;
        }
    }
    int child_at[8];  // candidate in slot s, -1 = empty
    for (int s = 0; s < 8; ++s) child_at[s] = -1;
    for (int k = 0; k < nc; ++k) child_at[slot_of[k]] = k;
    int n_int = 0, n_leaf_prims = 0;
    for (int k = 0; k < nc; ++k) {
        if (kind[k] == 2)
            ++n_int;
        else
            n_leaf_prims += nodes2[cand[k]].count;
    }
    int base = 0, pos = 0, pbase = 0;
    if (n_int > 0) {
        base = atomicAdd(n8, n_int);
        pos = atomicAdd(n_out, n_int);
        if (base + n_int > cap8) {
            atomicExch(err, 3);
            return;
        }
    }
    if (n_leaf_prims > 0) {
        pbase = atomicAdd(n_p8, n_leaf_prims);
        if (pbase + n_leaf_prims > n_prims) {
            atomicExch(err, 4);
            return;
        }
    }
    Bvh8Node o;
    int ex[3];
    double org[3], qs[3];
    for (int a = 0; a < 3; ++a) {
        ex[a] = nc > 0 ? quant_exp((double)lo[a], (double)hi[a]) : 0;
        qs[a] = ldexp(1.0, ex[a]);
        org[a] = nc > 0 ? (double)(float)((double)lo[a] - qs[a]) : 0.0;
    }
    o.ox = (float)org[0];
    o.oy = (float)org[1];
    o.oz = (float)org[2];
    unsigned int imask = 0, cnt_lo = 0, cnt_hi = 0;
    unsigned int qlx[2] = {0, 0}, qly[2] = {0, 0}, qlz[2] = {0, 0}, qhx[2] = {0, 0}, qhy[2] = {0, 0},
                 qhz[2] = {0, 0};
    int j = 0, poff = 0;
    for (int s = 0; s < 8; ++s) {
        const int k = child_at[s];
        if (k < 0) continue;
        const BvhNode c = nodes2[cand[k]];
        const float clo[3] = {c.lo_x, c.lo_y, c.lo_z}, chi[3] = {c.hi_x, c.hi_y, c.hi_z};
        unsigned int ql[3], qh[3];
        for (int a = 0; a < 3; ++a) {
            const double xl = ((double)clo[a] - org[a]) / qs[a];
            const double xh = ((double)chi[a] - org[a]) / qs[a];
            const double l = ceil(xl) - 1.0, h = floor(xh) + 1.0;
            if (!(l >= 0.0 && l <= 255.0 && h >= 0.0 && h <= 255.0)) {
                atomicExch(err, 5);
                return;
            }
            ql[a] = (unsigned int)l;
            qh[a] = (unsigned int)h;
        }
        const int w = s >> 2, b = s & 3;
        qlx[w] = put_byte(qlx[w], b, ql[0]); qhx[w] = put_byte(qhx[w], b, qh[0]);
        qly[w] = put_byte(qly[w], b, ql[1]); qhy[w] = put_byte(qhy[w], b, qh[1]);
        qlz[w] = put_byte(qlz[w], b, ql[2]); qhz[w] = put_byte(qhz[w], b, qh[2]);
        if (kind[k] == 2) {
            imask |= 1u << s;
            out[pos + j] = Frontier8{cand[k], base + j};
            ++j;
        } else {
            if (c.count > 255 || c.first < 0 || c.first + c.count > n_prims) {
                atomicExch(err, 6);
                return;
            }
            if (s < 4)
                cnt_lo = put_byte(cnt_lo, b, (unsigned int)c.count);
            else
                cnt_hi = put_byte(cnt_hi, b, (unsigned int)c.count);
            for (int p = 0; p < c.count; ++p) {
                const int src = 3 * (c.first + p), dst = 3 * (pbase + poff + p);
                prims8[dst + 0] = prims2[src + 0];
                prims8[dst + 1] = prims2[src + 1];
                prims8[dst + 2] = prims2[src + 2];
            }
            poff += c.count;
        }
    }
    o.meta = (unsigned int)(ex[0] + 127) | ((unsigned int)(ex[1] + 127) << 8) | ((unsigned int)(ex[2] + 127) << 16) |
             (imask << 24);
    o.child_base = base;
    o.prim_base = pbase;
    o.cnt_lo = cnt_lo;
    o.cnt_hi = cnt_hi;
    for (int w = 0; w < 2; ++w) {
        o.qlo_x[w] = qlx[w]; o.qlo_y[w] = qly[w]; o.qlo_z[w] = qlz[w];
        o.qhi_x[w] = qhx[w]; o.qhi_y[w] = qhy[w]; o.qhi_z[w] = qhz[w];
    }
    nodes8[f.b8] = o;
}

}  // namespace

// Upper bound of eight-wide nodes for n primitives (one per binary interior node).
int bvh8_node_capacity(int n_prims) { return n_prims > 1 ? n_prims : 1; }

size_t bvh8_scratch_bytes(int n_prims) {
    const size_t cap = (size_t)bvh8_node_capacity(n_prims);
    return 2 * cap * sizeof(Frontier8) + 256;
}

// Returns the node count (> 0), 0 for a scene without primitives, or -1 on error.
int bvh8_collapse(const BvhNode *nodes2, int n_nodes2, const float4 *prims2, int n_prims, Bvh8Node *nodes8, int cap8,
                  float4 *prims8, void *scratch, cudaStream_t stream) {
    if (n_prims <= 0) return 0;
    Frontier8 *fa = (Frontier8 *)scratch;
    Frontier8 *fb = fa + cap8;
    int *counters = (int *)(fb + cap8);  // [0] n_in, [1] n_out, [2] n8, [3] err, [4] prims placed
    const int init[5] = {1, 0, 1, 0, 0};
    const Frontier8 root{0, 0};
    cudaMemcpyAsync(counters, init, sizeof(init), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(fa, &root, sizeof(root), cudaMemcpyHostToDevice, stream);
    int n_in = 1;
    for (int level = 0; level < 128 && n_in > 0; ++level) {
        collapse8_level<<<(n_in + 127) / 128, 128, 0, stream>>>(nodes2, n_nodes2, prims2, n_prims, fa, counters + 0,
                                                                fb, counters + 1, nodes8, counters + 2, cap8, prims8,
                                                                counters + 4, counters + 3);
        // next frontier: out -> in
        cudaMemcpyAsync(counters + 0, counters + 1, sizeof(int), cudaMemcpyDeviceToDevice, stream);
        cudaMemsetAsync(counters + 1, 0, sizeof(int), stream);
        cudaMemcpyAsync(&n_in, counters + 0, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
        Frontier8 *t = fa;
        fa = fb;
        fb = t;
    }
    int h[5];
    cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
    if (h[3] != 0 || n_in != 0 || h[4] > n_prims) return -1;
    return h[2];
}

}  // namespace rumi
