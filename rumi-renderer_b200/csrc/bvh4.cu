// Collapse of the binary SAH tree into the four-wide tree the traversal kernels walk.
//
// Each four-wide node is made from one binary interior node: start from its two
// children and, while fewer than four, open the interior candidate of largest surface
// area (its two children take its place).  Leaves keep their primitive ranges.  The
// collapse runs breadth first, one launch per level of the four-wide tree: a thread per
// frontier node fills its node, allocates its interior children as one contiguous block
// (siblings adjacent in memory) and appends them to the next frontier.
#include "renderer.h"
#include <cfloat>

namespace rumi {

namespace {

struct Frontier {
    int b2;  // binary node
    int b4;  // four-wide node to fill
};

__device__ __forceinline__ float half_area(const BvhNode &n) {
    const float dx = n.hi_x - n.lo_x, dy = n.hi_y - n.lo_y, dz = n.hi_z - n.lo_z;
    return dx * dy + dy * dz + dz * dx;
}

// 1: leaf, 2: interior with a usable child pair and a non-empty box, 0: nothing to keep
// (the binary builder leaves an empty side of a degenerate split as a count-0 node with
// an empty box and no children; the binary traversal never enters it, the collapse drops it).
__device__ __forceinline__ int node_kind(const BvhNode &c, int n_nodes2) {
    if (c.count > 0) return 1;
    if (c.count == 0 && c.first >= 2 && c.first + 1 < n_nodes2 && c.lo_x <= c.hi_x && c.lo_y <= c.hi_y &&
        c.lo_z <= c.hi_z)
        return 2;
    return 0;
}

__global__ void collapse_level(const BvhNode *__restrict__ nodes2, int n_nodes2, const Frontier *__restrict__ in,
                               const int *__restrict__ n_in, Frontier *__restrict__ out, int *__restrict__ n_out,
                               Bvh4Node *__restrict__ nodes4, int *__restrict__ n4, int cap4, int *__restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *n_in) return;
    const Frontier f = in[i];
    if (f.b2 < 0 || f.b2 >= n_nodes2 || f.b4 < 0 || f.b4 >= cap4) {
        atomicExch(err, 1);
        return;
    }
    int cand[4], kind[4];
    int nc = 0;
    const BvhNode root = nodes2[f.b2];
    const int rk = node_kind(root, n_nodes2);
    if (rk == 1) {
        cand[0] = f.b2;  // a leaf root: one leaf child
        kind[0] = 1;
        nc = 1;
    } else if (rk == 2) {
        for (int s = 0; s < 2; ++s) {
            const int k = node_kind(nodes2[root.first + s], n_nodes2);
            if (k) {
                cand[nc] = root.first + s;
                kind[nc] = k;
                ++nc;
            }
        }
        // open the interior candidate of largest surface area while there is room
        while (nc < 4) {
            int best = -1;
            float best_a = -1.0f;
            for (int k = 0; k < nc; ++k) {
                if (kind[k] != 2) continue;
                const float a = half_area(nodes2[cand[k]]);
                if (a > best_a) {
                    best_a = a;
                    best = k;
                }
            }
            if (best < 0) break;
            const int first = nodes2[cand[best]].first;
            // remove `best`, append its usable children
            for (int k = best; k + 1 < nc; ++k) {
                cand[k] = cand[k + 1];
                kind[k] = kind[k + 1];
            }
            --nc;
            for (int s = 0; s < 2; ++s) {
                const int k = node_kind(nodes2[first + s], n_nodes2);
                if (k) {
                    cand[nc] = first + s;
                    kind[nc] = k;
                    ++nc;
                }
            }
        }
    }
    int n_int = 0;
    for (int k = 0; k < nc; ++k) n_int += kind[k] == 2 ? 1 : 0;
    int base = 0, pos = 0;
    if (n_int > 0) {
        base = atomicAdd(n4, n_int);
        pos = atomicAdd(n_out, n_int);
        if (base + n_int > cap4) {
            atomicExch(err, 3);
            return;
        }
    }
    Bvh4Node o;
    int j = 0;
    for (int k = 0; k < 4; ++k) {
        if (k < nc) {
            const BvhNode c = nodes2[cand[k]];
            o.lo_x[k] = c.lo_x; o.hi_x[k] = c.hi_x;
            o.lo_y[k] = c.lo_y; o.hi_y[k] = c.hi_y;
            o.lo_z[k] = c.lo_z; o.hi_z[k] = c.hi_z;
            if (kind[k] == 1) {
                o.child[k] = c.first;
                o.count[k] = c.count;
            } else {
                o.child[k] = base + j;
                o.count[k] = 0;
                out[pos + j] = Frontier{cand[k], base + j};
                ++j;
            }
        } else {
            o.lo_x[k] = o.lo_y[k] = o.lo_z[k] = FLT_MAX;
            o.hi_x[k] = o.hi_y[k] = o.hi_z[k] = -FLT_MAX;
            o.child[k] = 0;
            o.count[k] = -1;
        }
    }
    nodes4[f.b4] = o;
}

}  // namespace

// Upper bound of four-wide nodes for n primitives (one per binary interior node).
int bvh4_node_capacity(int n_prims) { return n_prims > 1 ? n_prims : 1; }

// scratch: bvh4_scratch_bytes(n_prims).  Returns the node count (> 0) or -1 on error.
size_t bvh4_scratch_bytes(int n_prims) {
    const size_t cap = (size_t)bvh4_node_capacity(n_prims);
    return 2 * cap * sizeof(Frontier) + 256;
}

int bvh4_collapse(const BvhNode *nodes2, int n_nodes2, Bvh4Node *nodes4, int cap4, void *scratch,
                  cudaStream_t stream) {
    Frontier *fa = (Frontier *)scratch;
    Frontier *fb = fa + cap4;
    int *counters = (int *)(fb + cap4);  // [0] n_in, [1] n_out, [2] n4, [3] err
    const int init[4] = {1, 0, 1, 0};
    const Frontier root{0, 0};
    cudaMemcpyAsync(counters, init, sizeof(init), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(fa, &root, sizeof(root), cudaMemcpyHostToDevice, stream);
    int n_in = 1;
    for (int level = 0; level < 128 && n_in > 0; ++level) {
        collapse_level<<<(n_in + 255) / 256, 256, 0, stream>>>(nodes2, n_nodes2, fa, counters + 0, fb, counters + 1,
                                                               nodes4, counters + 2, cap4, counters + 3);
        // next frontier: out -> in
        cudaMemcpyAsync(counters + 0, counters + 1, sizeof(int), cudaMemcpyDeviceToDevice, stream);
        cudaMemsetAsync(counters + 1, 0, sizeof(int), stream);
        cudaMemcpyAsync(&n_in, counters + 0, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
        Frontier *t = fa;
        fa = fb;
        fb = t;
    }
    int h[4];
    cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
    if (h[3] != 0 || n_in != 0) return -1;
    return h[2];
}

}  // namespace rumi
