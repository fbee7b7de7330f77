// On-device binned-SAH BVH build into 32-byte nodes.
//
// The reference builds an object-median BVH on the host (src/Acceleration/bvh.cpp:48-148:
// longest axis, shell sort, split at the middle index, leaves of <= 6).  Only the hits a
// BVH produces are observable, so this builder uses the surface area heuristic instead,
// entirely on the GPU and deterministically (same input -> same tree):
//
//  large phase (tasks with > SMALL_MAX primitives), one level per iteration:
//    make_chunks   one block: chunk list (CHUNK primitives each); reset_bins: empty bins
//                  for every task
//    bin           one block per chunk: 3 axes x 32 centroid bins in shared memory,
//                  merged into the task's bins with global atomics (ordered-int floats)
//    split         one warp per task, lane = bin: prefix/suffix scans, SAH argmin
//    count/scan/scatter  stable partition: per-chunk left counts, per-task scan,
//                  per-chunk block scan + scatter; child bounds by block reduction
//    emit          child nodes + next-level tasks, or small tasks
//  small phase: one warp per task with <= SMALL_MAX primitives builds its whole subtree
//    in shared memory (binned SAH, ballot-based stable partition, explicit stack),
//    allocating node pairs from a range reserved by its primitive range.
//
// Node index space: [0] root, [1] unused (pairs start 64-byte aligned), small-phase
// region [2, 2 + 2N), large-phase region after it.
#include "bvh_build.h"
#include <cstdio>

namespace rumi {

static constexpr int NBINS = 32;
static constexpr int CHUNK = 2048;
static constexpr int BIN_THREADS = 256;
static constexpr int SMALL_MAX = 256;
// Leaf size cap and SAH traversal cost (relative to one primitive test).  Measured on the
// 1024x1024x64 BVH-bound frame (ms): cap 8 / C_TRAV 1: 239; cap 16 / 1: 239; 16 / 1.5: 250;
// 16, 24 or 32 / 2: 225.5; 16 / 3: 231; 8 / 2: 250 (larger leaves pay only when the cap
// lets the SAH form them).
#ifndef RUMI_LEAF_MAX
#define RUMI_LEAF_MAX 16
#endif
static constexpr int LEAF_MAX = RUMI_LEAF_MAX;
static constexpr int MEDIAN_DEPTH = 40;    // past this depth split at the index median
static constexpr int MAX_DEPTH = 63;       // deepest node (traversal stack holds 64)
#ifndef RUMI_SAH_CTRAV
#define RUMI_SAH_CTRAV 2.0f
#endif
static constexpr float C_TRAV = RUMI_SAH_CTRAV;
static constexpr float C_ISECT = 1.0f;

struct BuildTask {
    int first, count, node, depth;
};

struct Bounds12 {  // ordered ints: aabb lo/hi, centroid lo/hi
    int v[12];
};

// --------------------------------------------------------------------- helpers
__device__ __forceinline__ float area_of(float3 lo, float3 hi) {
    float3 e = hi - lo;
    if (e.x < 0.0f || e.y < 0.0f || e.z < 0.0f) return 0.0f;
    return 2.0f * (e.x * e.y + e.x * e.z + e.y * e.z);
}

__device__ __forceinline__ void pad_bounds(float3 &lo, float3 &hi) {
    // conservative padding so the float slab test never rejects a surface lying on a
    // box face
    const float ex = fmaxf(fabsf(lo.x), fabsf(hi.x)) * 9.5367431640625e-7f + 1e-30f;
    const float ey = fmaxf(fabsf(lo.y), fabsf(hi.y)) * 9.5367431640625e-7f + 1e-30f;
    const float ez = fmaxf(fabsf(lo.z), fabsf(hi.z)) * 9.5367431640625e-7f + 1e-30f;
    lo = mk3(lo.x - ex, lo.y - ey, lo.z - ez);
    hi = mk3(hi.x + ex, hi.y + ey, hi.z + ez);
}

__device__ __forceinline__ void write_node_bounds(BvhNode *nodes, int n, float3 lo, float3 hi) {
    pad_bounds(lo, hi);
    BvhNode &nd = nodes[n];
    nd.lo_x = lo.x; nd.lo_y = lo.y; nd.lo_z = lo.z;
    nd.hi_x = hi.x; nd.hi_y = hi.y; nd.hi_z = hi.z;
}

__device__ __forceinline__ int bin_of(float c, float cmin, float scale) {
    int b = (int)((c - cmin) * scale);
    return b < 0 ? 0 : (b >= NBINS ? NBINS - 1 : b);
}

__device__ __forceinline__ float3 centroid(float4 lo, float4 hi) {
    return mk3((lo.x + hi.x) * 0.5f, (lo.y + hi.y) * 0.5f, (lo.z + hi.z) * 0.5f);
}

// ------------------------------------------------------------ primitive setup
// Bounds of every canonical primitive (from the original vertices, so they contain the
// triangle however its edges round) and its 48-byte intersection record.
__global__ void prim_prepare_kernel(const float *tri_v, int n_tris, const float4 *rects, int n_rects,
                                    const float4 *spheres, const int *prim_flags, int n_spheres,
                                    float4 *aabb_lo, float4 *aabb_hi, float4 *prims) {
    const int N = n_tris + n_rects + n_spheres;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        float3 lo, hi;
        float4 A, B, C;
        if (i < n_tris) {
            const float *t = tri_v + 9 * (size_t)i;
            float3 v0 = mk3(t[0], t[1], t[2]), v1 = mk3(t[3], t[4], t[5]), v2 = mk3(t[6], t[7], t[8]);
            lo = mk3(fminf(v0.x, fminf(v1.x, v2.x)), fminf(v0.y, fminf(v1.y, v2.y)), fminf(v0.z, fminf(v1.z, v2.z)));
            hi = mk3(fmaxf(v0.x, fmaxf(v1.x, v2.x)), fmaxf(v0.y, fmaxf(v1.y, v2.y)), fmaxf(v0.z, fmaxf(v1.z, v2.z)));
            float3 e1 = rn_sub(v1, v0), e2 = rn_sub(v2, v0);
            A = make_float4(v0.x, v0.y, v0.z, __int_as_float(i));
            B = make_float4(e1.x, e1.y, e1.z, __int_as_float(PRIM_TRI));
            C = make_float4(e2.x, e2.y, e2.z, 0.0f);
        } else if (i < n_tris + n_rects) {
            const int r = i - n_tris;
            float4 p = rects[3 * r], l = rects[3 * r + 1], w = rects[3 * r + 2];
            float3 q = mk3(p.x + l.x + w.x, p.y + l.y + w.y, p.z + l.z + w.z);
            float3 pl = mk3(p.x + l.x, p.y + l.y, p.z + l.z), pw = mk3(p.x + w.x, p.y + w.y, p.z + w.z);
            lo = mk3(fminf(fminf(p.x, q.x), fminf(pl.x, pw.x)), fminf(fminf(p.y, q.y), fminf(pl.y, pw.y)),
                     fminf(fminf(p.z, q.z), fminf(pl.z, pw.z)));
            hi = mk3(fmaxf(fmaxf(p.x, q.x), fmaxf(pl.x, pw.x)), fmaxf(fmaxf(p.y, q.y), fmaxf(pl.y, pw.y)),
                     fmaxf(fmaxf(p.z, q.z), fmaxf(pl.z, pw.z)));
            A = make_float4(p.x, p.y, p.z, __int_as_float(i));
            B = make_float4(l.x, l.y, l.z, __int_as_float(PRIM_RECT | (prim_flags[r] ? PRIM_FLAG_EMISSIVE : 0)));
            C = make_float4(w.x, w.y, w.z, 0.0f);
        } else {
            const int s = i - n_tris - n_rects;
            float4 c = spheres[s];
            lo = mk3(c.x - c.w, c.y - c.w, c.z - c.w);
            hi = mk3(c.x + c.w, c.y + c.w, c.z + c.w);
            A = make_float4(c.x, c.y, c.z, __int_as_float(i));
            B = make_float4(c.w, 0.0f, 0.0f,
                            __int_as_float(PRIM_SPHERE | (prim_flags[n_rects + s] ? PRIM_FLAG_IBL : 0)));
            C = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        aabb_lo[i] = make_float4(lo.x, lo.y, lo.z, 0.0f);
        aabb_hi[i] = make_float4(hi.x, hi.y, hi.z, 0.0f);
        prims[3 * (size_t)i + 0] = A;
        prims[3 * (size_t)i + 1] = B;
        prims[3 * (size_t)i + 2] = C;
    }
}

__global__ void iota_kernel(int *idx, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) idx[i] = i;
}

// Root bounds + root task (one block).
__global__ void root_kernel(const float4 *aabb_lo, const float4 *aabb_hi, int n, BvhNode *nodes,
                            BuildTask *large, int *n_large, BuildTask *small, int *n_small) {
    __shared__ float red[6][32];
    float3 lo = mk3(INFINITY, INFINITY, INFINITY), hi = mk3(-INFINITY, -INFINITY, -INFINITY);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        float4 a = aabb_lo[i], b = aabb_hi[i];
        lo = mk3(fminf(lo.x, a.x), fminf(lo.y, a.y), fminf(lo.z, a.z));
        hi = mk3(fmaxf(hi.x, b.x), fmaxf(hi.y, b.y), fmaxf(hi.z, b.z));
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo.x = fminf(lo.x, __shfl_xor_sync(0xffffffffu, lo.x, o));
        lo.y = fminf(lo.y, __shfl_xor_sync(0xffffffffu, lo.y, o));
        lo.z = fminf(lo.z, __shfl_xor_sync(0xffffffffu, lo.z, o));
        hi.x = fmaxf(hi.x, __shfl_xor_sync(0xffffffffu, hi.x, o));
        hi.y = fmaxf(hi.y, __shfl_xor_sync(0xffffffffu, hi.y, o));
        hi.z = fmaxf(hi.z, __shfl_xor_sync(0xffffffffu, hi.z, o));
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0) {
        red[0][w] = lo.x; red[1][w] = lo.y; red[2][w] = lo.z;
        red[3][w] = hi.x; red[4][w] = hi.y; red[5][w] = hi.z;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < nw; ++k) {
            lo.x = fminf(lo.x, red[0][k]); lo.y = fminf(lo.y, red[1][k]); lo.z = fminf(lo.z, red[2][k]);
            hi.x = fmaxf(hi.x, red[3][k]); hi.y = fmaxf(hi.y, red[4][k]); hi.z = fmaxf(hi.z, red[5][k]);
        }
        if (n == 0) {
            BvhNode &r = nodes[0];
            r.lo_x = r.lo_y = r.lo_z = INFINITY;
            r.hi_x = r.hi_y = r.hi_z = -INFINITY;
            r.first = 0;
            r.count = 1;  // an empty leaf that is never entered
            *n_large = 0;
            *n_small = 0;
            return;
        }
        write_node_bounds(nodes, 0, lo, hi);
        nodes[1] = nodes[0];
        nodes[1].count = -1;  // unused slot
        BuildTask t;
        t.first = 0; t.count = n; t.node = 0; t.depth = 0;
        if (n > SMALL_MAX) {
            large[0] = t;
            *n_large = 1;
            *n_small = 0;
        } else {
            small[0] = t;
            *n_small = 1;
            *n_large = 0;
        }
    }
}

// ------------------------------------------------------------- large phase
struct ChunkInfo {
    int task;
    int start;   // absolute index into idx
    int len;
};

// One block: chunk list for this level's tasks, bins reset, per-task centroid bounds
// (taken from the task's node box is not enough -- centroid bounds come from cb).
__global__ void make_chunks_kernel(const BuildTask *tasks, const int *n_tasks_p, ChunkInfo *chunks, int *n_chunks,
                                   int *bins /*[task][3][NBINS][7]*/) {
    __shared__ int s_scan[1024];
    __shared__ int s_base;
    const int n_tasks = *n_tasks_p;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (int t0 = 0; t0 < n_tasks; t0 += blockDim.x) {
        const int t = t0 + threadIdx.x;
        const int nc = t < n_tasks ? (tasks[t].count + CHUNK - 1) / CHUNK : 0;
        s_scan[threadIdx.x] = nc;
        __syncthreads();
        for (int o = 1; o < blockDim.x; o <<= 1) {
            int v = threadIdx.x >= o ? s_scan[threadIdx.x - o] : 0;
            __syncthreads();
            s_scan[threadIdx.x] += v;
            __syncthreads();
        }
        const int excl = s_scan[threadIdx.x] - nc + s_base;
        if (t < n_tasks) {
            const BuildTask tk = tasks[t];
            for (int c = 0; c < nc; ++c) {
                ChunkInfo ci;
                ci.task = t;
                ci.start = tk.first + c * CHUNK;
                ci.len = min(CHUNK, tk.count - c * CHUNK);
                chunks[excl + c] = ci;
            }
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_base = excl + nc;
        __syncthreads();
    }
    if (threadIdx.x == 0) *n_chunks = s_base;
}

// Empty bins for every task of the level (count 0, bounds +inf / -inf as ordered ints),
// grid-stride: a level can hold thousands of tasks.
__global__ void reset_bins_kernel(const int *n_tasks_p, int *bins /*[task][3][NBINS][7]*/) {
    const int n = *n_tasks_p * 3 * NBINS;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int *b = bins + 7 * (size_t)i;
        b[0] = 0;
        b[1] = b[2] = b[3] = f2o(INFINITY);
        b[4] = b[5] = b[6] = f2o(-INFINITY);
    }
}

// centroid bounds of each task, stored as ordered ints in cb[task][6]
__global__ void bin_kernel(const ChunkInfo *chunks, const int *n_chunks, const int *idx, const float4 *aabb_lo,
                           const float4 *aabb_hi, const int *cb, int *bins) {
    __shared__ int s_bins[3 * NBINS * 7];
    const int c = blockIdx.x;
    if (c >= *n_chunks) return;
    const ChunkInfo ci = chunks[c];
    for (int i = threadIdx.x; i < 3 * NBINS; i += blockDim.x) {
        s_bins[7 * i + 0] = 0;
        s_bins[7 * i + 1] = s_bins[7 * i + 2] = s_bins[7 * i + 3] = f2o(INFINITY);
        s_bins[7 * i + 4] = s_bins[7 * i + 5] = s_bins[7 * i + 6] = f2o(-INFINITY);
    }
    __syncthreads();
    const int *tcb = cb + 6 * ci.task;
    const float cmin[3] = {o2f(tcb[0]), o2f(tcb[1]), o2f(tcb[2])};
    const float cmax[3] = {o2f(tcb[3]), o2f(tcb[4]), o2f(tcb[5])};
    float scale[3];
    for (int a = 0; a < 3; ++a) {
        const float ext = cmax[a] - cmin[a];
        scale[a] = ext > 0.0f ? (float)NBINS * (1.0f - 1e-6f) / ext : 0.0f;
    }
    for (int k = threadIdx.x; k < ci.len; k += blockDim.x) {
        const int p = idx[ci.start + k];
        const float4 lo = aabb_lo[p], hi = aabb_hi[p];
        const float3 cc = centroid(lo, hi);
        const float cv[3] = {cc.x, cc.y, cc.z};
        for (int a = 0; a < 3; ++a) {
            int *b = s_bins + 7 * (a * NBINS + bin_of(cv[a], cmin[a], scale[a]));
            atomicAdd(b, 1);
            atomicMin(b + 1, f2o(lo.x)); atomicMin(b + 2, f2o(lo.y)); atomicMin(b + 3, f2o(lo.z));
            atomicMax(b + 4, f2o(hi.x)); atomicMax(b + 5, f2o(hi.y)); atomicMax(b + 6, f2o(hi.z));
        }
    }
    __syncthreads();
    int *gb = bins + (size_t)ci.task * 3 * NBINS * 7;
    for (int i = threadIdx.x; i < 3 * NBINS; i += blockDim.x) {
        const int *b = s_bins + 7 * i;
        if (b[0] == 0) continue;
        int *g = gb + 7 * i;
        atomicAdd(g, b[0]);
        atomicMin(g + 1, b[1]); atomicMin(g + 2, b[2]); atomicMin(g + 3, b[3]);
        atomicMax(g + 4, b[4]); atomicMax(g + 5, b[5]); atomicMax(g + 6, b[6]);
    }
}

struct SplitDecision {
    int axis;   // -1: index-median split
    int bin;    // primitives with bin <= this go left
    int nleft;
};

// Warp-level SAH sweep over 32 bins of three axes: lane j owns bin j.  Returns the best
// (cost, axis, bin, nleft) in every lane; cost = INF when no bin split separates anything.
__device__ void warp_sah(const int *bins /* [3][NBINS][7] */, float &best_cost, int &best_axis, int &best_bin,
                         int &best_nleft) {
    const int lane = threadIdx.x & 31;
    best_cost = INFINITY;
    best_axis = -1;
    best_bin = 0;
    best_nleft = 0;
    for (int a = 0; a < 3; ++a) {
        const int *b = bins + 7 * (a * NBINS + lane);
        int cnt = b[0];
        float lx = o2f(b[1]), ly = o2f(b[2]), lz = o2f(b[3]);
        float hx = o2f(b[4]), hy = o2f(b[5]), hz = o2f(b[6]);
        // inclusive prefix (left side ending at bin lane)
        int pc = cnt;
        float plx = lx, ply = ly, plz = lz, phx = hx, phy = hy, phz = hz;
        for (int o = 1; o < 32; o <<= 1) {
            int c2 = __shfl_up_sync(0xffffffffu, pc, o);
            float a0 = __shfl_up_sync(0xffffffffu, plx, o), a1 = __shfl_up_sync(0xffffffffu, ply, o);
            float a2 = __shfl_up_sync(0xffffffffu, plz, o), a3 = __shfl_up_sync(0xffffffffu, phx, o);
            float a4 = __shfl_up_sync(0xffffffffu, phy, o), a5 = __shfl_up_sync(0xffffffffu, phz, o);
            if (lane >= o) {
                pc += c2;
                plx = fminf(plx, a0); ply = fminf(ply, a1); plz = fminf(plz, a2);
                phx = fmaxf(phx, a3); phy = fmaxf(phy, a4); phz = fmaxf(phz, a5);
            }
        }
        // inclusive suffix (right side starting at bin lane)
        int sc = cnt;
        float slx = lx, sly = ly, slz = lz, shx = hx, shy = hy, shz = hz;
        for (int o = 1; o < 32; o <<= 1) {
            int c2 = __shfl_down_sync(0xffffffffu, sc, o);
            float a0 = __shfl_down_sync(0xffffffffu, slx, o), a1 = __shfl_down_sync(0xffffffffu, sly, o);
            float a2 = __shfl_down_sync(0xffffffffu, slz, o), a3 = __shfl_down_sync(0xffffffffu, shx, o);
            float a4 = __shfl_down_sync(0xffffffffu, shy, o), a5 = __shfl_down_sync(0xffffffffu, shz, o);
            if (lane + o < 32) {
                sc += c2;
                slx = fminf(slx, a0); sly = fminf(sly, a1); slz = fminf(slz, a2);
                shx = fmaxf(shx, a3); shy = fmaxf(shy, a4); shz = fmaxf(shz, a5);
            }
        }
        // right side of a split after bin lane = suffix of lane+1
        int rc = __shfl_down_sync(0xffffffffu, sc, 1);
        float r0 = __shfl_down_sync(0xffffffffu, slx, 1), r1 = __shfl_down_sync(0xffffffffu, sly, 1);
        float r2 = __shfl_down_sync(0xffffffffu, slz, 1), r3 = __shfl_down_sync(0xffffffffu, shx, 1);
        float r4 = __shfl_down_sync(0xffffffffu, shy, 1), r5 = __shfl_down_sync(0xffffffffu, shz, 1);
        float cost = INFINITY;
        if (lane < 31 && pc > 0 && rc > 0) {
            cost = area_of(mk3(plx, ply, plz), mk3(phx, phy, phz)) * (float)pc +
                   area_of(mk3(r0, r1, r2), mk3(r3, r4, r5)) * (float)rc;
        }
        // warp argmin (ties -> lowest lane)
        float bc = cost;
        int bl = lane;
        for (int o = 16; o > 0; o >>= 1) {
            float oc = __shfl_xor_sync(0xffffffffu, bc, o);
            int ol = __shfl_xor_sync(0xffffffffu, bl, o);
            if (oc < bc || (oc == bc && ol < bl)) {
                bc = oc;
                bl = ol;
            }
        }
        const int nl = __shfl_sync(0xffffffffu, pc, bl);
        if (bc < best_cost) {
            best_cost = bc;
            best_axis = a;
            best_bin = bl;
            best_nleft = nl;
        }
    }
}

__global__ void split_kernel(const BuildTask *tasks, const int *n_tasks, const int *bins, const BvhNode *nodes,
                             SplitDecision *dec) {
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= *n_tasks) return;
    const BuildTask tk = tasks[t];
    float cost;
    int axis, bin, nl;
    warp_sah(bins + (size_t)t * 3 * NBINS * 7, cost, axis, bin, nl);
    if ((threadIdx.x & 31) == 0) {
        SplitDecision d;
        if (axis < 0 || tk.depth >= MEDIAN_DEPTH) {
            d.axis = -1;
            d.bin = 0;
            d.nleft = tk.count / 2;
        } else {
            d.axis = axis;
            d.bin = bin;
            d.nleft = nl;
        }
        dec[t] = d;
    }
}

__device__ __forceinline__ bool goes_left(const SplitDecision &d, int pos_in_task, float3 c, const int *tcb) {
    if (d.axis < 0) return pos_in_task < d.nleft;
    const float cv = d.axis == 0 ? c.x : (d.axis == 1 ? c.y : c.z);
    const float cmin = o2f(tcb[d.axis]), cmax = o2f(tcb[3 + d.axis]);
    const float ext = cmax - cmin;
    const float scale = ext > 0.0f ? (float)NBINS * (1.0f - 1e-6f) / ext : 0.0f;
    return bin_of(cv, cmin, scale) <= d.bin;
}

static constexpr int PER_THREAD = CHUNK / BIN_THREADS;

__global__ void count_kernel(const ChunkInfo *chunks, const int *n_chunks, const BuildTask *tasks,
                             const SplitDecision *dec, const int *idx, const float4 *aabb_lo, const float4 *aabb_hi,
                             const int *cb, int *chunk_left) {
    __shared__ int s_red[BIN_THREADS / 32];
    const int c = blockIdx.x;
    if (c >= *n_chunks) return;
    const ChunkInfo ci = chunks[c];
    const BuildTask tk = tasks[ci.task];
    const SplitDecision d = dec[ci.task];
    const int *tcb = cb + 6 * ci.task;
    int cnt = 0;
    for (int k = threadIdx.x; k < ci.len; k += blockDim.x) {
        const int pos = ci.start + k;
        const int p = idx[pos];
        const float3 cc = centroid(aabb_lo[p], aabb_hi[p]);
        cnt += goes_left(d, pos - tk.first, cc, tcb) ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int i = 0; i < BIN_THREADS / 32; ++i) s += s_red[i];
        chunk_left[c] = s;
    }
}

// One warp per task: exclusive scan of its chunks' left counts (chunks of a task are
// consecutive in the chunk list).
__global__ void chunk_scan_kernel(const ChunkInfo *chunks, const int *n_chunks, const int *n_tasks,
                                  const int *chunk_left, int *chunk_loff, const int *task_first_chunk,
                                  SplitDecision *dec) {
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= *n_tasks) return;
    const int c0 = task_first_chunk[t];
    const int nch = *n_chunks;
    int running = 0;
    for (int base = c0;; base += 32) {
        const int c = base + lane;
        const bool valid = c < nch && chunks[c].task == t;
        int v = valid ? chunk_left[c] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            int x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += x;
        }
        if (valid) chunk_loff[c] = running + incl - v;
        running += __shfl_sync(0xffffffffu, incl, 31);
        const unsigned any_invalid = __ballot_sync(0xffffffffu, !valid);
        if (any_invalid) break;
    }
    if (lane == 0) dec[t].nleft = running;  // exact left count of the partition
}

__global__ void task_first_chunk_kernel(const ChunkInfo *chunks, const int *n_chunks, int *task_first_chunk) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= *n_chunks) return;
    const int t = chunks[c].task;
    if (c == 0 || chunks[c - 1].task != t) task_first_chunk[t] = c;
}

__global__ void scatter_kernel(const ChunkInfo *chunks, const int *n_chunks, const BuildTask *tasks,
                               const SplitDecision *dec, const int *idx, int *idx_tmp, const float4 *aabb_lo,
                               const float4 *aabb_hi, const int *cb, const int *chunk_loff, int *child_bounds) {
    __shared__ int s_scan[BIN_THREADS];
    __shared__ int s_b[2][12][BIN_THREADS / 32];
    const int c = blockIdx.x;
    if (c >= *n_chunks) return;
    const ChunkInfo ci = chunks[c];
    const BuildTask tk = tasks[ci.task];
    const SplitDecision d = dec[ci.task];
    const int *tcb = cb + 6 * ci.task;
    const int k0 = threadIdx.x * PER_THREAD;
    int pidx[PER_THREAD];
    bool left[PER_THREAD];
    int nl = 0;
    float bl[2][12];
    for (int s = 0; s < 2; ++s)
        for (int j = 0; j < 12; ++j) bl[s][j] = (j % 6) < 3 ? INFINITY : -INFINITY;
    for (int k = 0; k < PER_THREAD; ++k) {
        const int kk = k0 + k;
        left[k] = false;
        pidx[k] = -1;
        if (kk < ci.len) {
            const int pos = ci.start + kk;
            const int p = idx[pos];
            const float4 lo = aabb_lo[p], hi = aabb_hi[p];
            const float3 cc = centroid(lo, hi);
            const bool L = goes_left(d, pos - tk.first, cc, tcb);
            pidx[k] = p;
            left[k] = L;
            nl += L;
            float *b = bl[L ? 0 : 1];
            b[0] = fminf(b[0], lo.x); b[1] = fminf(b[1], lo.y); b[2] = fminf(b[2], lo.z);
            b[3] = fmaxf(b[3], hi.x); b[4] = fmaxf(b[4], hi.y); b[5] = fmaxf(b[5], hi.z);
            b[6] = fminf(b[6], cc.x); b[7] = fminf(b[7], cc.y); b[8] = fminf(b[8], cc.z);
            b[9] = fmaxf(b[9], cc.x); b[10] = fmaxf(b[10], cc.y); b[11] = fmaxf(b[11], cc.z);
        }
    }
    // block exclusive scan of nl
    s_scan[threadIdx.x] = nl;
    __syncthreads();
    for (int o = 1; o < BIN_THREADS; o <<= 1) {
        int v = threadIdx.x >= o ? s_scan[threadIdx.x - o] : 0;
        __syncthreads();
        s_scan[threadIdx.x] += v;
        __syncthreads();
    }
    const int lrank = s_scan[threadIdx.x] - nl;
    const int chunk_off = ci.start - tk.first;          // primitives of this task before the chunk
    const int loff = chunk_loff[c];
    const int roff = chunk_off - loff;                  // right primitives before the chunk
    const int my_off = k0;                              // primitives of this chunk before my first
    int li = lrank, ri = my_off - lrank;
    for (int k = 0; k < PER_THREAD; ++k) {
        if (pidx[k] < 0) continue;
        int dst;
        if (left[k])
            dst = tk.first + loff + li++;
        else
            dst = tk.first + d.nleft + roff + ri++;
        if (dst >= tk.first && dst < tk.first + tk.count) idx_tmp[dst] = pidx[k];
    }
    // child bounds: warp reduce then block reduce then global atomics
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int s = 0; s < 2; ++s)
        for (int j = 0; j < 12; ++j) {
            float v = bl[s][j];
            const bool mx = (j % 6) >= 3;
            for (int o = 16; o > 0; o >>= 1) {
                float x = __shfl_xor_sync(0xffffffffu, v, o);
                v = mx ? fmaxf(v, x) : fminf(v, x);
            }
            if (lane == 0) s_b[s][j][w] = __float_as_int(v);
        }
    __syncthreads();
    if (threadIdx.x < 24) {
        const int s = threadIdx.x / 12, j = threadIdx.x % 12;
        const bool mx = (j % 6) >= 3;
        float v = __int_as_float(s_b[s][j][0]);
        for (int i = 1; i < BIN_THREADS / 32; ++i) {
            float x = __int_as_float(s_b[s][j][i]);
            v = mx ? fmaxf(v, x) : fminf(v, x);
        }
        int *g = child_bounds + 12 * (2 * ci.task + s) + j;
        if (mx)
            atomicMax(g, f2o(v));
        else
            atomicMin(g, f2o(v));
    }
}

__global__ void copy_back_kernel(const ChunkInfo *chunks, const int *n_chunks, const int *idx_tmp, int *idx) {
    const int c = blockIdx.x;
    if (c >= *n_chunks) return;
    const ChunkInfo ci = chunks[c];
    for (int k = threadIdx.x; k < ci.len; k += blockDim.x) idx[ci.start + k] = idx_tmp[ci.start + k];
}

__global__ void reset_child_bounds_kernel(int *child_bounds, const int *n_tasks) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * (*n_tasks) * 12) return;
    const int j = i % 12;
    child_bounds[i] = ((j % 6) < 3) ? f2o(INFINITY) : f2o(-INFINITY);
}

// Children of every large task: node pair, bounds, next tasks.  Large children go to
// slot 2t+s of a sparse array (compacted in order afterwards, so the next level's task
// order -- and with it the node layout -- is deterministic); small children are
// appended with an atomic counter (their processing order does not matter: each small
// subtree writes only the node range reserved by its primitive range).
__global__ void emit_kernel(const BuildTask *tasks, const int *n_tasks, const SplitDecision *dec,
                            const int *child_bounds, BvhNode *nodes, int pair_base, BuildTask *sparse,
                            int *sparse_cb, BuildTask *small, int *n_small) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *n_tasks) return;
    const BuildTask tk = tasks[t];
    const SplitDecision d = dec[t];
    const int pair = pair_base + 2 * t;
    nodes[tk.node].first = pair;
    nodes[tk.node].count = 0;
    for (int s = 0; s < 2; ++s) {
        const int *b = child_bounds + 12 * (2 * t + s);
        const int node = pair + s;
        write_node_bounds(nodes, node, mk3(o2f(b[0]), o2f(b[1]), o2f(b[2])), mk3(o2f(b[3]), o2f(b[4]), o2f(b[5])));
        nodes[node].first = 0;
        nodes[node].count = 0;
        BuildTask ch;
        ch.first = s == 0 ? tk.first : tk.first + d.nleft;
        ch.count = s == 0 ? d.nleft : tk.count - d.nleft;
        ch.node = node;
        ch.depth = tk.depth + 1;
        BuildTask sl = ch;
        if (ch.count > SMALL_MAX) {
            for (int j = 0; j < 6; ++j) sparse_cb[6 * (2 * t + s) + j] = b[6 + j];
        } else {
            const int k = atomicAdd(n_small, 1);
            small[k] = ch;
            sl.count = 0;
        }
        sparse[2 * t + s] = sl;
    }
}

// One block: ordered compaction of the sparse child slots into the next level's tasks.
__global__ void compact_next_kernel(const BuildTask *sparse, const int *sparse_cb, const int *n_tasks_p,
                                    BuildTask *next, int *next_cb, int *n_next) {
    __shared__ int s_scan[1024];
    __shared__ int s_base;
    const int m = 2 * (*n_tasks_p);
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (int i0 = 0; i0 < m; i0 += blockDim.x) {
        const int i = i0 + threadIdx.x;
        const int f = (i < m && sparse[i].count > 0) ? 1 : 0;
        s_scan[threadIdx.x] = f;
        __syncthreads();
        for (int o = 1; o < blockDim.x; o <<= 1) {
            int v = threadIdx.x >= o ? s_scan[threadIdx.x - o] : 0;
            __syncthreads();
            s_scan[threadIdx.x] += v;
            __syncthreads();
        }
        const int base = s_base;
        const int dst = base + s_scan[threadIdx.x] - f;
        if (f) {
            next[dst] = sparse[i];
            for (int j = 0; j < 6; ++j) next_cb[6 * dst + j] = sparse_cb[6 * i + j];
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_base = base + s_scan[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) *n_next = s_base;
}

// ------------------------------------------------------------- small phase
static constexpr int SMALL_WARPS = 4;
static constexpr int SMALL_STACK = 24;

__global__ void __launch_bounds__(32 * SMALL_WARPS) small_build_kernel(const BuildTask *small, const int *n_small,
                                                                        int *idx, const float4 *aabb_lo,
                                                                        const float4 *aabb_hi, BvhNode *nodes,
                                                                        int small_region, int *error_flag) {
    __shared__ int s_idx[SMALL_WARPS][SMALL_MAX];
    __shared__ int s_tmp[SMALL_WARPS][SMALL_MAX];
    __shared__ int s_bins[SMALL_WARPS][3 * NBINS * 7];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x * SMALL_WARPS + w;
    if (t >= *n_small) return;
    const BuildTask root = small[t];
    int *sidx = s_idx[w];
    int *stmp = s_tmp[w];
    int *sb = s_bins[w];
    for (int k = lane; k < root.count; k += 32) sidx[k] = idx[root.first + k];
    __syncwarp();
    int alloc = small_region + 2 * root.first;  // reserved pairs for this subtree
    // stack entries: off, count, node, depth
    int st_off[SMALL_STACK], st_cnt[SMALL_STACK], st_node[SMALL_STACK], st_dep[SMALL_STACK];
    int sp = 0;
    int off = 0, cnt = root.count, node = root.node, dep = root.depth;
    for (;;) {
        // centroid bounds of this sub-range
        float3 cmn = mk3(INFINITY, INFINITY, INFINITY), cmx = mk3(-INFINITY, -INFINITY, -INFINITY);
        for (int k = lane; k < cnt; k += 32) {
            const int p = sidx[off + k];
            const float3 c = centroid(aabb_lo[p], aabb_hi[p]);
            cmn = mk3(fminf(cmn.x, c.x), fminf(cmn.y, c.y), fminf(cmn.z, c.z));
            cmx = mk3(fmaxf(cmx.x, c.x), fmaxf(cmx.y, c.y), fmaxf(cmx.z, c.z));
        }
        for (int o = 16; o > 0; o >>= 1) {
            cmn.x = fminf(cmn.x, __shfl_xor_sync(0xffffffffu, cmn.x, o));
            cmn.y = fminf(cmn.y, __shfl_xor_sync(0xffffffffu, cmn.y, o));
            cmn.z = fminf(cmn.z, __shfl_xor_sync(0xffffffffu, cmn.z, o));
            cmx.x = fmaxf(cmx.x, __shfl_xor_sync(0xffffffffu, cmx.x, o));
            cmx.y = fmaxf(cmx.y, __shfl_xor_sync(0xffffffffu, cmx.y, o));
            cmx.z = fmaxf(cmx.z, __shfl_xor_sync(0xffffffffu, cmx.z, o));
        }
        bool make_leaf = cnt <= 1 || dep >= MAX_DEPTH;
        float best_cost = INFINITY;
        int axis = -1, bin = 0, nleft = cnt / 2;
        const float cminv[3] = {cmn.x, cmn.y, cmn.z}, cmaxv[3] = {cmx.x, cmx.y, cmx.z};
        float scale[3];
        for (int a = 0; a < 3; ++a) {
            const float ext = cmaxv[a] - cminv[a];
            scale[a] = ext > 0.0f ? (float)NBINS * (1.0f - 1e-6f) / ext : 0.0f;
        }
        if (!make_leaf) {
            for (int i = lane; i < 3 * NBINS; i += 32) {
                sb[7 * i + 0] = 0;
                sb[7 * i + 1] = sb[7 * i + 2] = sb[7 * i + 3] = f2o(INFINITY);
                sb[7 * i + 4] = sb[7 * i + 5] = sb[7 * i + 6] = f2o(-INFINITY);
            }
            __syncwarp();
            for (int k = lane; k < cnt; k += 32) {
                const int p = sidx[off + k];
                const float4 lo = aabb_lo[p], hi = aabb_hi[p];
                const float3 c = centroid(lo, hi);
                const float cv[3] = {c.x, c.y, c.z};
                for (int a = 0; a < 3; ++a) {
                    int *b = sb + 7 * (a * NBINS + bin_of(cv[a], cminv[a], scale[a]));
                    atomicAdd(b, 1);
                    atomicMin(b + 1, f2o(lo.x)); atomicMin(b + 2, f2o(lo.y)); atomicMin(b + 3, f2o(lo.z));
                    atomicMax(b + 4, f2o(hi.x)); atomicMax(b + 5, f2o(hi.y)); atomicMax(b + 6, f2o(hi.z));
                }
            }
            __syncwarp();
            int bx, bb, bn;
            warp_sah(sb, best_cost, bx, bb, bn);
            const BvhNode &nd = nodes[node];
            const float parent_area = area_of(mk3(nd.lo_x, nd.lo_y, nd.lo_z), mk3(nd.hi_x, nd.hi_y, nd.hi_z));
            if (bx >= 0 && dep < MEDIAN_DEPTH) {
                const float split_cost = C_TRAV + C_ISECT * best_cost / fmaxf(parent_area, 1e-30f);
                const float leaf_cost = C_ISECT * (float)cnt;
                if (cnt <= LEAF_MAX && leaf_cost <= split_cost) make_leaf = true;
                axis = bx;
                bin = bb;
                nleft = bn;
            } else if (cnt <= 2 || (bx < 0 && cnt <= LEAF_MAX)) {
                make_leaf = true;
            }
        }
        if (make_leaf) {
            if (lane == 0) {
                nodes[node].first = root.first + off;
                nodes[node].count = cnt;
            }
        } else {
            // stable partition of sidx[off, off+cnt) by the decision
            int lbase = 0, rbase = 0;
            for (int g = 0; g < cnt; g += 32) {
                const int k = g + lane;
                bool L = false;
                int p = -1;
                if (k < cnt) {
                    p = sidx[off + k];
                    if (axis < 0) {
                        L = k < nleft;
                    } else {
                        const float3 c = centroid(aabb_lo[p], aabb_hi[p]);
                        const float cv = axis == 0 ? c.x : (axis == 1 ? c.y : c.z);
                        L = bin_of(cv, cminv[axis], scale[axis]) <= bin;
                    }
                }
                const unsigned bl = __ballot_sync(0xffffffffu, k < cnt && L);
                const unsigned br = __ballot_sync(0xffffffffu, k < cnt && !L);
                const unsigned lt = (1u << lane) - 1u;
                if (k < cnt) {
                    const int dst = L ? off + lbase + __popc(bl & lt) : off + nleft + rbase + __popc(br & lt);
                    if (dst >= off && dst < off + cnt)
                        stmp[dst] = p;
                    else
                        atomicExch(error_flag, 2);
                }
                lbase += __popc(bl);
                rbase += __popc(br);
            }
            __syncwarp();
            for (int k = lane; k < cnt; k += 32) sidx[off + k] = stmp[off + k];
            __syncwarp();
            // child bounds
            const int pair = alloc;
            alloc += 2;
            if (pair + 1 >= small_region + 2 * (root.first + root.count)) {  // cannot happen: <= cnt-1 splits
                if (lane == 0) {
                    atomicExch(error_flag, 3);
                    nodes[node].first = root.first + off;
                    nodes[node].count = cnt;
                }
                __syncwarp();
                if (sp == 0) break;
                --sp;
                off = st_off[sp]; cnt = st_cnt[sp]; node = st_node[sp]; dep = st_dep[sp];
                continue;
            }
            for (int s = 0; s < 2; ++s) {
                const int o2 = s == 0 ? off : off + nleft;
                const int c2 = s == 0 ? nleft : cnt - nleft;
                float3 lo = mk3(INFINITY, INFINITY, INFINITY), hi = mk3(-INFINITY, -INFINITY, -INFINITY);
                for (int k = lane; k < c2; k += 32) {
                    const int p = sidx[o2 + k];
                    const float4 a = aabb_lo[p], b = aabb_hi[p];
                    lo = mk3(fminf(lo.x, a.x), fminf(lo.y, a.y), fminf(lo.z, a.z));
                    hi = mk3(fmaxf(hi.x, b.x), fmaxf(hi.y, b.y), fmaxf(hi.z, b.z));
                }
                for (int o = 16; o > 0; o >>= 1) {
                    lo.x = fminf(lo.x, __shfl_xor_sync(0xffffffffu, lo.x, o));
                    lo.y = fminf(lo.y, __shfl_xor_sync(0xffffffffu, lo.y, o));
                    lo.z = fminf(lo.z, __shfl_xor_sync(0xffffffffu, lo.z, o));
                    hi.x = fmaxf(hi.x, __shfl_xor_sync(0xffffffffu, hi.x, o));
                    hi.y = fmaxf(hi.y, __shfl_xor_sync(0xffffffffu, hi.y, o));
                    hi.z = fmaxf(hi.z, __shfl_xor_sync(0xffffffffu, hi.z, o));
                }
                if (lane == 0) {
                    write_node_bounds(nodes, pair + s, lo, hi);
                    nodes[pair + s].first = 0;
                    nodes[pair + s].count = 0;
                }
            }
            if (lane == 0) {
                nodes[node].first = pair;
                nodes[node].count = 0;
            }
            // continue with the smaller child, push the larger one
            const int lc = nleft, rc = cnt - nleft;
            const bool left_small = lc <= rc;
            const int so = left_small ? off : off + nleft, sc = left_small ? lc : rc, sn = left_small ? pair : pair + 1;
            const int bo = left_small ? off + nleft : off, bc = left_small ? rc : lc, bn = left_small ? pair + 1 : pair;
            if (sp < SMALL_STACK) {
                st_off[sp] = bo; st_cnt[sp] = bc; st_node[sp] = bn; st_dep[sp] = dep + 1;
                ++sp;
            } else {
                // cannot happen (stack depth <= log2(SMALL_MAX)); record and make a leaf
                if (lane == 0) {
                    atomicExch(error_flag, 1);
                    nodes[bn].first = root.first + bo;
                    nodes[bn].count = bc;
                }
            }
            off = so; cnt = sc; node = sn; dep = dep + 1;
            __syncwarp();
            continue;
        }
        __syncwarp();
        if (sp == 0) break;
        --sp;
        off = st_off[sp]; cnt = st_cnt[sp]; node = st_node[sp]; dep = st_dep[sp];
    }
    __syncwarp();
    for (int k = lane; k < root.count; k += 32) idx[root.first + k] = sidx[k];
}

__global__ void gather_leaf_prims_kernel(const int *idx, int n, const float4 *prims_canon, float4 *leaf_prims) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = idx[i];
        leaf_prims[3 * (size_t)i + 0] = prims_canon[3 * (size_t)p + 0];
        leaf_prims[3 * (size_t)i + 1] = prims_canon[3 * (size_t)p + 1];
        leaf_prims[3 * (size_t)i + 2] = prims_canon[3 * (size_t)p + 2];
    }
}

// Centroid bounds of the root task (ordered ints) for the first large level.
__global__ void root_cb_kernel(const float4 *aabb_lo, const float4 *aabb_hi, int n, int *cb) {
    float3 lo = mk3(INFINITY, INFINITY, INFINITY), hi = mk3(-INFINITY, -INFINITY, -INFINITY);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float3 c = centroid(aabb_lo[i], aabb_hi[i]);
        lo = mk3(fminf(lo.x, c.x), fminf(lo.y, c.y), fminf(lo.z, c.z));
        hi = mk3(fmaxf(hi.x, c.x), fmaxf(hi.y, c.y), fmaxf(hi.z, c.z));
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo.x = fminf(lo.x, __shfl_xor_sync(0xffffffffu, lo.x, o));
        lo.y = fminf(lo.y, __shfl_xor_sync(0xffffffffu, lo.y, o));
        lo.z = fminf(lo.z, __shfl_xor_sync(0xffffffffu, lo.z, o));
        hi.x = fmaxf(hi.x, __shfl_xor_sync(0xffffffffu, hi.x, o));
        hi.y = fmaxf(hi.y, __shfl_xor_sync(0xffffffffu, hi.y, o));
        hi.z = fmaxf(hi.z, __shfl_xor_sync(0xffffffffu, hi.z, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(cb + 0, f2o(lo.x)); atomicMin(cb + 1, f2o(lo.y)); atomicMin(cb + 2, f2o(lo.z));
        atomicMax(cb + 3, f2o(hi.x)); atomicMax(cb + 4, f2o(hi.y)); atomicMax(cb + 5, f2o(hi.z));
    }
}

__global__ void init_cb_kernel(int *cb) {
    if (threadIdx.x < 6) cb[threadIdx.x] = threadIdx.x < 3 ? f2o(INFINITY) : f2o(-INFINITY);
}

// ---------------------------------------------------------------- host driver
static inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

int bvh_node_capacity(int n_prims) {
    const long long n = n_prims;
    // root + pad, small region 2N, large region: <= N / SMALL_MAX tasks per level, 64 levels
    long long cap = 2 + 2 * n + 2 * (n / SMALL_MAX + 1) * 64 + 64;
    return (int)cap;
}

size_t bvh_scratch_bytes(int n_prims) {
    const size_t n = (size_t)(n_prims > 0 ? n_prims : 1);
    const size_t max_tasks = n / SMALL_MAX + 2;
    const size_t max_chunks = n / CHUNK + max_tasks + 2;
    size_t b = 0;
    auto add = [&](size_t bytes) { b += (bytes + 255) & ~(size_t)255; };
    add(n * sizeof(float4));                         // aabb_lo
    add(n * sizeof(float4));                         // aabb_hi
    add(3 * n * sizeof(float4));                     // prims_canon
    add(n * sizeof(int));                            // idx
    add(n * sizeof(int));                            // idx_tmp
    add(2 * max_tasks * sizeof(BuildTask));          // large tasks (cur, next)
    add(2 * max_tasks * 6 * sizeof(int));            // centroid bounds (cur, next)
    add((n + 1) * sizeof(BuildTask));                // small tasks
    add(max_chunks * sizeof(ChunkInfo));
    add(max_chunks * sizeof(int) * 2);               // chunk_left, chunk_loff
    add(max_tasks * sizeof(int));                    // task_first_chunk
    add(max_tasks * sizeof(SplitDecision));
    add(max_tasks * 3 * NBINS * 7 * sizeof(int));    // bins
    add(2 * max_tasks * 12 * sizeof(int));           // child bounds
    add(2 * max_tasks * sizeof(BuildTask));          // sparse next tasks
    add(2 * max_tasks * 6 * sizeof(int));            // sparse centroid bounds
    add(16 * sizeof(int));                           // counters
    return b;
}

// Builds the BVH of the canonical primitives into `nodes` (bvh_node_capacity entries)
// and `leaf_prims` (3N float4).  scratch must hold bvh_scratch_bytes(N).  Returns 0 on
// success, else a cudaError_t value (or -1 when the builder's internal bounds were hit).
int bvh_build(const float *d_tri_v, int n_tris, const float4 *d_rects, const int *d_prim_flags, int n_rects,
              const float4 *d_spheres, int n_spheres, BvhNode *nodes, float4 *leaf_prims, void *scratch,
              cudaStream_t stream, BvhBuildInfo *info) {
    const int N = n_tris + n_rects + n_spheres;
    const size_t n = (size_t)(N > 0 ? N : 1);
    const size_t max_tasks = n / SMALL_MAX + 2;
    const size_t max_chunks = n / CHUNK + max_tasks + 2;
    char *p = (char *)scratch;
    auto take = [&](size_t bytes) {
        void *r = p;
        p += (bytes + 255) & ~(size_t)255;
        return r;
    };
    float4 *aabb_lo = (float4 *)take(n * sizeof(float4));
    float4 *aabb_hi = (float4 *)take(n * sizeof(float4));
    float4 *prims_canon = (float4 *)take(3 * n * sizeof(float4));
    int *idx = (int *)take(n * sizeof(int));
    int *idx_tmp = (int *)take(n * sizeof(int));
    BuildTask *tasks[2];
    tasks[0] = (BuildTask *)take(2 * max_tasks * sizeof(BuildTask));
    tasks[1] = tasks[0] + max_tasks;
    int *cbs[2];
    cbs[0] = (int *)take(2 * max_tasks * 6 * sizeof(int));
    cbs[1] = cbs[0] + max_tasks * 6;
    BuildTask *small = (BuildTask *)take((n + 1) * sizeof(BuildTask));
    ChunkInfo *chunks = (ChunkInfo *)take(max_chunks * sizeof(ChunkInfo));
    int *chunk_left = (int *)take(max_chunks * sizeof(int) * 2);
    int *chunk_loff = chunk_left + max_chunks;
    int *task_first_chunk = (int *)take(max_tasks * sizeof(int));
    SplitDecision *dec = (SplitDecision *)take(max_tasks * sizeof(SplitDecision));
    int *bins = (int *)take(max_tasks * 3 * NBINS * 7 * sizeof(int));
    int *child_bounds = (int *)take(2 * max_tasks * 12 * sizeof(int));
    BuildTask *sparse = (BuildTask *)take(2 * max_tasks * sizeof(BuildTask));
    int *sparse_cb = (int *)take(2 * max_tasks * 6 * sizeof(int));
    int *counters = (int *)take(16 * sizeof(int));
    // counters: [0] n_large cur [1] n_large next [2] n_small [3] n_chunks [4] error
    int *n_cur = counters + 0, *n_small = counters + 2, *n_chunks = counters + 3, *err = counters + 4;

    cudaMemsetAsync(counters, 0, 16 * sizeof(int), stream);
    const int small_region = 2;
    int pair_base = small_region + 2 * (int)n;
    const int grid_n = cdiv((long long)n, 256) < 148 * 8 ? cdiv((long long)n, 256) : 148 * 8;
    prim_prepare_kernel<<<grid_n > 0 ? grid_n : 1, 256, 0, stream>>>(d_tri_v, n_tris, d_rects, n_rects, d_spheres,
                                                                     d_prim_flags, n_spheres, aabb_lo, aabb_hi,
                                                                     prims_canon);
    iota_kernel<<<grid_n > 0 ? grid_n : 1, 256, 0, stream>>>(idx, N);
    root_kernel<<<1, 1024, 0, stream>>>(aabb_lo, aabb_hi, N, nodes, tasks[0], n_cur, small, n_small);
    init_cb_kernel<<<1, 32, 0, stream>>>(cbs[0]);
    root_cb_kernel<<<grid_n > 0 ? grid_n : 1, 256, 0, stream>>>(aabb_lo, aabb_hi, N, cbs[0]);

    int cur = 0;
    int levels = 0;
    int h_n_tasks = 0;
    cudaMemcpyAsync(&h_n_tasks, n_cur, sizeof(int), cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    while (h_n_tasks > 0) {
        if (levels > 80 || (size_t)h_n_tasks > max_tasks) {
            return -1;
        }
        int *ncur = counters + 0;  // current count lives in counters[0]
        int *nnext = counters + 1;
        const int max_ch = (int)(n / CHUNK) + h_n_tasks + 1;
        make_chunks_kernel<<<1, 1024, 0, stream>>>(tasks[cur], ncur, chunks, n_chunks, bins);
        reset_bins_kernel<<<cdiv(h_n_tasks * 3 * NBINS, 256), 256, 0, stream>>>(ncur, bins);
        bin_kernel<<<max_ch, BIN_THREADS, 0, stream>>>(chunks, n_chunks, idx, aabb_lo, aabb_hi, cbs[cur], bins);
        split_kernel<<<cdiv(h_n_tasks * 32, 128), 128, 0, stream>>>(tasks[cur], ncur, bins, nodes, dec);
        count_kernel<<<max_ch, BIN_THREADS, 0, stream>>>(chunks, n_chunks, tasks[cur], dec, idx, aabb_lo, aabb_hi,
                                                         cbs[cur], chunk_left);
        task_first_chunk_kernel<<<cdiv(max_ch, 256), 256, 0, stream>>>(chunks, n_chunks, task_first_chunk);
        chunk_scan_kernel<<<cdiv(h_n_tasks * 32, 128), 128, 0, stream>>>(chunks, n_chunks, ncur, chunk_left,
                                                                         chunk_loff, task_first_chunk, dec);
        reset_child_bounds_kernel<<<cdiv(2 * h_n_tasks * 12, 256), 256, 0, stream>>>(child_bounds, ncur);
        scatter_kernel<<<max_ch, BIN_THREADS, 0, stream>>>(chunks, n_chunks, tasks[cur], dec, idx, idx_tmp, aabb_lo,
                                                           aabb_hi, cbs[cur], chunk_loff, child_bounds);
        copy_back_kernel<<<max_ch, BIN_THREADS, 0, stream>>>(chunks, n_chunks, idx_tmp, idx);
        if (pair_base + 2 * h_n_tasks > bvh_node_capacity(N)) return -1;
        emit_kernel<<<cdiv(h_n_tasks, 128), 128, 0, stream>>>(tasks[cur], ncur, dec, child_bounds, nodes, pair_base,
                                                              sparse, sparse_cb, small, n_small);
        compact_next_kernel<<<1, 1024, 0, stream>>>(sparse, sparse_cb, ncur, tasks[cur ^ 1], cbs[cur ^ 1], nnext);
        pair_base += 2 * h_n_tasks;
        // next level: its count moves into counters[0]
        cudaMemcpyAsync(ncur, nnext, sizeof(int), cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(&h_n_tasks, nnext, sizeof(int), cudaMemcpyDeviceToHost, stream);
        cudaStreamSynchronize(stream);
        cur ^= 1;
        ++levels;
    }
    int h_small = 0;
    cudaMemcpyAsync(&h_small, n_small, sizeof(int), cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    if (h_small > 0)
        small_build_kernel<<<cdiv(h_small, SMALL_WARPS), 32 * SMALL_WARPS, 0, stream>>>(
            small, n_small, idx, aabb_lo, aabb_hi, nodes, small_region, err);
    gather_leaf_prims_kernel<<<grid_n > 0 ? grid_n : 1, 256, 0, stream>>>(idx, N, prims_canon, leaf_prims);
    int h_err = 0;
    cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, stream);
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return (int)e;
    if (h_err) return -1;
    if (info) {
        info->large_levels = levels;
        info->small_tasks = h_small;
        info->node_capacity = bvh_node_capacity(N);
        info->node_high_water = pair_base;
    }
    return 0;
}

}  // namespace rumi
