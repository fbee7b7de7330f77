// Multi-scene batches (rumi_batch_* in include/rumi_b200.h): many scenes of uneven size
// and sample count rendered as one frame from shared ray queues, optionally replayed from
// a CUDA graph captured on the first frame.  Each scene keeps its own Philox key and its
// scene-local path numbering, so its image equals what rumi_render produces for it alone
// with the same seed.
#include "renderer.h"
#include <cstring>
#include <vector>

using namespace rumi;

struct rumi_batch {
    std::vector<rumi_scene *> scenes;
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t aux = nullptr;  // second stream of the two-stream schedule
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // device tables
    DevScene *d_scenes = nullptr;
    long long *d_path0 = nullptr, *d_pix0 = nullptr;
    uint32_t *d_keys = nullptr;
    int *d_spp = nullptr;
    std::vector<long long> pix0;  // n + 1 prefix of pixels
    void *ws = nullptr;
    size_t ws_bytes = 0;
    float *d_films = nullptr;     // film staging for host-film calls
    bool lean = true;             // every scene (as the table holds it) qualifies for lean shading
    // the captured frame and what it was captured for
    cudaGraphExec_t graph = nullptr;
    std::vector<int> graph_spp;
    int graph_depth = 0;
    long long graph_wave = 0;
    int graph_blocks = 0;
    float *graph_films = nullptr;
    cudaStream_t graph_stream = nullptr;
};

namespace {

void drop_graph(rumi_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

// Waves of whole pixels, contiguous in the global pixel and path index spaces, each
// holding at most `wave` paths (a pixel with more samples than that gets a wave alone).
void plan_waves(const std::vector<long long> &pix0, const std::vector<int> &spp, long long wave,
                std::vector<BatchWave> &out) {
    out.clear();
    const long long total = pix0.back();
    long long gp = 0, gpath = 0, used = 0;
    BatchWave cur{0, 0, 0, 0};
    size_t k = 0;
    while (gp < total) {
        while (pix0[k + 1] <= gp) ++k;
        long long take = (wave - used) / spp[k];
        const long long remain = pix0[k + 1] - gp;
        if (take > remain) take = remain;
        if (take <= 0) {
            if (used > 0) {
                cur.pix1 = gp;
                cur.path1 = gpath;
                out.push_back(cur);
                cur = BatchWave{gp, gp, gpath, gpath};
                used = 0;
                continue;
            }
            take = 1;
        }
        gp += take;
        gpath += take * spp[k];
        used += take * spp[k];
    }
    cur.pix1 = gp;
    cur.path1 = gpath;
    if (cur.pix1 > cur.pix0) out.push_back(cur);
}

}  // namespace

extern "C" {

rumi_status rumi_batch_create(rumi_scene *const *scenes, int32_t n, rumi_batch **out) {
    if (!out || !scenes || n <= 0) {
        set_error("rumi_batch_create: NULL argument or empty batch");
        return RUMI_ERR_INVALID_ARG;
    }
    *out = nullptr;
    int dev = 0;
    cudaGetDevice(&dev);
    for (int i = 0; i < n; ++i) {
        if (!scenes[i]) {
            set_error("rumi_batch_create: NULL scene");
            return RUMI_ERR_INVALID_ARG;
        }
        if (scenes[i]->device != dev) {
            set_error("rumi_batch_create: scene on another device");
            return RUMI_ERR_INVALID_ARG;
        }
    }
    rumi_batch *b = new rumi_batch();
    b->device = dev;
    b->scenes.assign(scenes, scenes + n);
    b->num_sms = scenes[0]->num_sms;
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete b;
        return cuda_status(e, "cudaStreamCreate");
    }
    e = cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        rumi_batch_destroy(b);
        return cuda_status(e, "batch auxiliary stream");
    }
    std::vector<DevScene> table(n);
    b->pix0.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        table[i] = scenes[i]->dev;
        if (!shade_lean(scenes[i])) b->lean = false;
        b->pix0[i + 1] = b->pix0[i] + (long long)table[i].width * table[i].height;
    }
    e = dalloc((void **)&b->d_scenes, sizeof(DevScene) * n, b->stream);
    if (e == cudaSuccess) e = dalloc((void **)&b->d_path0, sizeof(long long) * (n + 1), b->stream);
    if (e == cudaSuccess) e = dalloc((void **)&b->d_pix0, sizeof(long long) * (n + 1), b->stream);
    if (e == cudaSuccess) e = dalloc((void **)&b->d_keys, sizeof(uint32_t) * 2 * n, b->stream);
    if (e == cudaSuccess) e = dalloc((void **)&b->d_spp, sizeof(int) * n, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_scenes, table.data(), sizeof(DevScene) * n, cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_pix0, b->pix0.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) {
        rumi_status st = cuda_status(e, "rumi_batch_create");
        rumi_batch_destroy(b);
        return st;
    }
    *out = b;
    return RUMI_OK;
}

rumi_status rumi_batch_destroy(rumi_batch *b) {
    if (!b) return RUMI_OK;
    drop_graph(b);
    cudaStream_t s = b->stream;
    if (s) cudaStreamSynchronize(s);
    dfree(b->d_scenes, s);
    dfree(b->d_path0, s);
    dfree(b->d_pix0, s);
    dfree(b->d_keys, s);
    dfree(b->d_spp, s);
    dfree(b->ws, s);
    dfree(b->d_films, s);
    if (b->aux) {
        cudaStreamSynchronize(b->aux);
        cudaStreamDestroy(b->aux);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    delete b;
    return RUMI_OK;
}

int64_t rumi_batch_film_floats(const rumi_batch *b) { return b ? b->pix0.back() * 3 : 0; }

rumi_status rumi_render_batch(rumi_batch *b, const rumi_batch_params *p, float *films, int32_t films_on_device,
                              rumi_render_stats *stats) {
    if (!b || !p || !films || !p->spp || !p->seeds) {
        set_error("rumi_render_batch: NULL argument");
        return RUMI_ERR_INVALID_ARG;
    }
    if (p->max_depth <= 0 || p->max_depth > 64) {
        set_error("rumi_render_batch: max_depth must be in [1, 64]");
        return RUMI_ERR_INVALID_ARG;
    }
    const int n = (int)b->scenes.size();
    cudaStream_t s = p->stream ? (cudaStream_t)p->stream : b->stream;
    std::vector<int> spp(n);
    std::vector<long long> path0(n + 1, 0);
    std::vector<uint32_t> keys(2 * n);
    int max_spp = 1;
    for (int i = 0; i < n; ++i) {
        if (p->spp[i] <= 0) {
            set_error("rumi_render_batch: spp must be positive");
            return RUMI_ERR_INVALID_ARG;
        }
        spp[i] = p->spp[i];
        max_spp = spp[i] > max_spp ? spp[i] : max_spp;
        path0[i + 1] = path0[i] + (b->pix0[i + 1] - b->pix0[i]) * spp[i];
        keys[2 * i] = (uint32_t)p->seeds[i];
        keys[2 * i + 1] = (uint32_t)(p->seeds[i] >> 32) ^ 0x5851F42Du;  // rumi_render's key schedule
    }
    long long wave = p->wave_paths > 0 ? p->wave_paths : RUMI_DEFAULT_WAVE_PATHS;
    if (wave < max_spp) wave = max_spp;
    if (wave > path0.back()) wave = path0.back();
    if (wave < max_spp) wave = max_spp;
    if (wave > 0x3fffffffLL) return set_error("wave_paths too large"), RUMI_ERR_INVALID_ARG;  // 30-bit slots
    BatchFrame F;
    F.lean = b->lean;
    F.n_scenes = n;
    F.max_depth = p->max_depth;
    F.wave_paths = wave;
    F.blocks_per_sm = p->blocks_per_sm;
    plan_waves(b->pix0, spp, wave, F.waves);
    F.scenes = b->d_scenes;
    F.scene_path0 = b->d_path0;
    F.scene_pix0 = b->d_pix0;
    F.scene_key = b->d_keys;
    F.scene_spp = b->d_spp;

    const size_t need = pt_batch_workspace_bytes(wave);
    if (b->ws_bytes < need) {
        drop_graph(b);
        cudaStreamSynchronize(s);
        dfree(b->ws, b->stream);
        b->ws = nullptr;
        b->ws_bytes = 0;
        cudaError_t e = dalloc(&b->ws, need, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) return cuda_status(e, "batch workspace");
        b->ws_bytes = need;
    }
    const size_t film_bytes = sizeof(float) * 3 * (size_t)b->pix0.back();
    float *films_dev = films;
    if (!films_on_device) {
        if (!b->d_films) {
            cudaError_t e = dalloc((void **)&b->d_films, film_bytes, b->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
            if (e != cudaSuccess) return cuda_status(e, "batch film");
        }
        films_dev = b->d_films;
    }
    // per-frame tables: the captured graph reads them from device memory
    cudaError_t e = cudaMemcpyAsync(b->d_path0, path0.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_keys, keys.data(), sizeof(uint32_t) * 2 * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_spp, spp.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_status(e, "batch tables");

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const bool timing = (p->flags & RUMI_FLAG_TIMING) != 0;
    if (timing) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
    }
    rumi_status st = RUMI_OK;
    if (p->flags & RUMI_BATCH_GRAPH) {
        const bool same = b->graph && b->graph_spp == spp && b->graph_depth == p->max_depth && b->graph_wave == wave &&
                          b->graph_blocks == p->blocks_per_sm && b->graph_films == films_dev;
        if (!same) {
            drop_graph(b);
            // capture on the batch's own stream (a legacy or foreign stream may not be capturable)
            cudaStreamSynchronize(s);
            cudaGraph_t g = nullptr;
            e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_status(e, "cudaStreamBeginCapture");
            st = pt_enqueue_batch(F, b->ws, films_dev, b->stream, b->num_sms, b->aux, b->ev_fork, b->ev_join);
            e = cudaStreamEndCapture(b->stream, &g);
            if (st != RUMI_OK) {
                if (g) cudaGraphDestroy(g);
                return st;
            }
            if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                b->graph = nullptr;
                return cuda_status(e, "cudaGraphInstantiate");
            }
            b->graph_spp = spp;
            b->graph_depth = p->max_depth;
            b->graph_wave = wave;
            b->graph_blocks = p->blocks_per_sm;
            b->graph_films = films_dev;
        }
        if (e0) cudaEventRecord(e0, s);
        e = cudaGraphLaunch(b->graph, s);
        if (e != cudaSuccess) return cuda_status(e, "cudaGraphLaunch");
    } else {
        if (e0) cudaEventRecord(e0, s);
        st = pt_enqueue_batch(F, b->ws, films_dev, s, b->num_sms, b->aux, b->ev_fork, b->ev_join);
        if (st != RUMI_OK) return st;
    }
    if (e1) cudaEventRecord(e1, s);
    unsigned long long h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    e = cudaMemcpyAsync(h, pt_batch_stats_ptr(b->ws, wave), sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && !films_on_device)
        e = cudaMemcpyAsync(films, films_dev, film_bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        return cuda_status(e, "rumi_render_batch");
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->paths = path0.back();
        stats->rays_extend = (int64_t)h[0];
        stats->rays_shadow = (int64_t)h[1];
        stats->nan_samples = (int64_t)h[2];
        stats->extend_launches = (int64_t)F.waves.size() * p->max_depth;
        stats->shade_launches = stats->extend_launches;
        stats->shadow_launches = stats->extend_launches;
        if (timing) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            stats->total_ms = ms;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return RUMI_OK;
}

}  // extern "C"
