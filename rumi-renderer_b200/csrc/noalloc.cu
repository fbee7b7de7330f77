// rumi_render_noalloc: the path tracer's frame loop with its wave state (ray queues,
// hit records, shadow queue, per-path throughput and radiance, counters) placed in a
// fixed file-scope device array instead of memory obtained from cudaMalloc.
//
// Who needs it: callers that may not allocate device memory once they are running --
// an embedding application that owns a fixed device-memory budget and forbids
// allocation after start-up, or a real-time loop that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree imply.  Such a caller creates its scene once at
// set-up time (rumi_scene_create allocates) and then renders frames into a device film
// it owns.
//
// Limits and rules:
//  - The array holds RUMI_NOALLOC_SCRATCH_BYTES (16 MiB) on every GPU that loads the
//    library, for the life of the process.  At 176 bytes per path in flight (eleven
//    float4 per path, pt_workspace_bytes) that is about 95k paths per wave; a frame is
//    rendered in as many waves as it needs.  A request whose single pixel (spp paths)
//    does not fit, or whose wave_paths exceeds the capacity, is rejected with
//    RUMI_ERR_INVALID_ARG before anything is launched.
//  - Host code cannot use the array's name as a device address.  The first call on a
//    device (with that device current) looks the address up with cudaGetSymbolAddress
//    and caches it per device index; make that first call before any stream capture.
//    The cache does not survive cudaDeviceReset (the module, and with it the array, may
//    be reloaded at another address): do not call this entry point after a reset.
//  - Every call shares the one array and its counters are cleared at the start of each
//    call; calls whose work overlaps on the GPU (different streams, other threads) race
//    on it and must be serialised by the caller.
//  - film must be a device pointer; RUMI_FLAG_TIMING is refused (it would create events).
#include "renderer.h"
#include <mutex>

namespace {

constexpr size_t RUMI_NOALLOC_SCRATCH_BYTES = 16u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[RUMI_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
void *g_scratch_addr[MAX_DEVICES] = {};
std::mutex g_scratch_mu;

rumi_status scratch_address(void **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return rumi::cuda_status(e, "rumi_render_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= MAX_DEVICES) {
        rumi::set_error("rumi_render_noalloc: device index beyond the set-up table");
        return RUMI_ERR_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return rumi::cuda_status(e, "rumi_render_noalloc: cudaGetSymbolAddress");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return RUMI_OK;
}

}  // namespace

extern "C" rumi_status rumi_render_noalloc(rumi_scene *sc, const rumi_render_params *p, float *film,
                                           rumi_render_stats *stats) {
    using namespace rumi;
    if (!sc || !p || !film) return set_error("rumi_render_noalloc: NULL argument"), RUMI_ERR_INVALID_ARG;
    if (p->integrator != RUMI_PATH_TRACER || p->max_depth <= 0)
        return set_error("rumi_render_noalloc: path tracer with max_depth > 0 only"), RUMI_ERR_INVALID_ARG;
    if (p->spp <= 0) return set_error("rumi_render_noalloc: spp must be positive"), RUMI_ERR_INVALID_ARG;
    if (p->flags & RUMI_FLAG_TIMING)
        return set_error("rumi_render_noalloc: RUMI_FLAG_TIMING is not available"), RUMI_ERR_INVALID_ARG;
    // largest number of paths whose wave state fits the array
    long long lo = 0, hi = (long long)(RUMI_NOALLOC_SCRATCH_BYTES / 160) + 1;
    while (lo + 1 < hi) {
        const long long mid = (lo + hi) / 2;
        if (pt_workspace_bytes(mid) <= RUMI_NOALLOC_SCRATCH_BYTES)
            lo = mid;
        else
            hi = mid;
    }
    const long long max_paths = lo;
    if ((long long)p->spp > max_paths) {
        set_error("rumi_render_noalloc: spp " + std::to_string(p->spp) + " exceeds the " +
                  std::to_string(max_paths) + " paths the 16 MiB scratch holds");
        return RUMI_ERR_INVALID_ARG;
    }
    if ((long long)p->wave_paths > max_paths) {
        set_error("rumi_render_noalloc: wave_paths " + std::to_string(p->wave_paths) + " exceeds the " +
                  std::to_string(max_paths) + " paths the 16 MiB scratch holds");
        return RUMI_ERR_INVALID_ARG;
    }
    if (uses_bvh8(p->trace_mode) && !sc->nodes8) {  // building it would allocate
        set_error("rumi_render_noalloc: the eight-wide tree (trace_mode 5) is built by the scene's first "
                  "rumi_render or rumi_trace_rays call that asks for it; none has yet");
        return RUMI_ERR_INVALID_ARG;
    }
    const long long total_pix = (long long)sc->dev.width * sc->dev.height;
    long long pix_per_wave = (p->wave_paths > 0 ? (long long)p->wave_paths : max_paths) / p->spp;
    if (pix_per_wave < 1) pix_per_wave = 1;
    if (pix_per_wave > total_pix) pix_per_wave = total_pix;
    void *ws = nullptr;
    rumi_status st = scratch_address(&ws);
    if (st != RUMI_OK) return st;
    cudaStream_t s = p->stream ? (cudaStream_t)p->stream : sc->stream;
    return pt_render_in(sc, p, film, stats, s, ws, pix_per_wave);
}
