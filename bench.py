#!/usr/bin/env python3
"""Benchmark of the B200 rendering path on the BVH-bound path-tracing workload:
the Cornell box holding a seeded 1,048,576-triangle displaced sphere, 1024x1024 pixels,
64 samples per pixel, max depth 10, next-event estimation (67,108,864 paths per frame).

One step = one path-traced frame of that workload.  Our arm times the frames on the
device (scene and BVH resident in HBM), measures the closest-hit kernel's launches with
CUDA events for the roofline, repeats the frame end to end through the C-ABI from pinned
host buffers (scene upload + GPU BVH build + render + film read-back), and times the
reference renderer itself (oracle/_ref) on a bounded sample of the same workload on the
host cores.  ``--impl reference`` times only the reference, with every host core.

Multi-GPU (torchrun): one process per GPU renders its own frame (an independent spp
shard with its own seed); no data exchange on the path; value = all ranks' paths / the
slowest rank's time.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rumi-renderer_b200"))

WORKLOAD = dict(width=1024, height=1024, spp=64, max_depth=10, levels=9, seed=7)
METRIC = "path samples/sec"
UNIT = "paths/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ray-sets", action="store_true", help="skip the primary / secondary / shadow ray-set rates")
    ap.add_argument("--wave-paths", type=int, default=0)
    ap.add_argument("--small", action="store_true", help="256x256 at 16 spp (profiling runs)")
    ap.add_argument("--workload", default="bvh_bound", choices=["bvh_bound", "batched", "adjoint", "bdpt_caustic", "cornell"],
                    help="batched: 256 seeded scenes as one frame vs the per-scene loop; "
                         "adjoint: inverse rendering with the path-replay adjoint")
    ap.add_argument("--adam-steps", type=int, default=200, help="adjoint workload: optimisation steps")
    ap.add_argument("--adjoint-spp", type=int, default=0,
                    help="adjoint workload: samples per pixel of the gradient pass (0 = the forward's 64)")
    ap.add_argument("--adam-lr", type=float, default=1e-2, help="adjoint workload: Adam learning rate")
    ap.add_argument("--adam-lr-end", type=float, default=0.0,
                    help="adjoint workload: learning rate at the last step, reached by exponential decay "
                         "(0: constant --adam-lr)")
    ap.add_argument("--adjoint-levels", type=int, default=7,
                    help="adjoint workload: displaced-sphere subdivision levels (4 * 4**levels triangles)")
    ap.add_argument("--scenes", type=int, default=256, help="batched workload: number of scenes")
    ap.add_argument("--breakdown", action="store_true",
                    help="batched workload: also time every scene alone and report the per-size-class rates and "
                         "the bound they put on any batching")
    ap.add_argument("--trace-mode", type=int, default=0,
                    help="bvh_bound workload: rumi_render_params.trace_mode (0 = library default)")
    return ap.parse_args()


def workload(args):
    w = dict(WORKLOAD)
    if args.small:
        w.update(width=256, height=256, spp=16)
    return w


DATA = "synthetic (seeded 1,048,576-triangle displaced sphere, random per-triangle albedo)"


def bench_config(w, world):
    """The workload's `config` object, the same on both arms."""
    return dict(workload="bvh_bound_pt: Cornell box + displaced sphere", width=w["width"], height=w["height"],
                spp=w["spp"], max_depth=w["max_depth"], triangles=4 * 4 ** w["levels"],
                parallelism=f"replicas x{world} (spp shards)",
                l2="inputs larger than L2 (scene ~170 MB + wave queues ~5.9 GB per GPU)")


def build_scene(w):
    from rumi_b200 import scenes
    return scenes.bvh_bound_pt(w["width"], w["height"], w["spp"], w["max_depth"], levels=w["levels"], seed=w["seed"])


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# --------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = tempfile.mktemp(prefix="rumi_clocks_", suffix=".csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() in ("active", "1"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------ reference (CPU) arm
def _ref_worker(conn, w, pin=None):
    """One host process: builds the reference scene once, then renders the rows it is sent.
    pin: a host core the process is bound to (like `taskset -c <core>`)."""
    if pin is not None:
        os.sched_setaffinity(0, {pin})
    sys.path.insert(0, os.path.join(ROOT, "rumi-renderer_b200"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import refimpl
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)  # the reference prints progress to stdout
    sc = build_scene(w)
    rs = refimpl.RefScene(sc, seed=1)
    conn.send(("ready", rs.spp))
    while True:
        msg = conn.recv()
        if msg is None:
            break
        if msg[0] == "trace":  # BVHAccel::Travel over a ray set, one thread
            _, rays, anyhit = msg
            t0 = time.perf_counter()
            rs.trace(rays, anyhit=anyhit)
            conn.send((rays.shape[0], time.perf_counter() - t0))
            continue
        seed, rows = msg
        t0 = time.perf_counter()
        paths = 0
        for r in rows:
            rs.render_rows(seed, r, r + 1)
            paths += w["width"] * rs.spp
        conn.send((paths, time.perf_counter() - t0))
    rs.close()


class RefPool:
    def __init__(self, w, n_procs, pin=None):
        ctx = mp.get_context("spawn")
        self.w = w
        self.conns, self.procs = [], []
        for _ in range(n_procs):
            a, b = ctx.Pipe()
            p = ctx.Process(target=_ref_worker, args=(b, w, pin), daemon=True)
            p.start()
            self.conns.append(a)
            self.procs.append(p)
        self.spp = None
        for c in self.conns:
            tag, spp = c.recv()
            self.spp = spp

    def step(self, seed, rows_per_proc, offset):
        """Every process renders rows_per_proc rows spread over the image; returns
        (paths, seconds) with seconds = wall time of the slowest process."""
        H = self.w["height"]
        n = len(self.conns)
        total = n * rows_per_proc
        t0 = time.perf_counter()
        for i, c in enumerate(self.conns):
            rows = [((i * rows_per_proc + k) * H // total + offset) % H for k in range(rows_per_proc)]
            c.send((seed, rows))
        paths = 0
        for c in self.conns:
            p, _ = c.recv()
            paths += p
        return paths, time.perf_counter() - t0

    def close(self):
        for c in self.conns:
            c.send(None)
        for p in self.procs:
            p.join(timeout=30)


def ref_procs(limit=None):
    n = os.cpu_count() or 1
    try:
        import psutil
        n = min(n, max(1, int(psutil.virtual_memory().available / (1.2 * 1024 ** 3))))
    except Exception:
        pass
    return max(1, min(n, limit or n))


def single_core_sample(w):
    """The reference renderer single-threaded on one pinned host core (taskset -c 0, or the
    lowest core this process may use): one full row of the workload (1024 px at the
    workload's spp)."""
    allowed = os.sched_getaffinity(0)
    core = 0 if 0 in allowed else min(allowed)
    pool = RefPool(w, 1, pin=core)
    paths, secs = pool.step(seed=5, rows_per_proc=1, offset=w["height"] // 2)
    pool.close()
    return dict(value=paths / secs, unit=UNIT, cores=1, pinned_core=core, kind="reference",
                sample=f"{paths} paths = 1 row of {w['width']} px x {pool.spp} spp of the same workload, one "
                       f"process pinned to host core {core}, reference renderer built from its sources "
                       f"(oracle/_ref), CPU {cpu_model()}",
                seconds=secs)


def cpu_baseline_sample(w, procs, rows_per_proc=1):
    pool = RefPool(w, procs)
    paths, secs = pool.step(seed=3, rows_per_proc=rows_per_proc, offset=0)
    pool.close()
    return dict(value=paths / secs, unit=UNIT, cores=procs, kind="reference",
                sample=f"{paths} paths = {procs} processes x {rows_per_proc} row(s) of 1024 px x {pool.spp} spp "
                       f"of the same workload, reference renderer built from its sources (oracle/_ref), "
                       f"one thread per process, CPU {cpu_model()}",
                seconds=secs, single_core=single_core_sample(w))


def make_ray_sets(sc, gs, n, seed=5):
    """The three ray sets of the BVH-bound workload (host arrays (n, 7): o, d, tmax):
    primary camera rays through jittered pixels of the 1024x1024 film; secondary rays
    leaving the primary hits in cosine-distributed directions about the face normal
    (diffuse bounce); shadow rays from those hits to uniform points on the light."""
    import numpy as np
    rng = np.random.default_rng(seed)
    fs = sc.flatten()
    W, H = fs.image.width, fs.image.height
    cam = sc.camera
    tan = np.tan(np.radians(cam.fov) * 0.5)
    px = rng.integers(0, W, n) + rng.random(n)
    py = rng.integers(0, H, n) + rng.random(n)
    x = -((px - W / 2) / (W / 2)) * tan
    y = -((py - H / 2) / (H / 2)) * tan * cam.y_ratio
    d = np.stack([x, y, np.ones(n)], 1)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = np.tile(np.asarray(cam.position, np.float64), (n, 1))
    big = np.float32(3.0e38)
    primary = np.concatenate([o, d, np.full((n, 1), big)], 1).astype(np.float32)
    t, prim, _, _ = gs.trace(primary)
    hit = (prim >= 0) & (prim < fs.tri_vertices.shape[0])
    p = (o + d * t[:, None])[hit]
    tri = fs.tri_vertices[prim[hit]].astype(np.float64)
    nrm = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm *= -np.sign((nrm * d[hit]).sum(1))[:, None]  # face the incoming ray
    m = p.shape[0]
    u1, u2 = rng.random(m), rng.random(m)
    a = np.where(np.abs(nrm[:, :1]) > 0.9, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    tu = np.cross(nrm, a)
    tu /= np.linalg.norm(tu, axis=1, keepdims=True)
    tv = np.cross(nrm, tu)
    r, phi = np.sqrt(u1), 2 * np.pi * u2
    wi = tu * (r * np.cos(phi))[:, None] + tv * (r * np.sin(phi))[:, None] + nrm * np.sqrt(1 - u1)[:, None]
    secondary = np.concatenate([p, wi, np.full((m, 1), big)], 1).astype(np.float32)
    lp = np.array([0.375, 0.999, 0.375]) + rng.random((m, 1)) * np.array([0.25, 0, 0]) + \
        rng.random((m, 1)) * np.array([0, 0, 0.25])
    sd = lp - p
    dist = np.linalg.norm(sd, axis=1)
    shadow = np.concatenate([p, sd / dist[:, None], (dist - 1e-4)[:, None]], 1).astype(np.float32)
    return dict(primary=primary, secondary=secondary, shadow=shadow)


def gpu_rays_per_s(gs, rays, anyhit, repeats=3):
    """Device time of rumi_trace_rays (plain kernel) over a device-resident ray set."""
    import numpy as np
    import torch
    r8 = np.zeros((rays.shape[0], 8), np.float32)
    r8[:, 0:3], r8[:, 4:7], r8[:, 7] = rays[:, 0:3], rays[:, 3:6], rays[:, 6]
    dr = torch.from_numpy(r8).cuda()
    dt = torch.empty(rays.shape[0], device="cuda")
    dp = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    best = float("inf")
    for _ in range(repeats + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        gs.trace_device(rays.shape[0], dr.data_ptr(), dt.data_ptr(), dp.data_ptr(), anyhit=anyhit, stream=stream,
                        count=False)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return rays.shape[0] / (best / 1000.0)


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    w = workload(args)
    procs = ref_procs()
    pool = RefPool(w, procs)
    for s in range(args.warmup):
        pool.step(100 + s, 1, offset=s)
    total_paths, total_s = 0, 0.0
    for s in range(args.steps):
        p, sec = pool.step(200 + s, 1, offset=args.warmup + s)
        total_paths += p
        total_s += sec
    pool.close()
    value = total_paths / total_s
    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                ms_per_step=1000.0 * total_s / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f32", data=DATA, impl="reference", config=bench_config(w, args.gpus),
                cpu_baseline=dict(value=value, unit=UNIT, cores=procs, kind="reference",
                                  sample=f"each step: {procs} processes x 1 row of {w['width']} px x {pool.spp} spp, "
                                         f"CPU {cpu_model()}"),
                e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- our arm
def peaks():
    """({"hbm_gbs": copy bandwidth}, "measured" | "fallback"): the measured copy bandwidth of
    MEASURED_PEAKS.json (its `hbm_gbs`, at the top level or one level down), else a
    fallback copy bandwidth of 6650 GB/s measured earlier on B200s of the same kind."""
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        cands = [d] + [v for v in d.values() if isinstance(v, dict)]
        for c in cands:
            v = c.get("hbm_gbs")
            if isinstance(v, (int, float)) and v > 0:
                return {"hbm_gbs": float(v)}, "measured"
    except Exception:
        pass
    return {"hbm_gbs": 6650.0}, "fallback"


def l2_read_gbs(mbytes=64, passes=50):
    """L2 read bandwidth: one launch re-reading a 64 MiB device buffer (smaller than the
    126 MB L2) `passes` times (rumi_test_read_bandwidth, float4 loads cached in L2 only)."""
    import ctypes as C
    import torch
    from rumi_b200 import _capi
    buf = torch.ones(mbytes * (1 << 20) // 4, dtype=torch.float32, device="cuda")
    ms = C.c_double()
    best = float("inf")
    for _ in range(5):
        _capi.check(_capi.load().rumi_test_read_bandwidth(C.c_void_p(buf.data_ptr()), buf.numel() * 4, passes,
                                                          C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                                          C.byref(ms)), "rumi_test_read_bandwidth")
        best = min(best, ms.value)
    return buf.numel() * 4.0 * passes / (best / 1000.0) / 1e9


def extend_traffic():
    """DRAM bytes per closest-hit launch from the committed ncu summary, if any."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "extend_traffic.json")))
    except Exception:
        return None


def our_arm(args):
    import numpy as np
    import torch
    import rumi_b200
    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    w = workload(args)
    sc = build_scene(w)
    gs = rumi_b200.GpuScene(sc)
    bvh = gs.bvh_info()
    paths_per_frame = w["width"] * w["height"] * w["spp"]
    film = torch.empty((w["height"], w["width"], 3), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    from rumi_b200 import shard
    seed0 = shard.replica_seed(0, rank)  # each rank renders an independent spp shard

    # algorithmic bytes per closest-hit ray, from an instrumented (untimed) frame
    _, st0 = gs.render(seed=seed0 + 999, film_device_ptr=film.data_ptr(), stream=stream, count_stats=True,
                       wave_paths=args.wave_paths, trace_mode=args.trace_mode)
    nodes_per_ray = st0["extend_node_fetches"] / st0["rays_extend"]
    prims_per_ray = st0["extend_prim_tests"] / st0["rays_extend"]
    bytes_per_ray = 32.0 * nodes_per_ray + 48.0 * prims_per_ray + 32.0 + 16.0

    for s in range(args.warmup):
        gs.render(seed=seed0 + s, film_device_ptr=film.data_ptr(), stream=stream, wave_paths=args.wave_paths, trace_mode=args.trace_mode)
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rays_ext, rays_sh, launches = 0, 0, 0
    barrier()
    ev0.record()
    # the frames as the library renders them: each bounce's shadow rays traced on a second
    # stream beside the next bounce's closest-hit rays, no per-kernel events
    for s in range(args.steps):
        _, st = gs.render(seed=seed0 + 100 + s, film_device_ptr=film.data_ptr(), stream=stream,
                          wave_paths=args.wave_paths, trace_mode=args.trace_mode)
        rays_ext += st["rays_extend"]
        rays_sh += st["rays_shadow"]
        waves = st["extend_launches"] // w["max_depth"]
        launches += waves * (3 + 5 * w["max_depth"])
    ev1.record()
    barrier()
    clocks_info = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms)
    value = world * paths_per_frame * args.steps / (ms / 1000.0)
    rays_per_s = world * (rays_ext + rays_sh) / (ms / 1000.0)
    # the same frames with every launch in order on one stream and CUDA events around each
    # kernel (RUMI_FLAG_SERIAL | RUMI_FLAG_TIMING): each kernel's own device time, for the
    # roofline of the closest-hit kernel and the per-kernel breakdown
    ext_ms, ext_launches, ext_rays, kern = 0.0, 0, 0, dict(extend_ms=0.0, shadow_ms=0.0, shade_ms=0.0, total_ms=0.0)
    for s in range(args.steps):
        _, st = gs.render(seed=seed0 + 100 + s, film_device_ptr=film.data_ptr(), stream=stream, timing=True,
                          serial=True, wave_paths=args.wave_paths, trace_mode=args.trace_mode)
        ext_ms += st["extend_ms"]
        ext_launches += st["extend_launches"]
        ext_rays += st["rays_extend"]
        for k in kern:
            kern[k] += st[k] / args.steps
    avg_launch_ms = ext_ms / ext_launches
    rays_per_launch = ext_rays / ext_launches
    achieved = bytes_per_ray * rays_per_launch / (avg_launch_ms / 1000.0) / 1e9
    pk, pk_kind = peaks()
    traffic = extend_traffic()
    roofline = dict(bound="hbm", achieved=achieved, peak=pk["hbm_gbs"], unit="GB/s", frac=achieved / pk["hbm_gbs"],
                    # DRAM bytes per closest-hit ray from the committed ncu capture, times this
                    # run's rays per launch (the capture's launches may hold another wave size)
                    traffic=traffic["dram_bytes_per_ray"] * rays_per_launch if traffic else None,
                    kernel="pt_extend (closest-hit)", peak_kind=pk_kind,
                    algorithmic_bytes_per_ray=bytes_per_ray, nodes_per_ray=nodes_per_ray, prims_per_ray=prims_per_ray,
                    rays_per_launch=rays_per_launch, avg_launch_ms=avg_launch_ms,
                    closest_hit_rays_per_s=ext_rays / (ext_ms / 1000.0),
                    measured="CUDA events around every closest-hit launch of --steps frames rendered with "
                             "RUMI_FLAG_SERIAL (each kernel alone on the GPU), after the timed frames",
                    per_frame_ms_serial={k: round(v, 2) for k, v in kern.items()})
    # the tree and primitives are served mostly from L2 (see the ncu summary), so the same
    # algorithmic bytes are also set against an L2-resident copy measured here
    l2 = l2_read_gbs()
    roofline["l2"] = dict(peak=l2, unit="GB/s", frac=achieved / l2,
                          how="one launch re-reading a 64 MiB buffer 50 times (rumi_test_read_bandwidth), "
                              "best of 5, CUDA events")

    # ---- end to end through the C-ABI: pinned host scene -> device, BVH build, render, film -> host
    e2e = None
    if not args.no_e2e:
        from rumi_b200 import _capi, build_desc
        import ctypes as C
        fs = sc.flatten()
        pinned = {}
        for name in ("tri_vertices", "tri_normals", "tri_material", "tri_albedo", "rects", "rect_material",
                     "spheres", "sphere_material"):
            a = getattr(fs, name)
            if a is None:
                continue
            t = torch.empty(a.shape, dtype=torch.from_numpy(np.ascontiguousarray(a)).dtype, pin_memory=True)
            t.copy_(torch.from_numpy(np.ascontiguousarray(a)))
            pinned[name] = t
            setattr(fs, name, t.numpy())
        desc, keep = build_desc(fs)
        h2d = sum(t.numel() * t.element_size() for t in pinned.values())
        film_host = torch.empty((w["height"], w["width"], 3), dtype=torch.float32, pin_memory=True)
        d2h = film_host.numel() * 4
        lib = _capi.load()
        params = _capi.rumi_render_params()
        params.integrator, params.max_depth, params.spp = 0, w["max_depth"], w["spp"]
        params.wave_paths = args.wave_paths

        def e2e_step(seed):
            hnd = C.c_void_p()
            _capi.check(lib.rumi_scene_create(C.byref(desc), C.byref(hnd)), "rumi_scene_create")
            params.seed = seed
            _capi.check(lib.rumi_render(hnd, C.byref(params), C.c_void_p(film_host.data_ptr()), 0, None), "rumi_render")
            lib.rumi_scene_destroy(hnd)

        e2e_step(seed0 + 500)
        barrier()
        t0 = time.perf_counter()
        step_ms = []
        for s in range(args.steps):
            ts = time.perf_counter()
            e2e_step(seed0 + 600 + s)
            step_ms.append(round(1000.0 * (time.perf_counter() - ts), 1))
        barrier()
        sec = max_over_ranks(time.perf_counter() - t0)
        e2e = dict(value=world * paths_per_frame * args.steps / sec, unit=UNIT, h2d_bytes_per_step=h2d,
                   d2h_bytes_per_step=d2h, ms_per_step=1000.0 * sec / args.steps, step_ms=step_ms)
        film_np = film_host.numpy()
        assert np.isfinite(film_np).all()

    # closest-hit / any-hit rays/s on the three ray sets, and the reference's BVHAccel::Travel
    # on a sample of the same rays (one thread)
    ray_sets = None
    if rank == 0 and not args.no_ray_sets:
        sets = make_ray_sets(sc, gs, 1 << 21)
        ray_sets = {}
        for name, rays in sets.items():
            anyhit = name == "shadow"
            ray_sets[name] = dict(rays=int(rays.shape[0]), anyhit=anyhit,
                                  gpu_rays_per_s=gpu_rays_per_s(gs, rays, anyhit))
        if world == 1 and not args.no_cpu_baseline:
            pool = RefPool(w, 1)
            for name, rays in sets.items():
                sample = rays[:20000]
                pool.conns[0].send(("trace", sample, name == "shadow"))
                n, sec = pool.conns[0].recv()
                ray_sets[name]["ref_rays_per_s_1_thread"] = n / sec
                ray_sets[name]["ref_sample"] = n
            pool.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(w, ref_procs(limit=16))

    gs.close()
    if rank == 0:
        line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
                    ms_per_step=ms / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
                    data=DATA, config=bench_config(w, world), bvh_build_ms=bvh["build_ms"],
                    rays_per_sec=rays_per_s, ray_sets=ray_sets, roofline=roofline, cpu_baseline=cpu, e2e=e2e, gpu_launches=launches,
                    clocks=clocks_info)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def batched_arm(args):
    """Batched wavefront workload: scene i (scenes.batch_scene) has a log-uniform 1k-200k
    triangle terrain, a resolution from {64,128,256,512}^2 and spp from {4,16,64}, depth 8.
    One step renders every scene once.  Plain arm: the scenes one at a time through
    rumi_render; batched arm: one rumi_render_batch frame replayed from its CUDA graph.
    Both arms produce bit-identical films for the same seeds (checked on the last step),
    so their RMSE is equal and samples/sec compare directly."""
    import torch
    import rumi_b200
    from rumi_b200 import scenes
    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    depth = 8
    # scenes are sharded across ranks (scene i on rank i % world); no exchange
    from rumi_b200 import shard
    ids = shard.scene_shard(args.scenes, rank, world)
    t0 = time.perf_counter()
    gss = [rumi_b200.GpuScene(scenes.batch_scene(i, depth)) for i in ids]
    setup_s = time.perf_counter() - t0
    spp = [g.flat.image.n_samples for g in gss]
    paths = sum(g.width * g.height * s for g, s in zip(gss, spp))
    tris = sum(int(g.flat.tri_vertices.shape[0]) for g in gss)
    batch = rumi_b200.GpuBatch(gss)
    films_plain = torch.zeros(batch.n_floats, dtype=torch.float32, device="cuda")
    films_batch = torch.zeros(batch.n_floats, dtype=torch.float32, device="cuda")
    offs, o = [], 0
    for g in gss:
        offs.append(o)
        o += g.width * g.height * 3
    stream = torch.cuda.current_stream().cuda_stream

    def seeds(step):
        return [1 + i + 100000 * step for i in ids]

    def plain(step):
        for g, s, sd, off in zip(gss, spp, seeds(step), offs):
            g.render(spp=s, seed=sd, film_device_ptr=films_plain.data_ptr() + 4 * off, stream=stream)
        return len(gss) * (3 + 5 * depth)  # rumi_render: per bounce two resets, extend, shade, shadow

    def batched(step):
        _, st = batch.render(spp, seeds(step), depth, graph=True, films_device_ptr=films_batch.data_ptr(),
                             stream=stream)
        waves = st["extend_launches"] // depth
        return waves * (3 + 5 * depth)

    def timed(fn):
        for s in range(args.warmup):
            fn(s)
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        launches = 0
        for s in range(args.steps):
            launches += fn(args.warmup + s)
        ev1.record()
        barrier()
        return max_over_ranks(ev0.elapsed_time(ev1)), launches

    clocks = ClockSampler(local)
    clocks.start()
    ms_plain, l_plain = timed(plain)
    ms_batch, l_batch = timed(batched)
    clocks_info = clocks.stop()
    equal = bool(torch.equal(films_plain, films_batch))
    breakdown = None
    if args.breakdown:
        breakdown = scene_breakdown(gss, spp, stream)
    batch.close()
    for g in gss:
        g.close()
    all_paths = paths
    if dist:
        t = torch.tensor([paths], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        all_paths = float(t.item())
    value = all_paths * args.steps / (ms_batch / 1000.0)
    plain_value = all_paths * args.steps / (ms_plain / 1000.0)
    if rank == 0:
        line = dict(metric="path samples/sec at equal RMSE (batched vs plain per-scene loop)", value=value,
                    unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup, ms_per_step=ms_batch / args.steps,
                    higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
                    data="synthetic (seeded fBm terrains in the Cornell box)",
                    config=dict(workload=f"batched: {args.scenes} scenes, tris log-uniform 1k-200k, res "
                                         "{64..512}^2, spp {4,16,64}, depth 8", scenes=len(gss), paths=paths,
                                triangles=tris, setup_s=setup_s, parallelism=f"scene shards x{world}",
                                l2="inputs larger than L2 (scenes + wave queues)"),
                    plain_loop=dict(value=plain_value, ms_per_step=ms_plain / args.steps, gpu_launches=l_plain),
                    speedup_vs_plain=value / plain_value, equal_images=equal, gpu_launches=l_batch,
                    clocks=clocks_info)
        if breakdown:
            line["per_scene_breakdown"] = breakdown
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0 if equal else 1


def scene_breakdown(gss, spp, stream):
    """Every scene rendered alone (CUDA events around three frames after two warm-up
    frames), grouped by paths per frame: each class's share of the paths and of the loop's
    time and its rate; and the bound on any batching of the frame -- the frame time if every
    path ran at the rate the largest scenes reach alone, or at the best single scene's."""
    import torch
    rows = []
    for g, s in zip(gss, spp):
        film = torch.zeros((g.height, g.width, 3), device="cuda")
        for w in range(2):
            g.render(spp=s, seed=w, film_device_ptr=film.data_ptr(), stream=stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(3):
            g.render(spp=s, seed=10 + k, film_device_ptr=film.data_ptr(), stream=stream)
        e1.record()
        torch.cuda.synchronize()
        rows.append((g.width * g.height * s, e0.elapsed_time(e1) / 3))
    tot_p = sum(p for p, _ in rows)
    tot_ms = sum(m for _, m in rows)
    classes = []
    for lo, hi in [(0, 1e5), (1e5, 1e6), (1e6, 4e6), (4e6, 1e18)]:
        sel = [(p, m) for p, m in rows if lo <= p < hi]
        if sel:
            p = sum(x for x, _ in sel)
            m = sum(x for _, x in sel)
            classes.append(dict(paths_from=lo, paths_to=hi, scenes=len(sel), path_share=p / tot_p,
                                time_share=m / tot_ms, m_paths_per_s=p / m / 1e3))
    big = [(p, m) for p, m in rows if p >= 4e6] or rows
    rate_big = sum(p for p, _ in big) / sum(m for _, m in big)
    best = max(p / m for p, m in rows)
    return dict(loop_ms=tot_ms, classes=classes, bound_at_large_scene_rate=tot_ms / (tot_p / rate_big),
                bound_at_best_scene_rate=tot_ms / (tot_p / best))


def adjoint_arm(args):
    """Differentiable inverse rendering: the Cornell box with a seeded 65,536-triangle
    displaced sphere (per-triangle RGB albedo, 196,608 parameters) in a homogeneous medium
    (sigma_s, sigma_a RGB and HG g: 7 parameters); target rendered from the hidden
    parameters at 256x256, 64 spp, depth 8; L2 image loss; Adam (lr 1e-2) from a uniform
    0.5 albedo and a wrong medium.  One step = forward + path-replay backward + update.
    value = gradient evaluations (of all parameters) per second over the timed steps."""
    import numpy as np
    import torch
    import rumi_b200
    from rumi_b200 import scenes
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from adjoint_torch import render, visible_triangles, footprint_albedo_rmse
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    size, spp, depth, levels = 256, 64, 8, args.adjoint_levels
    gt = rumi_b200.GpuScene(scenes.inverse_rendering(size, size, spp, depth, levels=levels))
    target = torch.from_numpy(gt.forward(seed=1)[0] / spp).cuda()
    gt.close()
    n_mesh = 4 * 4 ** levels
    hidden = scenes.random_albedo(n_mesh, 23)
    start = scenes.inverse_rendering(size, size, spp, depth, levels=levels,
                                     albedo=np.full((n_mesh, 3), 0.5, np.float32), medium=scenes.INVERSE_START_MEDIUM)
    g = rumi_b200.GpuScene(start)
    alb_all = torch.from_numpy(start.flatten().tri_albedo.copy()).cuda()
    walls = alb_all[:-n_mesh].clone()
    mesh = torch.nn.Parameter(alb_all[-n_mesh:].clone())
    m0 = scenes.INVERSE_START_MEDIUM
    med = torch.nn.Parameter(torch.tensor(list(m0["sigma_s"]) + list(m0["sigma_a"]) + [m0["g"]],
                                          dtype=torch.float32, device="cuda"))
    opt = torch.optim.Adam([mesh, med], lr=args.adam_lr)
    decay = (args.adam_lr_end / args.adam_lr) ** (1.0 / max(args.adam_steps - 1, 1)) if args.adam_lr_end > 0 else 1.0
    sched = torch.optim.lr_scheduler.ExponentialLR(opt, gamma=decay)
    grad_spp = args.adjoint_spp or spp
    hidden_t = torch.from_numpy(hidden).cuda()

    def step(it):
        film = render(torch.cat([walls, mesh]), med, g, spp, 100 + it, grad_spp=grad_spp) / spp
        loss = ((film - target) ** 2).mean()
        opt.zero_grad()
        loss.backward()
        opt.step()
        with torch.no_grad():
            mesh.clamp_(0.01, 1.0)
            med[0:6].clamp_(1e-3, 5.0)
            med[6].clamp_(-0.9, 0.9)
        return loss.detach()

    # forward / backward split, measured on the start parameters before optimising
    d = np.ones((size, size, 3), np.float32)
    for _ in range(3):
        g.forward(seed=7, timing=True)
        g.backward(d, seed=7, timing=True)
    fwd_ms = statistics.median(g.forward(seed=8 + i, timing=True)[1]["total_ms"] for i in range(5))
    bwd_ms = statistics.median(g.backward(d, seed=8 + i, timing=True)[2]["total_ms"] for i in range(5))
    # the same backward right after a forward of the same frame that kept its per-path
    # radiance (RUMI_FLAG_KEEP_RADIANCE): only the replay pass is traced.  (The optimisation
    # loop below draws the adjoint's paths with another seed, so it cannot use this.)
    kept = []
    for i in range(5):
        g.forward(seed=8 + i, keep=True)
        kept.append(g.backward(d, seed=8 + i, timing=True)[2]["total_ms"])
    bwd_kept_ms = statistics.median(kept)
    def crn_loss():
        """The image loss against the target rendered with the same seed as the target
        (common random numbers): what remains is the parameters' difference, not noise."""
        with torch.no_grad():
            film = render(torch.cat([walls, mesh]), med, g, spp, 1) / spp
            return float(((film - target) ** 2).mean())

    crn0 = crn_loss()
    alb_rmse0 = float(((mesh.detach() - hidden_t) ** 2).mean().sqrt())
    # the triangles the camera sees (>= 1 pixel): only their albedo is observable
    vis = torch.from_numpy(visible_triangles(g, start, alb_all.shape[0] - n_mesh, n_mesh)).cuda()
    vis_rmse0 = float(((mesh.detach() - hidden_t)[vis] ** 2).mean().sqrt())
    # what a 256x256 image observes of the albedo: its average over each pixel's footprint
    first_mesh = alb_all.shape[0] - n_mesh
    fp_rmse0 = footprint_albedo_rmse(g, start, first_mesh, n_mesh, mesh.detach(), hidden_t)
    for it in range(args.warmup):
        step(-1 - it)
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    losses = []
    for it in range(args.adam_steps):
        losses.append(step(it))
        sched.step()
    ev1.record()
    torch.cuda.synchronize()
    clocks_info = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    losses = [float(x) for x in losses]
    crn1 = crn_loss()
    alb_rmse = float(((mesh.detach() - hidden_t) ** 2).mean().sqrt())
    vis_rmse = float(((mesh.detach() - hidden_t)[vis] ** 2).mean().sqrt())
    fp_rmse = footprint_albedo_rmse(g, start, first_mesh, n_mesh, mesh.detach(), hidden_t)
    t = scenes.INVERSE_TARGET_MEDIUM
    m_tgt = np.array(list(t["sigma_s"]) + list(t["sigma_a"]) + [t["g"]])
    m_start = np.array(list(m0["sigma_s"]) + list(m0["sigma_a"]) + [m0["g"]])
    m_end = med.detach().cpu().numpy()
    line = dict(metric="adjoint grads/s", value=args.adam_steps / (ms / 1000.0), unit="gradient evaluations/s",
                n_gpus=1, steps=args.adam_steps, warmup=args.warmup, ms_per_step=ms / args.adam_steps,
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
                data=f"synthetic (seeded {n_mesh:,}-triangle displaced sphere, hidden seeded albedo and medium)",
                config=dict(workload=f"inverse rendering: 256x256, 64 spp, depth 8, {n_mesh:,} triangles in a medium",
                            params=3 * n_mesh + 7,
                            optimiser=f"Adam lr {args.adam_lr:g}" + (f" -> {args.adam_lr_end:g} (exponential)"
                                                                    if args.adam_lr_end > 0 else ""),
                            loss="L2 image",
                            gradient_spp=grad_spp),
                forward_ms=fwd_ms, backward_ms=bwd_ms, backward_over_forward=bwd_ms / fwd_ms,
                backward_after_kept_forward_ms=bwd_kept_ms,
                paths_per_step=size * size * spp, loss_first=losses[0], loss_last=losses[-1],
                loss_first20_mean=float(np.mean(losses[:20])), loss_last20_mean=float(np.mean(losses[-20:])),
                loss_same_seed_as_target_start=crn0, loss_same_seed_as_target_end=crn1,
                albedo_rmse_start=alb_rmse0, albedo_rmse_end=alb_rmse,
                visible_triangles=int(vis.sum()), visible_albedo_rmse_start=vis_rmse0,
                visible_albedo_rmse_end=vis_rmse, footprint_albedo_rmse_start=fp_rmse0,
                footprint_albedo_rmse_end=fp_rmse,
                medium_end=[float(x) for x in med.detach().cpu()],
                medium_target=list(t["sigma_s"]) + list(t["sigma_a"]) + [t["g"]],
                # sums of absolute errors: sigma_s RGB, sigma_a RGB, g
                medium_error_start=[float(np.abs(m_start - m_tgt)[0:3].sum()), float(np.abs(m_start - m_tgt)[3:6].sum()),
                                    float(abs(m_start[6] - m_tgt[6]))],
                medium_error_end=[float(np.abs(m_end - m_tgt)[0:3].sum()), float(np.abs(m_end - m_tgt)[3:6].sum()),
                                  float(abs(m_end[6] - m_tgt[6]))],
                gpu_launches=args.adam_steps * ((3 + 5 * depth) + 2 * (3 + 4 * depth)), clocks=clocks_info)
    print(json.dumps(line), flush=True)
    g.close()
    return 0


def bdpt_arm(args):
    """BDPT with MIS on the volumetric caustic: glass sphere (IOR 1.5, r 0.3) in a
    homogeneous medium (sigma_a 0.05, sigma_s 0.4, HG g 0.7) lit by a 30-degree spot of
    intensity 50; 512x512, 32 spp, max path length 12 (6 light + 7 eye vertices).
    One step = one frame; value = camera samples (full bidirectional paths) per second.
    cpu_baseline: the reference's BidirectionalPathTracer on the variant it can express
    (isotropic medium, small area light in place of the spot), a bounded row sample."""
    import torch
    import rumi_b200
    from rumi_b200 import scenes
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    W, H, spp, nL, nE = 512, 512, 32, 6, 7
    if args.small:  # 128x128: one wave, for profiler captures
        W = H = 128
    gs = rumi_b200.GpuScene(scenes.volumetric_caustic(W, H, spp, nL, nE))
    stream = torch.cuda.current_stream().cuda_stream
    film = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    for s in range(args.warmup):
        gs.render(seed=s, film_device_ptr=film.data_ptr(), stream=stream)
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    launches = 0
    for s in range(args.steps):
        _, st = gs.render(seed=100 + s, film_device_ptr=film.data_ptr(), stream=stream)
        launches += st["extend_launches"] + 1  # per wave: bdpt_kernel + bdpt_write_film; + add_light_film
    ev1.record()
    torch.cuda.synchronize()
    clocks_info = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    paths = W * H * spp
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import refimpl
        sc = scenes.volumetric_caustic(W, H, spp, nL, nE, parity=True)
        rs = refimpl.RefScene(sc, seed=1)
        t0 = time.perf_counter()
        rows = 2
        rs.render_rows(5, 0, rows)
        sec = time.perf_counter() - t0
        n = rows * W * rs.spp
        cpu = dict(value=n / sec, unit="paths/s", cores=1, kind="reference",
                   sample=f"{n} camera samples = {rows} rows x {W} px x {rs.spp} spp of the area-light, isotropic "
                          "variant (the reference has no spot light or HG phase; it truncates spp to a square), "
                          "BidirectionalPathTracer(6, 7), one thread", seconds=sec)
        rs.close()
    gs.close()
    line = dict(metric="path samples/sec (BDPT camera samples)", value=args.steps * paths / (ms / 1000.0),
                unit="paths/s", n_gpus=1, steps=args.steps, warmup=args.warmup, ms_per_step=ms / args.steps,
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
                data="synthetic (analytic scene)",
                config=dict(workload="volumetric caustic BDPT: glass sphere in HG medium, 30-degree spot", width=W,
                            height=H, spp=spp, n_light=nL, n_eye=nE, max_path_length=nL + nE - 1),
                cpu_baseline=cpu, gpu_launches=launches, clocks=clocks_info)
    print(json.dumps(line), flush=True)
    return 0


def cornell_arm(args):
    """The plain path-tracer Cornell workload, the reference's own CPU-runnable case:
    5 walls, area light, a Lambertian and a mirror sphere; 256x256, 16 spp, depth 8
    (1,048,576 paths per frame).  value = paths/s on the device; cpu_baseline = the
    reference renderer itself on a row sample of the same frame, one thread."""
    import torch
    import rumi_b200
    from rumi_b200 import scenes
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    W, H, spp, depth = 256, 256, 16, 8
    sc = scenes.cornell_pt(W, H, spp, depth)
    gs = rumi_b200.GpuScene(sc)
    stream = torch.cuda.current_stream().cuda_stream
    film = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    steps = max(args.steps, 20)
    for s in range(args.warmup):
        gs.render(seed=s, film_device_ptr=film.data_ptr(), stream=stream)
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    launches = 0
    for s in range(steps):
        _, st = gs.render(seed=100 + s, film_device_ptr=film.data_ptr(), stream=stream)
        launches += (st["extend_launches"] // depth) * (3 + 5 * depth)
    ev1.record()
    torch.cuda.synchronize()
    clocks_info = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import refimpl
        rs = refimpl.RefScene(sc, seed=1)
        rows = 16
        t0 = time.perf_counter()
        rs.render_rows(5, 0, rows)
        sec = time.perf_counter() - t0
        n = rows * W * rs.spp
        cpu = dict(value=n / sec, unit="paths/s", cores=1, kind="reference",
                   sample=f"{n} paths = {rows} rows x {W} px x {rs.spp} spp of the same frame, PathTracer(8), "
                          f"one thread, CPU {cpu_model()}", seconds=sec)
        rs.close()
    gs.close()
    line = dict(metric="path samples/sec", value=steps * W * H * spp / (ms / 1000.0), unit="paths/s", n_gpus=1,
                steps=steps, warmup=args.warmup, ms_per_step=ms / steps, higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f32", data="synthetic (analytic scene)",
                config=dict(workload="cornell_pt: plain path tracer, Cornell box", width=W, height=H, spp=spp,
                            max_depth=depth),
                cpu_baseline=cpu, gpu_launches=launches, clocks=clocks_info)
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "batched":
        return batched_arm(args)
    if args.workload == "adjoint":
        return adjoint_arm(args)
    if args.workload == "bdpt_caustic":
        return bdpt_arm(args)
    if args.workload == "cornell":
        return cornell_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
