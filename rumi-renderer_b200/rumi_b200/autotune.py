"""Autotuner of the renderer's launch parameters.

Knobs (fields of rumi_render_params): ``trace_mode`` (traversal scheme of the persistent
ray kernels), ``blocks_per_sm`` (persistent traversal blocks per SM, i.e. warps per SM in
steps of 4), ``refill_min`` (idle lanes that trigger a per-lane refill), ``wave_paths``
(queue capacity: paths in flight per wave) and ``stack_depth`` (traversal stack entries
per thread in shared memory).  Each candidate renders the given scene and is
timed on the device (RUMI_FLAG_TIMING); the search is coordinate descent from the library
defaults.  Results are cached per GPU model and workload key in a JSON file.
"""
from __future__ import annotations

import json
import os
import time

# What the library uses when a knob is 0 (include/rumi_b200.h, rumi_render_params): the
# speculative while-while walk (trace_mode 4), the occupancy limit of traversal blocks, a
# refill at 8 idle lanes, 2^25 paths per wave and 16 stack entries in shared memory.  The
# search starts there.
DEFAULTS = dict(trace_mode=4, blocks_per_sm=0, refill_min=8, wave_paths=1 << 25, stack_depth=16)
SPACE = dict(trace_mode=[4, 5, 1, 2, 3], blocks_per_sm=[0, 4, 5, 6], refill_min=[4, 8, 16],
             wave_paths=[1 << 25, 1 << 22, 1 << 23, 1 << 24], stack_depth=[16, 32, 8])
def default_cache_path() -> str:
    """$RUMI_TUNING_CACHE, else autotune_cache.json under the user's cache directory
    ($XDG_CACHE_HOME or ~/.cache)/rumi_b200 -- never inside the package tree."""
    if os.environ.get("RUMI_TUNING_CACHE"):
        return os.environ["RUMI_TUNING_CACHE"]
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "rumi_b200", "autotune_cache.json")


CACHE = default_cache_path()


def gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown-gpu"


def measure(gs, tuning: dict, spp: int, seed: int = 12345, repeats: int = 1, film_ptr=None) -> float:
    """Device milliseconds of one frame with these launch parameters (best of repeats)."""
    best = float("inf")
    for r in range(repeats):
        _, st = gs.render(spp=spp, seed=seed + r, timing=True, tuning=tuning, film_device_ptr=film_ptr)
        best = min(best, st["total_ms"])
    return best


def tune(gs, spp: int, key: str, space: dict = None, repeats: int = 2, film_ptr=None, log=None,
         cache_path: str = CACHE) -> dict:
    """Coordinate descent over the knobs; returns the best parameters and caches them."""
    space = space or SPACE
    cur = dict(DEFAULTS)
    cur_ms = measure(gs, cur, spp, repeats=repeats, film_ptr=film_ptr)
    history = [(dict(cur), cur_ms)]
    seen = {tuple(sorted(cur.items()))}
    for knob in ("trace_mode", "blocks_per_sm", "refill_min", "wave_paths", "stack_depth"):
        for v in space[knob]:
            cand = dict(cur)
            cand[knob] = v
            if tuple(sorted(cand.items())) in seen:
                continue
            seen.add(tuple(sorted(cand.items())))
            ms = measure(gs, cand, spp, repeats=repeats, film_ptr=film_ptr)
            history.append((dict(cand), ms))
            if log:
                log(f"{knob}={v}: {ms:.2f} ms (best {cur_ms:.2f})")
            if ms < cur_ms:
                cur, cur_ms = cand, ms
    result = dict(params=cur, ms=cur_ms, gpu=gpu_name(), key=key, when=time.strftime("%Y-%m-%dT%H:%M:%S"),
                  history=[dict(params=p, ms=m) for p, m in history])
    save(key, result, cache_path)
    return result


BATCH_WAVES = [1 << 22, 1 << 23, 1 << 24, 1 << 25]


def tune_batch(batch, spp, seeds, max_depth: int, key: str, waves=None, repeats: int = 2, log=None,
               cache_path: str = CACHE) -> dict:
    """Queue capacity (paths in flight per wave) of a multi-scene batch: each candidate
    renders the batch eagerly (no graph) and is timed on the device; the best is cached
    and is the capacity to capture the frame's CUDA graph with."""
    best, best_ms, history = None, float("inf"), []
    for w in waves or BATCH_WAVES:
        ms = float("inf")
        for r in range(repeats):
            _, st = batch.render(spp, seeds, max_depth, graph=False, timing=True, wave_paths=w)
            ms = min(ms, st["total_ms"])
        history.append(dict(params=dict(wave_paths=w), ms=ms))
        if log:
            log(f"batch wave_paths={w}: {ms:.2f} ms")
        if ms < best_ms:
            best, best_ms = w, ms
    result = dict(params=dict(wave_paths=best), ms=best_ms, gpu=gpu_name(), key=key,
                  when=time.strftime("%Y-%m-%dT%H:%M:%S"), history=history)
    save(key, result, cache_path)
    return result


def load(key: str, cache_path: str = CACHE):
    try:
        data = json.load(open(cache_path))
    except Exception:
        return None
    return data.get(f"{gpu_name()}|{key}")


def save(key: str, result: dict, cache_path: str = CACHE):
    os.makedirs(os.path.dirname(cache_path), exist_ok=True)
    try:
        data = json.load(open(cache_path))
    except Exception:
        data = {}
    data[f"{result['gpu']}|{key}"] = result
    json.dump(data, open(cache_path, "w"), indent=1)
