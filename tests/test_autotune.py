"""The autotuner's search and cache on CPU, against fake render objects with a known
cost surface (the GPU measurement itself is exercised by bench runs)."""
import os

import pytest

from rumi_b200 import autotune


class FakeScene:
    """total_ms is smallest at trace_mode=2, blocks_per_sm=5, refill_min=4, wave 8M."""

    def __init__(self):
        self.calls = 0

    def render(self, spp=None, seed=0, timing=False, tuning=None, film_device_ptr=None):
        self.calls += 1
        t = tuning
        ms = 100.0
        ms += {1: 10.0, 2: 0.0, 3: 30.0, 4: 6.0, 5: 7.0}[t["trace_mode"]]
        ms += {0: 4.0, 4: 8.0, 5: 0.0, 6: 2.0}[t["blocks_per_sm"]]
        ms += {4: 0.0, 8: 1.0, 16: 3.0}[t["refill_min"]]
        ms += {1 << 22: 5.0, 1 << 23: 2.0, 1 << 24: 0.0, 1 << 25: 1.0}[t["wave_paths"]]
        ms += {32: 1.0, 16: 0.0, 8: 0.5}[t["stack_depth"]]
        return None, {"total_ms": ms}


class FakeBatch:
    def render(self, spp, seeds, max_depth, graph=False, timing=False, wave_paths=0):
        return None, {"total_ms": {1 << 22: 9.0, 1 << 23: 7.0, 1 << 24: 8.0, 1 << 25: 10.0}[wave_paths]}


def test_coordinate_descent_finds_the_optimum_and_caches(tmp_path):
    cache = str(tmp_path / "cache.json")
    g = FakeScene()
    res = autotune.tune(g, spp=4, key="fake", repeats=1, cache_path=cache)
    assert res["params"] == dict(trace_mode=2, blocks_per_sm=5, refill_min=4, wave_paths=1 << 24, stack_depth=16)
    assert res["ms"] == 100.0
    # one baseline + every alternative value of every knob
    assert g.calls == 1 + sum(len(v) - 1 for v in autotune.SPACE.values())
    again = autotune.load("fake", cache_path=cache)
    assert again["params"] == res["params"] and again["gpu"] == res["gpu"]


def test_batch_queue_capacity(tmp_path):
    cache = str(tmp_path / "cache.json")
    res = autotune.tune_batch(FakeBatch(), [4], [1], 8, key="batch", repeats=1, cache_path=cache)
    assert res["params"] == dict(wave_paths=1 << 23)
    assert autotune.load("batch", cache_path=cache)["ms"] == 7.0


def test_search_starts_from_the_library_defaults():
    """The starting point is what the library does with every knob at 0 (the speculative
    walk, trace_mode 4), and every traversal scheme of rumi_render_params is searched."""
    assert autotune.DEFAULTS["trace_mode"] == 4
    assert sorted(autotune.SPACE["trace_mode"]) == [1, 2, 3, 4, 5]
    for k, v in autotune.DEFAULTS.items():
        assert v in autotune.SPACE[k], k
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "rumi_b200.h")).read()
    assert "4: speculative while-while walk" in hdr


def test_cache_lives_outside_the_package(monkeypatch, tmp_path):
    monkeypatch.delenv("RUMI_TUNING_CACHE", raising=False)
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    assert autotune.default_cache_path() == str(tmp_path / "rumi_b200" / "autotune_cache.json")
    monkeypatch.setenv("RUMI_TUNING_CACHE", str(tmp_path / "x.json"))
    assert autotune.default_cache_path() == str(tmp_path / "x.json")
    pkg = os.path.dirname(os.path.abspath(autotune.__file__))
    assert not autotune.CACHE.startswith(os.path.dirname(pkg))


@pytest.mark.gpu
def test_gpu_tune_on_a_small_scene_keeps_the_film(tmp_path):
    """tune() on the device over a small scene: it measures every candidate, caches the
    best, and the chosen launch parameters render the film the defaults render (launch
    parameters change the schedule, never a result)."""
    import numpy as np
    import torch
    import rumi_b200
    from rumi_b200 import scenes
    torch.cuda.set_device(0)
    gs = rumi_b200.GpuScene(scenes.bvh_bound_pt(64, 64, 4, 6, levels=5, seed=7))
    space = dict(trace_mode=[autotune.DEFAULTS["trace_mode"], 1], blocks_per_sm=[0, 4], refill_min=[8, 16],
                 wave_paths=[autotune.DEFAULTS["wave_paths"], 1 << 14], stack_depth=[16, 8])
    res = autotune.tune(gs, spp=4, key="small", space=space, repeats=1, cache_path=str(tmp_path / "c.json"))
    assert len(res["history"]) == 1 + 5 and all(h["ms"] > 0 for h in res["history"])
    assert autotune.load("small", cache_path=str(tmp_path / "c.json"))["params"] == res["params"]
    want, _ = gs.render(spp=4, seed=77)
    got, _ = gs.render(spp=4, seed=77, tuning=res["params"])
    np.testing.assert_array_equal(got, want)
    gs.close()
