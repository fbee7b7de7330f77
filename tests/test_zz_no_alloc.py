"""rumi_render_noalloc -- the render entry point that allocates no device memory, for
callers that may not call cudaMalloc once running (a fixed device-memory budget owned
by the embedding application, real-time loops that cannot take the allocator's
device-wide synchronisation).

It must produce the same film as rumi_render (the regular entry point) on two calls in a
row -- the second call reuses the shared scratch array the first one left behind -- and
refuse requests that do not fit its fixed array.  Further cases: a caller's own stream,
waves shorter than one pixel's samples, traversal counters, and a pixel of exactly the
largest sample count the array holds.  This file is collected last so that a run stopping
at the first failure has run every other test first; it also passes when run alone in a
fresh process."""
import ctypes as C

import numpy as np
import pytest

import rumi_b200
from rumi_b200 import _capi, scenes

pytestmark = pytest.mark.gpu


def _params(spp, depth, seed, wave_paths=0, flags=0):
    p = _capi.rumi_render_params()
    p.integrator, p.max_depth, p.spp, p.seed = 0, depth, spp, seed
    p.wave_paths, p.flags = wave_paths, flags
    return p


def test_noalloc_render_matches_rumi_render_on_two_calls():
    import torch
    torch.cuda.set_device(0)
    lib = _capi.load()
    sc = scenes.cornell_pt(96, 80, 16, 6)
    gs = rumi_b200.GpuScene(sc)
    film_dev = torch.zeros((80, 96, 3), dtype=torch.float32, device="cuda")
    for seed in (21, 22):  # two calls in a row on the shared scratch
        want, wst = gs.render(spp=16, seed=seed)
        st = _capi.rumi_render_stats()
        film_dev.fill_(-1.0)
        torch.cuda.synchronize()
        rc = lib.rumi_render_noalloc(gs.h, C.byref(_params(16, 6, seed)), C.c_void_p(film_dev.data_ptr()),
                                     C.byref(st))
        assert rc == 0, lib.rumi_last_error_string()
        got = film_dev.cpu().numpy()
        # same per-path random streams and per-pixel summation order -> same film
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=0)
        assert st.paths == wst["paths"] == 96 * 80 * 16
        assert st.nan_samples == wst["nan_samples"] == 0
        assert st.rays_extend == wst["rays_extend"]
    gs.close()


def test_noalloc_rejects_requests_beyond_its_scratch():
    import torch
    torch.cuda.set_device(0)
    lib = _capi.load()
    gs = rumi_b200.GpuScene(scenes.cornell_pt(16, 16, 1, 2))
    film_dev = torch.zeros((16, 16, 3), dtype=torch.float32, device="cuda")
    ptr = C.c_void_p(film_dev.data_ptr())
    assert lib.rumi_render_noalloc(gs.h, C.byref(_params(1 << 20, 2, 1)), ptr, None) == 1
    assert b"exceeds" in lib.rumi_last_error_string()
    assert lib.rumi_render_noalloc(gs.h, C.byref(_params(4, 2, 1, wave_paths=1 << 24)), ptr, None) == 1
    assert lib.rumi_render_noalloc(gs.h, C.byref(_params(4, 2, 1, flags=1)), ptr, None) == 1
    assert lib.rumi_render_noalloc(gs.h, C.byref(_params(4, 2, 1)), None, None) == 1
    # a valid call still works after the rejected ones
    assert lib.rumi_render_noalloc(gs.h, C.byref(_params(4, 2, 1)), ptr, None) == 0
    torch.cuda.synchronize()
    assert np.isfinite(film_dev.cpu().numpy()).all()
    gs.close()


def _noalloc(lib, gs, params, film_dev):
    st = _capi.rumi_render_stats()
    rc = lib.rumi_render_noalloc(gs.h, C.byref(params), C.c_void_p(film_dev.data_ptr()), C.byref(st))
    assert rc == 0, lib.rumi_last_error_string()
    return st


def test_noalloc_on_a_caller_stream_and_short_waves():
    import torch
    torch.cuda.set_device(0)
    lib = _capi.load()
    sc = scenes.cornell_pt(40, 24, 16, 5)
    gs = rumi_b200.GpuScene(sc)
    want, _ = gs.render(spp=16, seed=5)
    film_dev = torch.zeros((24, 40, 3), dtype=torch.float32, device="cuda")
    # a caller-owned stream
    s = torch.cuda.Stream()
    p = _params(16, 5, 5)
    p.stream = C.c_void_p(s.cuda_stream)
    with torch.cuda.stream(s):
        film_dev.fill_(-1.0)
    _noalloc(lib, gs, p, film_dev)
    s.synchronize()
    np.testing.assert_allclose(film_dev.cpu().numpy(), want, rtol=1e-6, atol=0)
    # waves of fewer paths than one pixel's samples: one pixel per wave
    film_dev.fill_(-1.0)
    torch.cuda.synchronize()
    _noalloc(lib, gs, _params(16, 5, 5, wave_paths=7), film_dev)
    np.testing.assert_allclose(film_dev.cpu().numpy(), want, rtol=1e-6, atol=0)
    gs.close()


def test_noalloc_traversal_counters_match_rumi_render():
    import torch
    torch.cuda.set_device(0)
    lib = _capi.load()
    gs = rumi_b200.GpuScene(scenes.cornell_pt(32, 32, 4, 4))
    want, wst = gs.render(spp=4, seed=9, count_stats=True)
    film_dev = torch.zeros((32, 32, 3), dtype=torch.float32, device="cuda")
    st = _noalloc(lib, gs, _params(4, 4, 9, flags=2), film_dev)  # RUMI_FLAG_STATS
    np.testing.assert_allclose(film_dev.cpu().numpy(), want, rtol=1e-6, atol=0)
    assert st.rays_extend == wst["rays_extend"]
    # the speculative walk's culling depends on which rays share a warp (work is fetched
    # dynamically), so the counts agree closely rather than exactly
    assert wst["extend_node_fetches"] > 0 and wst["extend_prim_tests"] > 0
    assert abs(st.extend_node_fetches / wst["extend_node_fetches"] - 1.0) < 0.05
    assert abs(st.extend_prim_tests / wst["extend_prim_tests"] - 1.0) < 0.05
    gs.close()


def test_noalloc_pixel_at_the_array_capacity():
    import re
    import torch
    torch.cuda.set_device(0)
    lib = _capi.load()
    gs = rumi_b200.GpuScene(scenes.cornell_pt(2, 1, 1, 2))
    film_dev = torch.zeros((1, 2, 3), dtype=torch.float32, device="cuda")
    ptr = C.c_void_p(film_dev.data_ptr())
    assert lib.rumi_render_noalloc(gs.h, C.byref(_params(1 << 24, 2, 1)), ptr, None) == 1
    cap = int(re.search(rb"the (\d+) paths", lib.rumi_last_error_string()).group(1))
    assert 90000 < cap < 100000  # 16 MiB at 176 bytes per path
    assert lib.rumi_render_noalloc(gs.h, C.byref(_params(cap + 1, 2, 1)), ptr, None) == 1
    want, wst = gs.render(spp=cap, seed=3)
    st = _noalloc(lib, gs, _params(cap, 2, 3), film_dev)
    np.testing.assert_allclose(film_dev.cpu().numpy(), want, rtol=1e-6, atol=0)
    assert st.paths == wst["paths"] == 2 * cap
    gs.close()


def test_noalloc_eight_wide_walk_only_after_its_tree_is_built():
    """trace_mode 5 needs the eight-wide tree, which the library collapses on first use;
    the no-allocation entry point cannot build it, so it refuses 5 until a regular call
    has, and afterwards renders the film rumi_render renders with 5."""
    import torch
    torch.cuda.set_device(0)
    lib = _capi.load()
    gs = rumi_b200.GpuScene(scenes.cornell_pt(48, 40, 4, 4))
    film_dev = torch.zeros((40, 48, 3), dtype=torch.float32, device="cuda")
    p = _params(4, 4, 5)
    p.trace_mode = 5
    st = _capi.rumi_render_stats()
    assert lib.rumi_render_noalloc(gs.h, C.byref(p), C.c_void_p(film_dev.data_ptr()), C.byref(st)) != 0
    assert b"eight-wide" in lib.rumi_last_error_string()
    want, _ = gs.render(spp=4, seed=5, trace_mode=5)  # builds the tree
    rc = lib.rumi_render_noalloc(gs.h, C.byref(p), C.c_void_p(film_dev.data_ptr()), C.byref(st))
    assert rc == 0, lib.rumi_last_error_string()
    np.testing.assert_allclose(film_dev.cpu().numpy(), want, rtol=1e-6, atol=0)
    gs.close()
