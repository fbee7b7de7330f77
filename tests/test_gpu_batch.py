"""Multi-scene batches (rumi_render_batch): scenes of uneven size, sample count and
material rendered as one frame from shared queues must produce, for every scene, the
film rumi_render produces for that scene alone with the same seed -- bit for bit, since
each scene keeps its own Philox key and path numbering.  Equal images mean equal RMSE,
which is what the batched-vs-plain throughput comparison rests on."""
import numpy as np
import pytest

import rumi_b200
from rumi_b200 import scenes

pytestmark = pytest.mark.gpu

# (res, spp, n_tris): non-square spp, a pixel count that is not a multiple of any wave
CASES = [(32, 4, 1200), (48, 16, 5000), (16, 1, 2000), (40, 5, 30000), (24, 64, 1000), (8, 3, 1500)]
DEPTH = 5


@pytest.fixture(scope="module")
def batch_scenes():
    gs = [rumi_b200.GpuScene(scenes.batch_scene(i, DEPTH, res=r, spp=s, n_tris=n))
          for i, (r, s, n) in enumerate(CASES)]
    yield gs
    for g in gs:
        g.close()


def singles(gs, seeds, wave_paths=0, with_stats=False):
    out = [g.render(spp=s, seed=int(sd), wave_paths=wave_paths)
           for g, (_, s, _), sd in zip(gs, CASES, seeds)]
    return out if with_stats else [f for f, _ in out]


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("wave_paths", [0, 1000, 4099])
def test_batch_equals_per_scene_renders(batch_scenes, graph, wave_paths):
    seeds = [11 + 7 * i for i in range(len(CASES))]
    ref_st = singles(batch_scenes, seeds, with_stats=True)
    ref = [f for f, _ in ref_st]
    b = rumi_b200.GpuBatch(batch_scenes)
    try:
        films, st = b.render([c[1] for c in CASES], seeds, DEPTH, graph=graph, wave_paths=wave_paths)
        assert st["paths"] == sum(r * r * s for r, s, _ in CASES)
        # the frame's ray counts are the scenes' own, read from the batch workspace
        for k in ("rays_extend", "rays_shadow", "nan_samples"):
            assert st[k] == sum(x[k] for _, x in ref_st), k
        for k, (f, r) in enumerate(zip(films, ref)):
            assert np.array_equal(f, r), k
            assert f.sum() > 0
        if graph:
            # replay with new seeds: the graph reads the key table, nothing is re-captured
            seeds2 = [1000 + s for s in seeds]
            films2, _ = b.render([c[1] for c in CASES], seeds2, DEPTH, graph=True, wave_paths=wave_paths)
            for f, r in zip(films2, singles(batch_scenes, seeds2)):
                assert np.array_equal(f, r)
    finally:
        b.close()


def test_batch_device_films_and_scene_order(batch_scenes):
    """Films land concatenated in scene order; reversing the batch reverses them."""
    import torch
    seeds = [5] * len(CASES)
    rev = batch_scenes[::-1]
    b = rumi_b200.GpuBatch(rev)
    try:
        n = b.n_floats
        buf = torch.zeros(n, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        _, st = b.render([c[1] for c in CASES[::-1]], seeds, DEPTH, films_device_ptr=buf.data_ptr(), timing=True)
        torch.cuda.synchronize()
        flat = buf.cpu().numpy()
        o = 0
        for g, f in zip(rev, singles(batch_scenes, seeds)[::-1]):
            m = g.height * g.width * 3
            assert np.array_equal(flat[o:o + m].reshape(f.shape), f)
            o += m
        assert o == n and st["total_ms"] > 0
    finally:
        b.close()


def test_batch_rejects_bad_arguments(batch_scenes):
    b = rumi_b200.GpuBatch(batch_scenes[:2])
    try:
        with pytest.raises(rumi_b200._capi.RumiError):
            b.render([4, 0], [1, 2], DEPTH)
        with pytest.raises(rumi_b200._capi.RumiError):
            b.render([4, 16], [1, 2], 0)
    finally:
        b.close()
