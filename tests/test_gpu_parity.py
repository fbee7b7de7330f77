"""GPU parity: the CUDA path (through the C-ABI) against the reference's own outputs
(golden vectors and the live reference build in oracle/_ref) and against the CPU oracle
on identical seeded inputs.

Tolerances: primitive ids bit-exact except exact-t ties; hit distances bit-exact (the
intersection arithmetic is restated with correctly rounded operations); BSDF / phase /
medium / camera routines within 1e-5; renders: per-pixel agreement with the oracle on the
same random stream, and per-pixel means within 3 sigma of the reference's frames."""
import ctypes as C

import numpy as np
import pytest

import oraclelib as O
import refimpl
import rumi_b200
from rumi_b200 import _capi, scenes
from test_oracle_golden import KAT, MATERIALS, material_from_params, rays8, tie_mask

pytestmark = pytest.mark.gpu


def vp(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.fixture(scope="module")
def lib():
    return _capi.load()


def test_gpu_philox_known_answers_and_oracle(lib):
    rng = np.random.default_rng(5)
    ctr = rng.integers(0, 2 ** 32, size=(4096, 4), dtype=np.uint64).astype(np.uint32)
    for c, k, want in KAT:
        ctr1 = np.array([c], np.uint32)
        out = np.zeros((1, 4), np.uint32)
        assert lib.rumi_test_philox(1, vp(ctr1), vp(np.array(k, np.uint32)), vp(out)) == 0
        assert tuple(int(x) for x in out[0]) == want
    key = np.array([0x12345678, 0x9ABCDEF0], np.uint32)
    out = np.zeros((4096, 4), np.uint32)
    assert lib.rumi_test_philox(4096, vp(ctr), vp(key), vp(out)) == 0
    for i in range(0, 4096, 97):
        assert list(out[i]) == O.philox([int(x) for x in ctr[i]], [int(x) for x in key])


@pytest.mark.parametrize("fixture,builder", [
    ("hits_cornell.npz", lambda: scenes.cornell_pt(64, 64, 16, 8)),
    ("hits_mesh5.npz", lambda: scenes.bvh_bound_pt(64, 64, 4, 10, levels=5, seed=7)),
])
def test_gpu_hits_match_reference_golden(golden, fixture, builder):
    g = golden(fixture)
    gs = rumi_b200.GpuScene(builder())
    t, prim, nv, pt = gs.trace(g["rays"])
    ties = tie_mask(t, prim, g["t"], g["prim"])
    assert np.all((prim == g["prim"]) | ties)
    assert ties.mean() < 0.01
    np.testing.assert_array_equal(t, g["t"])
    for key in ("shadow", "shadow2"):
        _, occ, _, _ = gs.trace(g[f"{key}_rays"], anyhit=True)
        np.testing.assert_array_equal(occ, g[f"{key}_occluded"])
    gs.close()


def test_gpu_hits_1m_mesh_match_live_reference():
    """The 1,048,576-triangle workload mesh: GPU SAH BVH vs the reference's own BVHAccel."""
    sc = scenes.bvh_bound_pt(64, 64, 4, 10, levels=9, seed=7)
    rng = np.random.default_rng(11)
    n = 16384
    o = np.tile(np.array([[0.5, 0.5, -1.4]], np.float32), (n, 1))
    tgt = rng.uniform([0.2, 0.1, 0.2], [0.8, 0.6, 0.8], (n, 3)).astype(np.float32)
    d = tgt - o
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    rays = np.concatenate([o, d, np.full((n, 1), 3.4e38, np.float32)], 1).astype(np.float32)
    # secondary rays from inside the box toward the mesh
    o2 = rng.uniform(0.05, 0.95, (n, 3)).astype(np.float32)
    d2 = rng.normal(size=(n, 3)).astype(np.float32)
    d2 /= np.linalg.norm(d2, axis=1, keepdims=True)
    rays = np.concatenate([rays, np.concatenate([o2, d2, np.full((n, 1), 3.4e38, np.float32)], 1)]).astype(np.float32)
    gs = rumi_b200.GpuScene(sc)
    t, prim, nv, pt = gs.trace(rays)
    rs = refimpl.RefScene(sc, seed=1)
    rt, rid = rs.trace(rays)
    ties = tie_mask(t, prim, rt, rid)
    assert np.all((prim == rid) | ties)
    np.testing.assert_array_equal(t, rt)
    sh = rays.copy()
    sh[:, 6] = np.where(rt > 0, rt * 0.5, 0.5)
    _, occ, _, _ = gs.trace(sh, anyhit=True)
    _, rocc = rs.trace(sh, anyhit=True)
    np.testing.assert_array_equal(occ, rocc)
    rs.close()
    gs.close()


@pytest.mark.parametrize("name", MATERIALS)
def test_gpu_material_sample_and_fr_match_reference(golden, lib, name):
    g = golden("materials.npz")
    m = O.material_struct(material_from_params(g[f"{name}_type"], g[f"{name}_params"]))
    n, wo, u, ref = g[f"{name}_n"], g[f"{name}_wo"], g[f"{name}_u"], g[f"{name}_sample"]
    N = n.shape[0]
    out = np.zeros((N, 9), np.float32)
    assert lib.rumi_test_material_sample(C.byref(m), N, vp(wo), vp(n), vp(u), vp(out)) == 0
    np.testing.assert_allclose(out[:, 0:3], ref[:, 0:3], rtol=0, atol=1e-5)
    np.testing.assert_array_equal(out[:, 3:5], ref[:, 3:5])
    np.testing.assert_allclose(out[:, 5:9], ref[:, 5:9], rtol=1e-5, atol=1e-7)
    fr = np.zeros((N, 3), np.float32)
    wi = np.ascontiguousarray(ref[:, 0:3])
    xi = np.ascontiguousarray(ref[:, 5])
    pp = np.ascontiguousarray(ref[:, 6])
    inobj = np.ascontiguousarray(g[f"{name}_inobj"].astype(np.int32))
    assert lib.rumi_test_material_fr(C.byref(m), N, vp(n), vp(wi), vp(wo), vp(inobj), vp(xi), vp(pp),
                                     vp(g[f"{name}_tin"]), vp(g[f"{name}_vr"]), vp(fr)) == 0
    np.testing.assert_allclose(fr, g[f"{name}_fr"], rtol=1e-5, atol=1e-7)


def test_gpu_medium_phase_camera_match_reference(golden, lib):
    v = golden("volume.npz")
    N = v["smax"].shape[0]
    out = np.zeros((N, 9), np.float32)
    assert lib.rumi_test_distance_sample(vp(v["sigma_s"]), vp(v["sigma_a"]), N, vp(v["smax"]), vp(v["xi"]),
                                         vp(v["xa"]), vp(out)) == 0
    ref = v["out"]
    outcome = np.where(ref[:, 0] == 1, 1, np.where(ref[:, 2] == 1, 2, 0))
    np.testing.assert_array_equal(out[:, 0].astype(int), outcome)
    sc = outcome == 1
    np.testing.assert_allclose(out[sc, 1], ref[sc, 1], rtol=1e-5)
    np.testing.assert_allclose(out[:, 2:5], ref[:, 3:6], rtol=1e-5)
    np.testing.assert_allclose(out[:, 5:8], ref[:, 6:9], rtol=1e-5)
    g = golden("materials.npz")
    N = g["iso_d"].shape[0]
    ph = np.zeros((N, 4), np.float32)
    assert lib.rumi_test_phase_sample(N, vp(g["iso_d"]), 0.0, vp(g["iso_u"]), vp(ph)) == 0
    np.testing.assert_allclose(ph, g["iso_out"], rtol=0, atol=1e-5)
    c = golden("camera.npz")
    cam = _capi.rumi_camera()
    cam.position = _capi.f3(*c["pos"])
    cam.basis = _capi.f16(*c["basis"])
    cam.y_ratio, cam.fov_deg = float(c["y_ratio"]), float(c["fov"])
    N = c["pix"].shape[0]
    co = np.zeros((N, 6), np.float32)
    assert lib.rumi_test_camera_rays(C.byref(cam), int(c["W"]), int(c["H"]), N, vp(c["pix"].astype(np.int32)),
                                     vp(c["smp"]), None, vp(co)) == 0
    np.testing.assert_allclose(co, c["out"][:, 0:6], rtol=0, atol=1e-6)


def test_gpu_thin_lens_rays_match_reference(lib, golden):
    """Thin-lens camera rays (Pinhole::DepthOfField) against the reference's own rays for
    the same lens uniforms; device sinf/cosf differ from the host's by an ulp or two."""
    from test_oracle_golden import _dof_camera
    g = golden("camera_dof.npz")
    N = g["pix"].shape[0]
    pix = np.ascontiguousarray(g["pix"].astype(np.int32))
    lens_u = np.ascontiguousarray(g["out"][:, 8:10])
    for i in range(N):
        cam = _dof_camera(g, i)
        out = np.zeros(6, np.float32)
        assert lib.rumi_test_camera_rays(C.byref(cam), int(g["W"]), int(g["H"]), 1, vp(pix[i]),
                                         vp(np.ascontiguousarray(g["smp"][i])), vp(lens_u[i]), vp(out)) == 0
        np.testing.assert_allclose(out, g["out"][i, 0:6], rtol=0, atol=2e-6)


@pytest.mark.parametrize("builder", [lambda: scenes.cornell_pt(32, 32, 4, 2), lambda: scenes.cornell_dof_pt(32, 32, 4, 2)])
def test_gpu_frame_matches_oracle_per_pixel_two_vertices(builder):
    """With the same Philox streams, paths of two vertices (camera ray, one bounce, light
    sampling at both) agree with the oracle pixel by pixel to float rounding."""
    sc = builder()
    gs = rumi_b200.GpuScene(sc)
    film, st = gs.render(spp=4, seed=21)
    gs.close()
    ofilm, onan = O.OracleScene(sc).render_pt(2, 4, 21)
    assert st["nan_samples"] == onan == 0
    rel = np.abs(film - ofilm) / np.maximum(np.abs(ofilm), 1e-3)
    assert np.mean(rel.max(2) > 1e-3) <= 2.0 / (32 * 32), float(rel.max())


@pytest.mark.parametrize("fixture,builder", __import__("test_oracle_golden").WHITTED_CASES)
def test_gpu_whitted_matches_reference_3sigma(golden, fixture, builder):
    from test_oracle_golden import frames_vs_reference
    frames_vs_reference(gpu_frames(builder(), 32, 15000), golden(fixture))


@pytest.mark.parametrize("fixture,builder", __import__("test_oracle_golden").WHITTED_CASES)
def test_gpu_whitted_matches_oracle_per_pixel(fixture, builder):
    """No hemisphere sampling on the Whitted path: with the same Philox streams the GPU's
    frame equals the oracle's pixel by pixel, up to float rounding; a glass lobe or
    medium-shadow decision that lands within an ulp of its threshold may flip."""
    sc = builder()
    gs = rumi_b200.GpuScene(sc)
    film, st = gs.render(spp=4, seed=31)
    gs.close()
    ofilm, onan = O.OracleScene(sc).render_whitted(sc.tracer.max_depth, 4, 31)
    assert st["nan_samples"] == onan == 0
    rel = np.abs(film - ofilm) / np.maximum(np.abs(ofilm), 1e-3)
    assert np.mean(rel.max(2) > 1e-3) <= 0.01, float(np.mean(rel.max(2) > 1e-3))
    assert abs(film.sum() / ofilm.sum() - 1.0) < 5e-3


def test_gpu_whitted_depth_zero_is_direct_lighting_only():
    """max_depth 0: camera rays only; a mirror seen directly is black, the walls carry
    next-event estimation, the light its emission."""
    sc = scenes.whitted(scenes.cornell_pt(32, 32, 4, 8), max_depth=0)
    gs = rumi_b200.GpuScene(sc)
    film, _ = gs.render(spp=4, seed=5)
    gs.close()
    ofilm, _ = O.OracleScene(sc).render_whitted(0, 4, 5)
    rel = np.abs(film - ofilm) / np.maximum(np.abs(ofilm), 1e-3)
    assert rel.max() < 1e-3
    assert (ofilm.reshape(-1, 3).sum(1) == 0).any()


def test_gpu_thin_lens_frames_match_reference_3sigma(golden):
    from test_oracle_golden import frames_vs_reference
    frames_vs_reference(gpu_frames(scenes.cornell_dof_pt(32, 32, 16, 8), 32, 14000),
                        golden("image_cornell_dof32.npz"))


def test_gpu_hg_phase_matches_oracle(lib):
    rng = np.random.default_rng(3)
    N = 2048
    d = rng.normal(size=(N, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    u = (rng.integers(0, 1 << 24, (N, 2)) / float(1 << 24)).astype(np.float32)
    for gval in (0.7, -0.3):
        out = np.zeros((N, 4), np.float32)
        assert lib.rumi_test_phase_sample(N, vp(d), gval, vp(u), vp(out)) == 0
        ref = np.zeros(4, np.float32)
        for i in range(0, N, 7):
            O.lib().orc_phase_sample(O.P(O.f32(d[i])), gval, float(u[i, 0]), float(u[i, 1]), O.P(ref))
            np.testing.assert_allclose(out[i], ref, rtol=1e-4, atol=2e-5)
        # mean cosine of a Henyey-Greenstein lobe is g
        assert abs(np.mean(np.sum(out[:, 0:3] * d, 1)) - gval) < 0.03


def test_gpu_pixel_samples_match_oracle(lib):
    for spp in (16, 25, 32, 64):
        n = 4 * spp
        s = np.tile(np.arange(spp, dtype=np.int32), 4)
        pix = np.repeat(np.array([0, 7, 1000, 123456], np.int64), spp)
        out = np.zeros((n, 2), np.float32)
        assert lib.rumi_test_pixel_samples(n, vp(s), spp, vp(pix), 42, vp(out)) == 0
        ref = np.zeros(2, np.float32)
        for i in range(n):
            O.lib().orc_pixel_sample(int(s[i]), spp, int(pix[i]), 42, O.P(ref))
            np.testing.assert_array_equal(out[i], ref)


@pytest.mark.parametrize("depth,tol,max_frac", [(1, 1e-4, 0.0), (2, 1e-3, 0.10), (8, None, None)])
def test_gpu_render_matches_oracle_per_pixel(depth, tol, max_frac):
    """Same seed, same random stream: the GPU wavefront and the oracle's sequential
    restatement agree pixel by pixel up to float rounding.  Deep paths are chaotic --
    the oracle against itself with the camera moved by one ulp differs by more than 1e-3
    on ~30% of pixels at depth 8 and on none at depth 1 -- so depth 1 is compared
    tightly, depth 2 loosely, depth 8 through the image sum."""
    sc = scenes.cornell_pt(48, 48, 16, depth)
    gs = rumi_b200.GpuScene(sc)
    film, st = gs.render(spp=16, seed=77)
    gs.close()
    ofilm, onan = O.OracleScene(sc).render_pt(depth, 16, 77)
    assert st["nan_samples"] == onan == 0
    if tol is not None:
        rel = np.abs(film - ofilm) / np.maximum(np.abs(ofilm), 1e-3)
        assert np.mean(rel.max(2) > tol) <= max_frac
    assert abs(film.sum() / ofilm.sum() - 1.0) < 2e-3


def test_gpu_render_matches_reference_3sigma(golden):
    g = golden("image_cornell32.npz")
    sc = scenes.cornell_pt(32, 32, 16, 8)
    gs = rumi_b200.GpuScene(sc)
    frames = []
    for s in range(32):
        film, st = gs.render(spp=16, seed=9000 + s)
        assert st["nan_samples"] == 0
        frames.append(film / 16.0)
    gs.close()
    fr = np.stack(frames).astype(np.float64)
    m, se = fr.mean(0), fr.std(0, ddof=1) / np.sqrt(fr.shape[0])
    sig = np.sqrt(se ** 2 + g["stderr"].astype(np.float64) ** 2) + 1e-6
    z = np.abs(m - g["mean"]) / sig
    assert np.mean(z > 3.0) < 0.01, np.mean(z > 3.0)
    assert abs(m.mean() / g["mean"].mean() - 1.0) < 0.01


def test_gpu_render_is_deterministic_and_wave_size_invariant():
    sc = scenes.cornell_pt(40, 24, 9, 6)
    gs = rumi_b200.GpuScene(sc)
    a, _ = gs.render(spp=9, seed=5)
    b, _ = gs.render(spp=9, seed=5)
    c, _ = gs.render(spp=9, seed=5, wave_paths=999)  # 111 pixels per wave, ragged last wave
    d, _ = gs.render(spp=9, seed=6)
    gs.close()
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)
    assert not np.array_equal(a, d)


def test_gpu_edge_cases():
    # empty scene: no primitives, no lights -> black film, no error
    from rumi_b200.scene import Scene, Pinhole, Film, PathTracer
    sc = Scene()
    sc.camera, sc.image, sc.tracer = Pinhole((0, 0, -1)), Film(8, 4, 1), PathTracer(3)
    gs = rumi_b200.GpuScene(sc)
    film, st = gs.render(spp=1, seed=1)
    assert film.shape == (4, 8, 3) and not film.any()
    t, prim, _, _ = gs.trace(np.array([[0, 0, 0, 0, 0, 1, 1e30]], np.float32))
    assert t[0] == 0 and prim[0] == -1
    gs.close()
    # zero-direction ray (BVHAccel::Travel returns a miss), empty batch, depth 1
    sc = scenes.cornell_pt(8, 8, 1, 1)
    gs = rumi_b200.GpuScene(sc)
    t, prim, _, _ = gs.trace(np.array([[0.5, 0.5, 0.5, 0, 0, 0, 1e30]], np.float32))
    assert t[0] == 0 and prim[0] == -1
    t, prim, _, _ = gs.trace(np.zeros((0, 7), np.float32))
    assert t.shape == (0,)
    film, st = gs.render(spp=1, seed=1)
    assert np.isfinite(film).all()
    with pytest.raises(_capi.RumiError):
        gs.render(spp=0, seed=1)
    gs.close()


def test_gpu_full_size_bvh_bound_workload_properties():
    """The 1024x1024, 64 spp, depth-10 workload on the 1,048,576-triangle mesh: finite,
    NaN-free, and two independent seeds agree on the image mean within noise."""
    sc = scenes.bvh_bound_pt(1024, 1024, 64, 10, levels=9, seed=7)
    gs = rumi_b200.GpuScene(sc)
    a, sa = gs.render(seed=1)
    b, sb = gs.render(seed=2)
    gs.close()
    assert sa["paths"] == 1024 * 1024 * 64
    assert sa["nan_samples"] == 0 and sb["nan_samples"] == 0
    assert np.isfinite(a).all() and np.isfinite(b).all()
    ma, mb = a.mean() / 64, b.mean() / 64
    assert ma > 0.05
    assert abs(ma / mb - 1.0) < 2e-3


def test_gpu_bvh_bound_workload_rows_match_reference_3sigma(golden):
    """The headline workload itself -- 1,048,576-triangle displaced sphere with
    per-triangle albedo in the Cornell box, 1024x1024, 64 spp, depth 10, NEE -- against
    the reference renderer's frames of eight full image rows (48 independent reference
    frames of those rows): per-pixel means within 3 sigma on >= 99% of the pixels and the
    strip mean within 1%."""
    g = golden("image_bvh_bound_rows.npz")
    rows = [int(r) for r in g["rows"]]
    sc = scenes.bvh_bound_pt(1024, 1024, 64, 10, levels=9, seed=7)
    gs = rumi_b200.GpuScene(sc)
    frames = []
    for s in range(32):
        film, st = gs.render(seed=31000 + s)
        assert st["nan_samples"] == 0
        frames.append(film[rows] / 64.0)
    gs.close()
    fr = np.stack(frames).astype(np.float64)
    m, se = fr.mean(0), fr.std(0, ddof=1) / np.sqrt(fr.shape[0])
    sig = np.sqrt(se ** 2 + g["stderr"].astype(np.float64) ** 2) + 1e-6
    z = np.abs(m - g["mean"]) / sig
    assert np.mean(z > 3.0) < 0.01, np.mean(z > 3.0)
    ref_mean = float(np.mean(g["frame_means"]))
    ref_se = float(np.std(g["frame_means"], ddof=1) / np.sqrt(len(g["frame_means"])))
    gpu_se = float(np.std(fr.mean((1, 2, 3)), ddof=1) / np.sqrt(fr.shape[0]))
    assert abs(m.mean() / ref_mean - 1.0) < 0.01
    assert abs(m.mean() - ref_mean) < 4.0 * np.hypot(ref_se, gpu_se) + 1e-6


def gpu_frames(sc, n, seed0, spp=16):
    gs = rumi_b200.GpuScene(sc)
    frames = []
    for s in range(n):
        film, st = gs.render(spp=spp, seed=seed0 + s)
        assert st["nan_samples"] == 0
        frames.append(film / float(spp))
    gs.close()
    return frames


def test_gpu_pt_medium_and_glass_match_reference_3sigma(golden):
    from test_oracle_golden import frames_vs_reference
    sc = scenes.volumetric_caustic(32, 32, 16, 4, 5, parity=True)
    sc.tracer = scenes.PathTracer(8)
    frames_vs_reference(gpu_frames(sc, 32, 11000), golden("image_caustic_pt32.npz"))


def test_gpu_pt_subsurface_matches_reference_3sigma(golden):
    from test_oracle_golden import frames_vs_reference
    frames_vs_reference(gpu_frames(scenes.subsurface_cornell(32, 32, 16, 12), 32, 12000), golden("image_sss_pt32.npz"))


@pytest.mark.parametrize("fixture,bdpt", [("image_sss_medium_pt32.npz", False), ("image_sss_medium_bdpt32.npz", True)])
def test_gpu_subsurface_in_a_medium_matches_reference_3sigma(golden, fixture, bdpt):
    """A subsurface sphere inside the scene's medium: path traced (the sphere's walk
    inside, the medium outside) and under BDPT."""
    from test_oracle_golden import frames_vs_reference, sss_in_medium
    frames_vs_reference(gpu_frames(sss_in_medium(bdpt), 32, 15000), golden(fixture))


@pytest.mark.parametrize("fixture,builder", [
    ("image_glass_pt32.npz", lambda: scenes.absorbing_glass_cornell()),
    ("image_glass_bdpt32.npz", lambda: scenes.with_bdpt(scenes.absorbing_glass_cornell())),
    ("image_two_lights_medium_pt32.npz", lambda: scenes.with_medium(scenes.cornell_two_lights_pt(32, 32, 16, 8))),
    ("image_sphere_light_medium_bdpt32.npz",
     lambda: scenes.with_bdpt(scenes.with_medium(scenes.cornell_sphere_light_pt(32, 32, 16, 8)))),
    ("image_cornell_medium_bdpt32.npz", lambda: scenes.with_medium(scenes.cornell_bdpt(32, 32, 16, 4, 5))),
])
def test_gpu_glass_and_lights_in_a_medium_match_reference_3sigma(golden, fixture, builder):
    """Coloured glass (Beer-Lambert absorption inside) path traced and under BDPT; two area
    lights in a medium path traced; the spherical emitter in a medium under BDPT."""
    from test_oracle_golden import frames_vs_reference
    frames_vs_reference(gpu_frames(builder(), 32, 17000), golden(fixture))


@pytest.mark.parametrize("fixture,kind", [("image_sphere_light_medium_pt32.npz", "sphere"),
                                          ("image_two_lights_medium_bdpt32.npz", "two_bdpt")])
def test_gpu_lights_in_a_medium_match_reference_3sigma(golden, fixture, kind):
    """A spherical emitter inside the medium (path traced: NEE with the binary shadow
    transmittance) and two area lights inside it under BDPT."""
    from test_oracle_golden import frames_vs_reference, lights_in_medium
    frames_vs_reference(gpu_frames(lights_in_medium(kind), 32, 16000), golden(fixture))


@pytest.mark.parametrize("fixture,builder", [
    ("image_cornell_bdpt32.npz", lambda: scenes.cornell_bdpt(32, 32, 16, 4, 5)),
    ("image_caustic_bdpt32.npz", lambda: scenes.volumetric_caustic(32, 32, 16, 4, 5, parity=True)),
    # the volumetric-caustic workload's own subpath lengths (6 light, 7 eye vertices: the
    # 8-vertex kernel instantiation, every strategy up to path length 12)
    ("image_caustic_bdpt67_32.npz", lambda: scenes.volumetric_caustic(32, 32, 16, 6, 7, parity=True)),
    # a subsurface sphere (BSDF sampling and Fr of Subsurface, no random walk in BDPT) and a
    # glossy sphere
    ("image_sss_bdpt32.npz", lambda: _bdpt45(scenes.subsurface_cornell(32, 32, 16, 12))),
    # a thin-lens camera: the reference's BDPT turns depth of field off when constructed
    ("image_dof_bdpt32.npz", lambda: _bdpt45(scenes.cornell_dof_pt(32, 32, 16, 8))),
    # a displaced-sphere mesh with per-triangle albedo (the workload's mesh kind)
    ("image_mesh_bdpt32.npz", lambda: _bdpt45(scenes.bvh_bound_pt(32, 32, 16, 10, levels=3, seed=7))),
])
def test_gpu_bdpt_matches_reference_3sigma(golden, fixture, builder):
    """BDPT with MIS (all strategies incl. light tracing splats through the film plane)
    against the reference's BidirectionalPathTracer frames."""
    from test_oracle_golden import frames_vs_reference
    frames_vs_reference(gpu_frames(builder(), 32, 13000), golden(fixture))


def _bdpt45(sc):
    sc.tracer = scenes.BidirectionalPathTracer(4, 5)
    return sc


@pytest.mark.parametrize("fixture,builder", [
    ("image_sphere_light_pt32.npz", lambda: scenes.cornell_sphere_light_pt(32, 32, 16, 8)),
    ("image_two_lights_pt32.npz", lambda: scenes.cornell_two_lights_pt(32, 32, 16, 8)),
    ("image_sphere_light_bdpt32.npz", lambda: _bdpt45(scenes.cornell_sphere_light_pt(32, 32, 16, 8))),
    ("image_two_lights_bdpt32.npz", lambda: _bdpt45(scenes.cornell_two_lights_pt(32, 32, 16, 8))),
])
def test_gpu_sphere_and_multiple_area_lights_match_reference_3sigma(golden, fixture, builder):
    """An emissive sphere as the area light (points from Sphere::ShapeSampling,
    src/Shape/sphere.cpp:152-170, pdf 1 / (4 pi r^2); BDPT emission about Sphere::Normal)
    and two area lights picked uniformly (Scene::LightsUniformSampling,
    src/Scene/scene.cpp:91-97), path tracer and BDPT, against the reference's frames."""
    from test_oracle_golden import frames_vs_reference
    frames_vs_reference(gpu_frames(builder(), 32, 14000), golden(fixture))


def _floor_scene(light, size=48, spp=64):
    """A single Lambertian plane under one light: every path is direct illumination."""
    from rumi_b200.scene import (Scene, Model, Matte, Rect, Emissive, AreaLight, SpotLight, Pinhole, Film,
                                 PathTracer, identity16)
    sc = Scene()
    q = np.array([[-2, 0, -2], [3, 0, -2], [3, 0, 3], [-2, 0, 3]], np.float32)
    sc.add(Model(np.stack([np.stack([q[0], q[2], q[1]]), np.stack([q[0], q[3], q[2]])]).astype(np.float32)),
           Matte(1.0, (0.5, 0.5, 0.5)))
    if light == "spot":
        sc.lights.append(SpotLight((0.5, 0.98, 0.5), (0.0, -1.0, 0.0), 30.0, (50.0, 50.0, 50.0)))
    else:
        r = Rect((0.45, 0.98, 0.45), (0.1, 0.0, 0.0), (0.0, 0.0, 0.1), 64)
        sc.add(r, Emissive(1.0, (120.0, 120.0, 120.0)))
        sc.lights.append(AreaLight(r))
    sc.camera = Pinhole((0.5, 0.5, -1.4), identity16(), 1.0, fov=40.0)
    sc.image = Film(size, size, spp)
    sc.tracer = PathTracer(1)
    return sc


def test_gpu_bdpt_spot_light_direct_illumination_equals_pt():
    """Spot lights have no reference counterpart, so BDPT's handling of them (a delta
    light vertex: cone emission sampling, no cosine at the light, the eye-hits-light
    strategy weighted zero) is checked for consistency: on a single plane every path is
    direct illumination, which the path tracer's NEE computes exactly, and the MIS-combined
    BDPT strategies (NEE connection + light tracing) must give the same image."""
    from rumi_b200.scene import BidirectionalPathTracer
    g = rumi_b200.GpuScene(_floor_scene("spot"))
    try:
        pt = np.mean([g.render(seed=s)[0] for s in range(8)], 0).astype(np.float64)
        bd = np.mean([g.render(seed=100 + s, tracer=BidirectionalPathTracer(2, 3))[0] for s in range(8)], 0)
        assert abs(bd.sum() / pt.sum() - 1.0) < 0.01
        lit = pt.sum(-1) > 0.1 * pt.sum(-1).max()
        np.testing.assert_allclose(bd.sum(-1)[lit].sum(), pt.sum(-1)[lit].sum(), rtol=0.01)
    finally:
        g.close()


def test_gpu_bdpt_volumetric_caustic_spot_workload():
    """The volumetric-caustic workload proper (30 degree spot, HG g = 0.7): finite, free of
    NaN samples, reproducible up to the summation order of the light-tracing splats
    (atomics), and brighter than path tracing, which cannot sample the caustic (a delta
    light seen through glass)."""
    sc = scenes.volumetric_caustic(48, 48, 16, 6, 7)
    g = rumi_b200.GpuScene(sc)
    try:
        a, st = g.render(seed=3)
        b, _ = g.render(seed=3)
        assert np.isfinite(a).all() and st["nan_samples"] == 0 and a.sum() > 0
        np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-5 * float(np.abs(a).max()))
        pt, _ = g.render(seed=3, tracer=scenes.PathTracer(12))
        assert a.sum() > 1.5 * pt.sum()
    finally:
        g.close()


def test_gpu_rmse_at_matched_spp_within_5pct_of_reference(golden):
    """RMSE against the reference's own 65,536-spp image of the Cornell workload (32x32,
    depth 8), at matched spp (16): our mean over 1024 frames within 5% of the mean RMSE of
    256 reference frames (tests/golden/rmse_cornell32.npz)."""
    g = golden("rmse_cornell32.npz")
    gt = g["gt"].astype(np.float64)
    gs = rumi_b200.GpuScene(scenes.cornell_pt(32, 32, 16, 8))
    try:
        rm = []
        for s in range(1024):
            film, st = gs.render(seed=20000 + s)
            rm.append(float(np.sqrt(((film.astype(np.float64) / 16.0 - gt) ** 2).mean())))
        ratio = float(np.mean(rm) / np.mean(g["ref_rmse"]))
        assert abs(ratio - 1.0) < 0.05, (ratio, np.mean(rm), np.mean(g["ref_rmse"]))
    finally:
        gs.close()


@pytest.mark.parametrize("builder", [lambda: scenes.cornell_pt(48, 40, 9, 8),
                                     lambda: scenes.volumetric_caustic(40, 32, 4, 4, 5, parity=True),
                                     lambda: scenes.whitted(scenes.cornell_pt(32, 32, 4, 8))])
def test_gpu_overlapped_schedule_equals_serial(builder):
    """The default schedule traces each bounce's shadow rays on a second stream beside the
    next bounce's closest-hit rays; the film is bit-identical to the one-stream order
    (RUMI_FLAG_SERIAL), over several waves."""
    sc = builder()
    if not isinstance(sc.tracer, scenes.RayTracer):
        sc.tracer = scenes.PathTracer(8)
    gs = rumi_b200.GpuScene(sc)
    a, sa = gs.render(spp=9, seed=77, wave_paths=4000)
    b, sb = gs.render(spp=9, seed=77, wave_paths=4000, serial=True)
    gs.close()
    np.testing.assert_array_equal(a, b)
    assert sa["rays_extend"] == sb["rays_extend"] and sa["rays_shadow"] == sb["rays_shadow"]


@pytest.mark.parametrize("fixture,builder", [
    ("hits_cornell.npz", lambda: scenes.cornell_pt(64, 64, 16, 8)),
    ("hits_mesh5.npz", lambda: scenes.bvh_bound_pt(64, 64, 4, 10, levels=5, seed=7)),
])
def test_gpu_hits_equal_oracle_ties_included_in_any_order(golden, fixture, builder):
    """A primitive hit at exactly the best distance as another goes to the larger id
    whatever order the traversal meets them in: the GPU's ids equal the oracle's exhaustive
    scan (which reports the last tied primitive in canonical order), for the rays in their
    own order and shuffled (other rays share each warp)."""
    g = golden(fixture)
    sc = builder()
    gs = rumi_b200.GpuScene(sc)
    rays = np.ascontiguousarray(g["rays"], np.float32)
    ot, op = O.OracleScene(sc).trace(rays8(rays))
    t, prim, _, _ = gs.trace(rays)
    np.testing.assert_array_equal(t, ot)
    np.testing.assert_array_equal(prim, op)
    perm = np.random.default_rng(5).permutation(rays.shape[0])
    t2, prim2, _, _ = gs.trace(np.ascontiguousarray(rays[perm]))
    np.testing.assert_array_equal(prim2, prim[perm])
    np.testing.assert_array_equal(t2, t[perm])
    gs.close()


def _with_pt(sc, depth):
    sc.tracer = scenes.PathTracer(depth)
    return sc


@pytest.mark.parametrize("builder", [
    lambda: scenes.cornell_pt(48, 40, 9, 8),
    lambda: scenes.bvh_bound_pt(64, 48, 4, 10, levels=6, seed=7),
    lambda: _with_pt(scenes.volumetric_caustic(48, 40, 4, 4, 5, parity=True), 8),
])
def test_gpu_every_traversal_scheme_renders_the_same_film(builder):
    """Closest hits do not depend on the walk (exact primitive tests, conservative node
    culling -- the eight-wide tree's quantised boxes contain the exact ones -- and ties to
    the larger id), so every scheme of rumi_render_params.trace_mode, the binary walks (1-4)
    and the compressed eight-wide walk (5), renders the identical film."""
    sc = builder()
    gs = rumi_b200.GpuScene(sc)
    ref, st0 = gs.render(seed=3, trace_mode=4)
    assert st0["nan_samples"] == 0 and ref.sum() > 0
    for mode in (0, 1, 2, 3, 5):
        film, st = gs.render(seed=3, trace_mode=mode)
        np.testing.assert_array_equal(film, ref, err_msg=f"trace_mode {mode}")
        assert st["rays_extend"] == st0["rays_extend"] and st["rays_shadow"] == st0["rays_shadow"]
    gs.close()


def test_gpu_eight_wide_walk_hits_match_reference_on_the_1m_mesh():
    """The compressed eight-wide walk (trace_mode 5) on the 1,048,576-triangle workload mesh:
    camera rays rendered at depth 1 hit exactly what the binary walk hits (same film,
    same primary ray count), and its node bytes per ray are below the binary tree's."""
    sc = scenes.bvh_bound_pt(256, 256, 4, 1, levels=9, seed=7)
    gs = rumi_b200.GpuScene(sc)
    a, sa = gs.render(seed=5, trace_mode=4, count_stats=True)
    b, sb = gs.render(seed=5, trace_mode=5, count_stats=True)
    gs.close()
    np.testing.assert_array_equal(a, b)
    assert sa["extend_prim_tests"] > 0 and sb["extend_prim_tests"] > 0
    assert sb["extend_node_fetches"] < sa["extend_node_fetches"]


def _trace_scheme(gs, rays, mode, anyhit=False):
    """rumi_test_trace_scheme: ray queries (n, 7) through traversal scheme `mode`."""
    r8 = np.zeros((rays.shape[0], 8), np.float32)
    r8[:, 0:3], r8[:, 4:7], r8[:, 7] = rays[:, 0:3], rays[:, 3:6], rays[:, 6]
    t = np.zeros(rays.shape[0], np.float32)
    prim = np.zeros(rays.shape[0], np.int32)
    _capi.check(_capi.load().rumi_test_trace_scheme(gs.h, rays.shape[0], r8.ctypes.data_as(C.c_void_p),
                                                    1 if anyhit else 0, mode, t.ctypes.data_as(C.c_void_p),
                                                    prim.ctypes.data_as(C.c_void_p)), "rumi_test_trace_scheme")
    return t, prim


def _signed_zero_rays(rng, n):
    """Rays whose directions hold exact +0.0 and -0.0 components: axis-aligned ones (two
    zero components) and ones in a coordinate plane (one), zero signs drawn at random,
    origins inside the box."""
    o = rng.uniform(0.05, 0.95, (2 * n, 3)).astype(np.float32)
    d = np.zeros((2 * n, 3), np.float32)
    axis = rng.integers(0, 3, 2 * n)
    d[np.arange(n), axis[:n]] = rng.choice([-1.0, 1.0], n)
    ab = rng.normal(size=(n, 2))
    ab /= np.linalg.norm(ab, axis=1, keepdims=True)
    for k in range(n):
        a = axis[n + k]
        d[n + k, (a + 1) % 3], d[n + k, (a + 2) % 3] = ab[k]
    zero = d == 0.0
    d[zero] = np.where(rng.random(zero.sum()) < 0.5, np.float32(-0.0), np.float32(0.0))
    assert np.signbit(d[zero]).any() and (~np.signbit(d[zero])).any()
    return np.concatenate([o, d, np.full((2 * n, 1), 3.4e38, np.float32)], 1).astype(np.float32)


def test_gpu_every_traversal_scheme_finds_the_reference_hits_with_signed_zero_directions():
    """Direction components of exactly -0.0 and +0.0 (axis-aligned and in-plane rays): a
    -0.0 component has a negative reciprocal although it does not compare below zero, so a
    walk that picked near and far planes by `d < 0` would cull every box the ray starts in.
    Every scheme's closest hits and occlusion answers equal the reference's BVHAccel."""
    sc = scenes.bvh_bound_pt(64, 64, 4, 10, levels=5, seed=7)
    rng = np.random.default_rng(23)
    rays = _signed_zero_rays(rng, 2048)
    gs = rumi_b200.GpuScene(sc)
    rs = refimpl.RefScene(sc, seed=1)
    rt, rid = rs.trace(rays)
    assert (rid >= 0).mean() > 0.5  # the box is open toward the camera: rays leaving that way miss
    sh = rays.copy()
    sh[:, 6] = np.where(rt > 0, rt * 0.5, 0.5)
    _, rocc = rs.trace(sh, anyhit=True)
    for mode in (1, 2, 3, 4, 5):
        t, prim = _trace_scheme(gs, rays, mode)
        ties = tie_mask(t, prim, rt, rid)
        assert np.all((prim == rid) | ties), f"trace_mode {mode}: {np.sum((prim != rid) & ~ties)} rays differ"
        np.testing.assert_array_equal(t, rt, err_msg=f"trace_mode {mode}")
        _, occ = _trace_scheme(gs, sh, mode, anyhit=True)
        np.testing.assert_array_equal(occ, rocc, err_msg=f"trace_mode {mode} (any-hit)")
    gs.close()
