"""The CPU oracle (oracle/rumi_oracle.c) pinned to the reference: every check compares
the oracle with golden vectors produced by the reference's own routines
(tests/golden/make_golden.py) on identical inputs and injected uniforms."""
import numpy as np
import pytest

import oraclelib as O
from rumi_b200 import scenes
from rumi_b200.scene import Material

KAT = [  # Philox4x32-10 known answers (Salmon et al. 2011, Random123 distribution)
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    assert tuple(O.philox(ctr, key)) == want


def rays8(r7):
    r8 = np.zeros((r7.shape[0], 8), np.float32)
    r8[:, 0:3], r8[:, 4:7], r8[:, 7] = r7[:, 0:3], r7[:, 3:6], r7[:, 6]
    return r8


def tie_mask(t_a, id_a, t_b, id_b):
    """Rays whose ids differ only because two primitives are hit at the same t (the
    reference keeps whichever its traversal order tests last)."""
    return (id_a != id_b) & (t_a == t_b) & (t_a > 0)


@pytest.mark.parametrize("fixture,builder", [
    ("hits_cornell.npz", lambda: scenes.cornell_pt(64, 64, 16, 8)),
    ("hits_mesh5.npz", lambda: scenes.bvh_bound_pt(64, 64, 4, 10, levels=5, seed=7)),
])
def test_oracle_hits_match_reference(golden, fixture, builder):
    g = golden(fixture)
    sc = builder()
    if "mesh_checksum" in g.files:
        assert scenes.mesh_checksum(sc.flatten().tri_vertices) == str(g["mesh_checksum"])
    os_ = O.OracleScene(sc)
    t, prim = os_.trace(rays8(g["rays"]))
    ties = tie_mask(t, prim, g["t"], g["prim"])
    assert np.all((prim == g["prim"]) | ties)
    assert ties.mean() < 0.01
    assert np.array_equal(t, g["t"])  # same float operations -> same distances
    for key in ("shadow", "shadow2"):
        _, occ = os_.trace(rays8(g[f"{key}_rays"]), anyhit=True)
        assert np.array_equal(occ, g[f"{key}_occluded"])


MATERIALS = ["matte", "glossy", "glossy_ks_only", "specular", "dielectric", "subsurface", "emissive"]


def material_from_params(mtype, p):
    m = Material(int(mtype))
    if m.type in (0, 2, 3):
        m.kd = float(p[0])
    elif m.type == 1:
        m.kd, m.ks, m.exponent = float(p[0]), float(p[1]), float(p[2])
    else:
        m.eta_in, m.eta_out = float(p[0]), float(p[1])
    m.rgb = tuple(float(x) for x in p[3:6])
    m.rgb2 = tuple(float(x) for x in p[6:9])
    m.density = float(p[9])
    return m


@pytest.mark.parametrize("name", MATERIALS)
def test_oracle_material_sample_and_fr(golden, name):
    g = golden("materials.npz")
    m = O.material_struct(material_from_params(g[f"{name}_type"], g[f"{name}_params"]))
    n, wo, u, ref = g[f"{name}_n"], g[f"{name}_wo"], g[f"{name}_u"], g[f"{name}_sample"]
    L = O.lib()
    import ctypes as C
    out = np.zeros(9, np.float32)
    for i in range(n.shape[0]):
        L.orc_material_sample(C.byref(m), O.P(O.f32(wo[i])), O.P(O.f32(n[i])), O.P(O.f32(u[i])), O.P(out))
        np.testing.assert_allclose(out[0:3], ref[i, 0:3], rtol=0, atol=1e-5)
        np.testing.assert_array_equal(out[3:5], ref[i, 3:5])           # Le, go_into_object
        np.testing.assert_allclose(out[5:9], ref[i, 5:9], rtol=1e-5, atol=1e-7)
    fr = np.zeros(3, np.float32)
    for i in range(n.shape[0]):
        s = ref[i]
        L.orc_material_fr(C.byref(m), O.P(O.f32(n[i])), O.P(O.f32(s[0:3])), O.P(O.f32(wo[i])),
                          int(g[f"{name}_inobj"][i]), float(s[5]), float(s[6]), float(g[f"{name}_tin"][i]),
                          O.P(O.f32(g[f"{name}_vr"][i])), O.P(fr))
        np.testing.assert_allclose(fr, g[f"{name}_fr"][i], rtol=1e-5, atol=1e-7)


def test_oracle_fresnel_and_isotropic(golden):
    g = golden("materials.npz")
    L = O.lib()
    for d, n, kr in zip(g["fresnel_d"], g["fresnel_n"], g["fresnel_kr"]):
        assert L.orc_fresnel(O.P(O.f32(d)), O.P(O.f32(n)), 1.5, 1.00029) == pytest.approx(kr, rel=1e-6, abs=1e-7)
    out = np.zeros(4, np.float32)
    for d, u, ref in zip(g["iso_d"], g["iso_u"], g["iso_out"]):
        L.orc_phase_sample(O.P(O.f32(d)), 0.0, float(u[0]), float(u[1]), O.P(out))
        np.testing.assert_allclose(out, ref, rtol=0, atol=1e-5)


def test_oracle_distance_sampling(golden):
    g = golden("volume.npz")
    L = O.lib()
    out = np.zeros(9, np.float32)
    for smax, xi, xa, ref in zip(g["smax"], g["xi"], g["xa"], g["out"]):
        L.orc_distance_sample(O.P(g["sigma_s"]), O.P(g["sigma_a"]), float(smax), float(xi), float(xa), O.P(out))
        # reference out: [returned, s, absorb, tau rgb, pdf rgb]
        outcome = 1 if ref[0] else (2 if ref[2] else 0)
        assert int(out[0]) == outcome
        if outcome == 1:
            assert out[1] == pytest.approx(ref[1], rel=1e-5)
        np.testing.assert_allclose(out[2:5], ref[3:6], rtol=1e-5)
        np.testing.assert_allclose(out[5:8], ref[6:9], rtol=1e-5)


def test_oracle_camera_rays(golden):
    g = golden("camera.npz")
    from rumi_b200.scene import Pinhole
    import rumi_b200._capi as capi
    import ctypes as C
    cam = capi.rumi_camera()
    cam.position = capi.f3(*g["pos"])
    cam.basis = capi.f16(*g["basis"])
    cam.y_ratio, cam.fov_deg = float(g["y_ratio"]), float(g["fov"])
    out = np.zeros(6, np.float32)
    for pix, smp, ref in zip(g["pix"], g["smp"], g["out"]):
        O.lib().orc_camera_ray(C.byref(cam), int(g["W"]), int(g["H"]), int(pix[0]), int(pix[1]), float(smp[0]),
                               float(smp[1]), 0.0, 0.0, O.P(out))
        np.testing.assert_allclose(out, ref[0:6], rtol=0, atol=1e-6)


def _dof_camera(g, i):
    import rumi_b200._capi as capi
    cam = capi.rumi_camera()
    cam.position = capi.f3(*g["pos"])
    cam.basis = capi.f16(*g["basis"])
    cam.y_ratio, cam.fov_deg = float(g["y_ratio"]), float(g["fov"])
    cam.focal_distance, cam.lens_radius = float(g["focal"][i]), float(g["lens"][i])
    return cam


def test_oracle_thin_lens_rays(golden):
    """Pinhole::DepthOfField + CastViewRay: lens point from sqrt(u1) * radius and angle
    u2 * 2 PI along _up / _right (the basis applied with its translation column), aimed
    at the pinhole ray's focal-plane point; the reference's own two RandomFloat() draws
    fed to the oracle."""
    import ctypes as C
    g = golden("camera_dof.npz")
    out = np.zeros(6, np.float32)
    for i, (pix, smp, ref) in enumerate(zip(g["pix"], g["smp"], g["out"])):
        cam = _dof_camera(g, i)
        O.lib().orc_camera_ray(C.byref(cam), int(g["W"]), int(g["H"]), int(pix[0]), int(pix[1]), float(smp[0]),
                               float(smp[1]), float(ref[8]), float(ref[9]), O.P(out))
        np.testing.assert_allclose(out, ref[0:6], rtol=0, atol=1e-6)
    # the lens moves the origins: the fixture is not the pinhole case
    assert np.abs(g["out"][:, 0:3] - g["pos"][None]).max() > 0.05


def test_oracle_thin_lens_frames_match_reference_3sigma(golden):
    """Cornell box through a thin lens focused at the white sphere's depth."""
    frames_vs_reference(oracle_frames(scenes.cornell_dof_pt(32, 32, 16, 8), 8, 24, 800),
                        golden("image_cornell_dof32.npz"))


def test_pixel_sampler_is_a_stratified_permutation():
    """Each pixel's n samples use every jittered-grid column and row exactly once, as the
    reference's without-replacement draws from its sqrt(n)^2 grid do."""
    import ctypes as C
    L = O.lib()
    for spp in (1, 4, 16, 64, 25, 32):
        d = int(np.sqrt(spp))
        out = np.zeros(2, np.float32)
        xs, ys = [], []
        for s in range(spp):
            L.orc_pixel_sample(s, spp, 12345, 99, O.P(out))
            xs.append(out[0])
            ys.append(out[1])
        xs, ys = np.array(xs), np.array(ys)
        assert np.all((xs >= 0) & (xs < 1) & (ys >= 0) & (ys < 1))
        if d * d == spp:
            assert sorted(np.bincount(np.floor(xs * d).astype(int), minlength=d)) == [d] * d
            assert sorted(np.bincount(np.floor(ys * d).astype(int), minlength=d)) == [d] * d
        else:
            assert sorted(np.floor(xs * spp).astype(int)) == list(range(spp))
        for n in (1, 5, 16, 33, 64):
            assert sorted(L.orc_perm(i, n, 0xABCDEF) for i in range(n)) == list(range(n))


def frames_vs_reference(frames, g, max_frac=0.01):
    """Per-pixel means within 3 sigma of the reference's frames (sigma from both sides'
    frame-to-frame spread) on all but max_frac of the pixels, and the image mean within 4
    sigma of the reference's (sigma of the image mean from the same spreads, at least 0.2%:
    caustic and medium scenes carry ~1% of image-mean noise at these frame counts)."""
    fr = np.stack(frames).astype(np.float64)
    m, se = fr.mean(0), fr.std(0, ddof=1) / np.sqrt(fr.shape[0])
    gse = g["stderr"].astype(np.float64)
    sig = np.sqrt(se ** 2 + gse ** 2) + 1e-6
    z = np.abs(m - g["mean"]) / sig
    frac = float(np.mean(z > 3.0))
    ratio = float(m.mean() / g["mean"].mean())
    if "frame_means" in g.files:
        # image-mean spread measured frame to frame on both sides (frame-level correlation
        # of the reference's shared pixel and light sample sets included)
        fm, gm = fr.mean((1, 2, 3)), g["frame_means"]
        rel_sigma = np.sqrt(fm.var(ddof=1) / fm.size + gm.var(ddof=1) / gm.size) / float(gm.mean())
    else:
        rel_sigma = np.sqrt((se ** 2).sum() + (gse ** 2).sum()) / g["mean"].astype(np.float64).sum()
    assert frac < max_frac, (frac, ratio)
    assert abs(ratio - 1.0) < max(4.0 * rel_sigma, 0.002), (frac, ratio, rel_sigma)
    return frac, ratio


def oracle_frames(sc, depth, n, seed0):
    os_ = O.OracleScene(sc)
    frames = []
    for s in range(n):
        film, nan = os_.render_pt(depth, 16, seed=seed0 + s)
        assert nan == 0
        frames.append(film / 16.0)
    return frames


WHITTED_CASES = [
    ("image_whitted_cornell32.npz", lambda: scenes.whitted(scenes.cornell_pt(32, 32, 16, 8))),
    ("image_whitted_caustic32.npz", lambda: scenes.whitted(scenes.volumetric_caustic(32, 32, 16, 4, 5, parity=True))),
    ("image_sss_whitted32.npz", lambda: scenes.whitted(scenes.subsurface_cornell(32, 32, 16, 12))),
    ("image_two_lights_whitted32.npz", lambda: scenes.whitted(scenes.cornell_two_lights_pt(32, 32, 16, 8))),
    ("image_dof_whitted32.npz", lambda: scenes.whitted(scenes.cornell_dof_pt(32, 32, 16, 8))),
    ("image_glass_whitted32.npz", lambda: scenes.whitted(scenes.absorbing_glass_cornell())),
    ("image_sphere_light_whitted32.npz", lambda: scenes.whitted(scenes.cornell_sphere_light_pt(32, 32, 16, 8))),
]


@pytest.mark.parametrize("fixture,builder", WHITTED_CASES)
def test_oracle_whitted_matches_reference_3sigma(golden, fixture, builder):
    """RayTracer (Whitted): mirror and glass chains, direct lighting at the first other
    surface, against the reference's own RayTracer frames."""
    sc = builder()
    os_ = O.OracleScene(sc)
    frames = []
    for s in range(32):
        film, nan = os_.render_whitted(sc.tracer.max_depth, 16, seed=900 + s)
        assert nan == 0
        frames.append(film / 16.0)
    frames_vs_reference(frames, golden(fixture))


def test_oracle_image_matches_reference_3sigma(golden):
    """Oracle PT frames of the Cornell workload (32x32) against the reference's frames."""
    frames_vs_reference(oracle_frames(scenes.cornell_pt(32, 32, 16, 8), 8, 24, 500), golden("image_cornell32.npz"))


def test_oracle_medium_and_glass_match_reference_3sigma(golden):
    """Homogeneous medium (free flight, absorption roulette, binary shadow transmittance,
    isotropic phase) around a glass sphere, path traced."""
    sc = scenes.volumetric_caustic(32, 32, 16, 4, 5, parity=True)
    frames_vs_reference(oracle_frames(sc, 8, 24, 700), golden("image_caustic_pt32.npz"))


@pytest.mark.parametrize("fixture,builder", [
    ("image_sphere_light_pt32.npz", lambda: scenes.cornell_sphere_light_pt(32, 32, 16, 8)),
    ("image_two_lights_pt32.npz", lambda: scenes.cornell_two_lights_pt(32, 32, 16, 8)),
])
def test_oracle_sphere_and_multiple_area_lights_match_reference_3sigma(golden, fixture, builder):
    """Next-event estimation toward a spherical area light (uniform points on the sphere,
    pdf 1 / (4 pi r^2)) and toward one of two area lights picked uniformly."""
    frames_vs_reference(oracle_frames(builder(), 8, 24, 1300), golden(fixture))


def test_oracle_subsurface_matches_reference_3sigma(golden):
    """Subsurface random walk and a glossy sphere, path traced to depth 12."""
    frames_vs_reference(oracle_frames(scenes.subsurface_cornell(32, 32, 16, 12), 12, 24, 900),
                        golden("image_sss_pt32.npz"))


def sss_in_medium(bdpt=False):
    """The subsurface + glossy Cornell scene inside a homogeneous medium filling the box
    (sigma_s 0.3, sigma_a 0.05, isotropic): the sphere's own random walk inside, the scene's
    medium outside."""
    sc = scenes.subsurface_cornell(32, 32, 16, 12)
    sc.volume = scenes.HomogeneousVolume((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.3, 0.3, 0.3), (0.05, 0.05, 0.05), 0.0)
    if bdpt:
        sc.tracer = scenes.BidirectionalPathTracer(4, 5)
    return sc


def lights_in_medium(kind):
    """The spherical emitter (path traced) or the two area lights (BDPT (4, 5)) inside the
    medium of sss_in_medium."""
    sc = scenes.cornell_sphere_light_pt(32, 32, 16, 8) if kind == "sphere" else scenes.cornell_two_lights_pt(32, 32, 16, 8)
    sc.volume = scenes.HomogeneousVolume((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.3, 0.3, 0.3), (0.05, 0.05, 0.05), 0.0)
    if kind == "two_bdpt":
        sc.tracer = scenes.BidirectionalPathTracer(4, 5)
    return sc


def test_oracle_sphere_light_in_a_medium_matches_reference_3sigma(golden):
    frames_vs_reference(oracle_frames(lights_in_medium("sphere"), 8, 24, 1500),
                        golden("image_sphere_light_medium_pt32.npz"))


@pytest.mark.parametrize("fixture,builder", [
    ("image_glass_pt32.npz", lambda: scenes.absorbing_glass_cornell()),
    ("image_two_lights_medium_pt32.npz", lambda: scenes.with_medium(scenes.cornell_two_lights_pt(32, 32, 16, 8))),
])
def test_oracle_glass_and_two_lights_in_a_medium_match_reference_3sigma(golden, fixture, builder):
    """Coloured glass (Beer-Lambert absorption inside) and two area lights in a medium,
    path traced."""
    sc = builder()
    frames_vs_reference(oracle_frames(sc, sc.tracer.max_depth, 24, 1600), golden(fixture))


def test_oracle_subsurface_in_a_medium_matches_reference_3sigma(golden):
    frames_vs_reference(oracle_frames(sss_in_medium(), 12, 24, 1400), golden("image_sss_medium_pt32.npz"))


def test_oracle_rmse_at_matched_spp_within_5pct_of_reference(golden):
    """The oracle's 16-spp frames against the reference's 65,536-spp image: mean RMSE within
    5% of the reference's own 16-spp RMSE."""
    g = golden("rmse_cornell32.npz")
    gt = g["gt"].astype(np.float64)
    frames = oracle_frames(scenes.cornell_pt(32, 32, 16, 8), 8, 64, 30000)
    rm = [float(np.sqrt(((f.astype(np.float64) - gt) ** 2).mean())) for f in frames]
    ratio = float(np.mean(rm) / np.mean(g["ref_rmse"]))
    assert abs(ratio - 1.0) < 0.05, ratio
