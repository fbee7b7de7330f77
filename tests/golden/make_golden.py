#!/usr/bin/env python3
"""Generates the golden fixtures of tests/golden/ by running the REFERENCE renderer's own
routines (oracle/_ref/librumi_ref.so, built from the reference sources by
oracle/build_ref.py) on seeded inputs.  The reference ships no tests or fixtures, so
these are its outputs captured here; the fixtures travel with the repository so GPU tests
need no reference checkout.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "rumi-renderer_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import refimpl  # noqa: E402
from rumi_b200 import scenes  # noqa: E402
from rumi_b200.scene import Matte, Glossy, Specular, Dielectric, Subsurface, Emissive  # noqa: E402

F32 = np.float32


def u24(rng, shape):
    """Uniforms of the exact form m * 2^-24 (what the GPU's Philox conversion yields)."""
    return (rng.integers(0, 1 << 24, size=shape).astype(np.float64) / float(1 << 24)).astype(F32)


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v.astype(F32)


def rays_in_box(rng, n, lo=0.02, hi=0.98):
    o = rng.uniform(lo, hi, (n, 3)).astype(F32)
    d = unit(rng, n)
    return np.concatenate([o, d, np.full((n, 1), 3.4e38, F32)], 1).astype(F32)


def camera_rays(rng, n, cam=(0.5, 0.5, -1.4), lo=(0.05, 0.05, 0.05), hi=(0.95, 0.95, 0.95)):
    o = np.tile(np.asarray(cam, F32), (n, 1))
    tgt = rng.uniform(lo, hi, (n, 3)).astype(F32)
    d = (tgt - o)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(F32)
    return np.concatenate([o, d, np.full((n, 1), 3.4e38, F32)], 1).astype(F32)


def hit_fixture(scene, rays, path, extra=None):
    rs = refimpl.RefScene(scene, seed=1)
    t, ids, nrm = rs.trace(rays, want_normals=True)
    # shadow queries with a finite tmax (half of each closest-hit distance, or 0.7)
    tmax = np.where(t > 0, t * 0.5, 0.7).astype(F32)
    sh = rays.copy()
    sh[:, 6] = tmax
    ta, occ = rs.trace(sh, anyhit=True)
    sh2 = rays.copy()
    sh2[:, 6] = np.where(t > 0, t + 0.01, 0.7).astype(F32)
    tb, occ2 = rs.trace(sh2, anyhit=True)
    data = dict(rays=rays, t=t, prim=ids, normal=nrm, shadow_rays=sh, shadow_occluded=occ, shadow2_rays=sh2,
                shadow2_occluded=occ2)
    if extra:
        data.update(extra)
    np.savez_compressed(path, **data)
    rs.close()
    print(path, "hit fraction", float((ids >= 0).mean()))


def material_fixture(path, rng):
    L = refimpl.lib()
    mats = {
        "matte": Matte(0.8, (0.7, 0.4, 0.2)),
        "glossy": Glossy(0.5, 0.4, 20.0, (0.6, 0.6, 0.9)),
        "glossy_ks_only": Glossy(0.0, 0.9, 10.0, (1.0, 1.0, 1.0)),
        "specular": Specular(0.9, (1.0, 0.9, 0.8)),
        "dielectric": Dielectric(1.5, 1.00029, (0.1, 0.2, 0.3)),
        "subsurface": Subsurface(1.3, 1.0, (0.8, 0.6, 0.4), (0.05, 0.1, 0.2), 2.0),
        "emissive": Emissive(3.0, (17.0, 12.0, 4.0)),
    }
    N = 256
    out = {}
    for name, m in mats.items():
        p = refimpl.f32(m.ref_params())
        n = unit(rng, N)
        wo = unit(rng, N)
        # a quarter of the cases: wo in the same hemisphere as n, near grazing
        k = N // 4
        wo[:k] = np.where((np.sum(wo[:k] * n[:k], 1) < 0)[:, None], -wo[:k], wo[:k])
        u = u24(rng, (N, 3))
        samp = np.zeros((N, 9), F32)
        for i in range(N):
            # inject the uniforms in the order the reference draws them
            if m.type == 0:
                seq = u[i, 1:3]
            elif m.type == 1:
                seq = u[i, 0:3]
            elif m.type in (4, 5):
                seq = u[i, 0:1]
            else:
                seq = u[i, 0:0]
            keep = refimpl.inject(seq)
            L.ref_material_sample(m.type, refimpl.P(p), refimpl.P(refimpl.f32(wo[i])), refimpl.P(refimpl.f32(n[i])),
                                  refimpl.P(samp[i]))
            L.ref_inject_off()
            del keep
        # Fr with the sampled direction and the sampled lobe state
        inobj = rng.integers(0, 2, N).astype(np.int32)
        t_in = rng.uniform(0.01, 2.0, N).astype(F32)
        vr = rng.uniform(0.5, 1.5, (N, 3)).astype(F32)
        fr = np.zeros((N, 3), F32)
        for i in range(N):
            wi = samp[i, 0:3].copy()
            L.ref_material_fr(m.type, refimpl.P(p), refimpl.P(refimpl.f32(n[i])), refimpl.P(refimpl.f32(wi)),
                              refimpl.P(refimpl.f32(wo[i])), int(inobj[i]), float(samp[i, 5]), float(samp[i, 6]),
                              float(t_in[i]), refimpl.P(refimpl.f32(vr[i])), refimpl.P(refimpl.f32([1, 1, 1])),
                              refimpl.P(fr[i]))
        out.update({f"{name}_params": p, f"{name}_n": n, f"{name}_wo": wo, f"{name}_u": u, f"{name}_sample": samp,
                    f"{name}_inobj": inobj, f"{name}_tin": t_in, f"{name}_vr": vr, f"{name}_fr": fr,
                    f"{name}_type": np.int32(m.type)})
    # Fresnel over incidence angles and both sides
    d = unit(rng, N)
    n = unit(rng, N)
    kr = np.array([L.ref_fresnel(refimpl.P(refimpl.f32(d[i])), refimpl.P(refimpl.f32(n[i])), 1.5, 1.00029)
                   for i in range(N)], F32)
    out.update(fresnel_d=d, fresnel_n=n, fresnel_kr=kr)
    # isotropic phase
    dd = unit(rng, N)
    uu = u24(rng, (N, 2))
    iso = np.zeros((N, 4), F32)
    for i in range(N):
        keep = refimpl.inject(uu[i])
        L.ref_isotropic_sample(refimpl.P(refimpl.f32(dd[i])), refimpl.P(iso[i]))
        L.ref_inject_off()
        del keep
    out.update(iso_d=dd, iso_u=uu, iso_out=iso)
    np.savez_compressed(path, **out)
    print(path)


def volume_fixture(path, rng):
    L = refimpl.lib()
    N = 512
    ss = np.array([0.4, 0.3, 0.2], F32)
    sa = np.array([0.05, 0.1, 0.02], F32)
    smax = rng.uniform(0.0, 8.0, N).astype(F32)
    smax[:16] = 0.0
    xi = u24(rng, N)
    xa = u24(rng, N)
    out = np.zeros((N, 10), F32)
    for i in range(N):
        keep = refimpl.inject(np.array([xi[i], xa[i]], F32))
        L.ref_volume_distance_sampling(refimpl.P(ss), refimpl.P(sa), float(smax[i]), refimpl.P(out[i]))
        L.ref_inject_off()
        del keep
    # box segments (Intersect + MaxDistance)
    bmin, bmax = np.array([0, 0, 0], F32), np.array([1, 1, 1], F32)
    o = rng.uniform(-0.5, 1.5, (N, 3)).astype(F32)
    d = unit(rng, N)
    thit = np.where(rng.uniform(size=N) < 0.5, 0.0, rng.uniform(0.0, 2.0, N)).astype(F32)
    seg = np.zeros((N, 4), F32)
    for i in range(N):
        L.ref_volume_segment(refimpl.P(bmin), refimpl.P(bmax), refimpl.P(refimpl.f32(o[i])),
                             refimpl.P(refimpl.f32(d[i])), float(thit[i]), refimpl.P(seg[i]))
    np.savez_compressed(path, sigma_s=ss, sigma_a=sa, smax=smax, xi=xi, xa=xa, out=out, seg_o=o, seg_d=d,
                        seg_thit=thit, seg_out=seg, bmin=bmin, bmax=bmax)
    print(path)


def camera_fixture(path, rng):
    L = refimpl.lib()
    N = 256
    cam = scenes.cornell_camera()
    pos, basis = refimpl.f32(cam.position), refimpl.f32(cam.basis)
    W, H = 96, 64
    pix = np.stack([rng.integers(0, W, N), rng.integers(0, H, N)], 1).astype(np.int32)
    smp = u24(rng, (N, 2))
    out = np.zeros((N, 8), F32)
    for i in range(N):
        L.ref_camera_cast(refimpl.P(pos), refimpl.P(basis), 0.75, 40.0, W, H, int(pix[i, 0]), int(pix[i, 1]),
                          float(smp[i, 0]), float(smp[i, 1]), refimpl.P(out[i]))
    np.savez_compressed(path, pos=pos, basis=basis, y_ratio=np.float32(0.75), fov=np.float32(40.0), W=W, H=H, pix=pix,
                        smp=smp, out=out)
    print(path)


def camera_dof_fixture(path, rng):
    """Thin-lens camera rays of the reference (Pinhole::DepthOfField + CastViewRay) under
    a rotated basis with a translation column, which the reference also adds to _up and
    _right; each ray reports the two RandomFloat() values it drew."""
    L = refimpl.lib()
    N = 256
    ax, ay = 0.3, -0.45
    rx = np.array([[1, 0, 0], [0, np.cos(ax), -np.sin(ax)], [0, np.sin(ax), np.cos(ax)]])
    ry = np.array([[np.cos(ay), 0, np.sin(ay)], [0, 1, 0], [-np.sin(ay), 0, np.cos(ay)]])
    basis = np.eye(4)
    basis[:3, :3] = ry @ rx
    basis[:3, 3] = (0.02, -0.03, 0.01)
    basis = refimpl.f32(basis.reshape(16))
    pos = refimpl.f32([0.4, 0.6, -1.2])
    W, H = 80, 60
    pix = np.stack([rng.integers(0, W, N), rng.integers(0, H, N)], 1).astype(np.int32)
    smp = u24(rng, (N, 2))
    focal = rng.uniform(0.5, 5.0, N).astype(F32)
    lens = rng.uniform(0.01, 0.3, N).astype(F32)
    seeds = rng.integers(1, 1 << 30, N).astype(np.uint32)
    out = np.zeros((N, 10), F32)
    for i in range(N):
        L.ref_camera_cast_dof(refimpl.P(pos), refimpl.P(basis), 0.75, 35.0, float(focal[i]), float(lens[i]), W, H,
                              int(pix[i, 0]), int(pix[i, 1]), float(smp[i, 0]), float(smp[i, 1]), int(seeds[i]),
                              refimpl.P(out[i]))
    np.savez_compressed(path, pos=pos, basis=basis, y_ratio=np.float32(0.75), fov=np.float32(35.0), W=W, H=H,
                        pix=pix, smp=smp, focal=focal, lens=lens, out=out)
    print(path)


def TEXTURE_CASES(img, hdr):
    """(fixture name, scene) of the texture and image-based-light frames."""
    import texture_cases as TC
    return [("image_tex_pt32.npz", TC.textured_cornell(32, 32, 16, 8, img)),
            ("image_tex_whitted32.npz", scenes.whitted(TC.textured_cornell(32, 32, 16, 8, img))),
            ("image_ibl_pt32.npz", TC.ibl_scene(32, 32, 16, 8, hdr)),
            ("image_ibl_whitted32.npz", scenes.whitted(TC.ibl_scene(32, 32, 16, 8, hdr))),
            ("image_tex_bdpt32.npz", TC.textured_bdpt(32, 32, 16, img))]


def image_fixture(path, size=32, spp=16, depth=8, seeds=64, scene=None):
    """Reference renders of a workload at a small size: per-pixel mean radiance over
    `seeds` independent frames and its standard error (spread across frames, which
    includes the frame-level correlation of the reference's shared sample sets)."""
    sc = scene if scene is not None else scenes.cornell_pt(size, size, spp, depth)
    frames = []
    for s in range(seeds):
        rs = refimpl.RefScene(sc, seed=1000 + s)
        film, nans = rs.render(7000 + s)
        frames.append(film / rs.spp)
        rs.close()
    fr = np.stack(frames).astype(np.float64)
    mean = fr.mean(0).astype(F32)
    stderr = (fr.std(0, ddof=1) / np.sqrt(seeds)).astype(F32)
    # per-frame image means: the reference's frames share sample sets across pixels, so the
    # image mean's spread is not the per-pixel spreads added in quadrature
    frame_means = fr.mean((1, 2, 3)).astype(np.float64)
    np.savez_compressed(path, mean=mean, stderr=stderr, seeds=seeds, spp=spp, depth=depth, size=size,
                        frame_means=frame_means)
    print(path, "mean", mean.reshape(-1, 3).mean(0))


ADJOINT_MEDIUM = dict(sigma_s=(0.45, 0.35, 0.25), sigma_a=(0.04, 0.06, 0.09), g=0.0)


def adjoint_delta():
    """Positive loss weights (a weighted image sum), seeded."""
    return (0.5 + np.random.default_rng(77).random((32, 32, 3))).astype(F32)


def _adjoint_fd_seed(s, h):
    alb0 = scenes.random_albedo(4 * 4 ** 3, 23)
    d64 = adjoint_delta().astype(np.float64)
    row = []
    for c in range(3):
        ap, am = alb0.copy(), alb0.copy()
        ap[:, c] += F32(h)
        am[:, c] -= F32(h)
        sums = []
        for a in (ap, am):
            sc = scenes.inverse_rendering(32, 32, 16, 4, levels=3, albedo=a, medium=ADJOINT_MEDIUM)
            rs = refimpl.RefScene(sc, seed=1000 + s)
            film, _ = rs.render(7000 + s)
            rs.close()
            sums.append((d64 * film).sum())
        row.append((sums[0] - sums[1]) / (2.0 * h))
    return row


def adjoint_fixture(path, seeds=960, h=1e-3):
    """The reference renderer's own finite-difference gradient for the albedo adjoint: the
    inverse-rendering scene at 32x32, 16 spp, depth 4, with a 256-triangle mesh and the
    reference's isotropic medium.  For each colour channel c the whole mesh's albedo is
    moved by +-h in c and the frame is re-rendered with the same srand seed (albedo drives
    no sampling decision of the reference, so the two frames share every random number);
    fd[seed, c] = (<delta, film+> - <delta, film->) / 2h with seeded positive weights
    delta (adjoint_delta)."""
    base = scenes.inverse_rendering(32, 32, 16, 4, levels=3, medium=ADJOINT_MEDIUM)
    alb0 = scenes.random_albedo(4 * 4 ** 3, 23)
    assert np.array_equal(base.flatten().tri_albedo[-alb0.shape[0]:], alb0)
    delta = adjoint_delta()
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 1, 32)) as pool:
        rows = pool.starmap(_adjoint_fd_seed, [(s, h) for s in range(seeds)])
    fd = np.array(rows)
    np.savez_compressed(path, delta=delta, fd=fd, mean=fd.mean(0), stderr=fd.std(0, ddof=1) / np.sqrt(seeds),
                        h=h, seeds=seeds, sigma_s=np.array(ADJOINT_MEDIUM["sigma_s"], F32),
                        sigma_a=np.array(ADJOINT_MEDIUM["sigma_a"], F32))
    print(path, "fd mean", fd.mean(0), "stderr", fd.std(0, ddof=1) / np.sqrt(seeds))


def _gt_rows(args):
    size, spp, depth, row0, row1, seed = args
    sc = scenes.cornell_pt(size, size, spp, depth)
    rs = refimpl.RefScene(sc, seed=seed)
    film, _, nans = rs.render_rows(seed, row0, row1)
    n = rs.spp
    rs.close()
    return row0, row1, film[row0:row1] / n, nans


def rmse_fixture(path, size=32, depth=8, gt_spp=65536, spp=16, frames=256, procs=8):
    """Reference ground truth and the reference's own error at matched spp: the Cornell
    workload at 32x32 rendered by the reference with 65,536 spp per pixel (rows split over
    processes, each with its own srand seed), and the RMSE against it of 256 independent
    reference frames at 16 spp."""
    import multiprocessing as mp
    rows_per = size // procs
    jobs = [(size, gt_spp, depth, k * rows_per, (k + 1) * rows_per, 90000 + k) for k in range(procs)]
    gt = np.zeros((size, size, 3), np.float64)
    with mp.get_context("spawn").Pool(procs) as pool:
        for r0, r1, part, nans in pool.map(_gt_rows, jobs):
            gt[r0:r1] = part
    sc = scenes.cornell_pt(size, size, spp, depth)
    rmse = []
    for s in range(frames):
        rs = refimpl.RefScene(sc, seed=1000 + s)
        film, _ = rs.render(7000 + s)
        img = film.astype(np.float64) / rs.spp
        rs.close()
        rmse.append(float(np.sqrt(((img - gt) ** 2).mean())))
    np.savez_compressed(path, gt=gt.astype(F32), ref_rmse=np.array(rmse), gt_spp=gt_spp, spp=spp, depth=depth,
                        size=size)
    print(path, "reference RMSE at", spp, "spp:", np.mean(rmse), "+-", np.std(rmse) / np.sqrt(frames))


def LIGHT_CASES():
    """A spherical area light and two area lights, path traced and under BDPT (4, 5)."""
    from rumi_b200.scene import BidirectionalPathTracer

    def bdpt(sc):
        sc.tracer = BidirectionalPathTracer(4, 5)
        return sc
    return [("image_sphere_light_pt32.npz", scenes.cornell_sphere_light_pt(32, 32, 16, 8)),
            ("image_two_lights_pt32.npz", scenes.cornell_two_lights_pt(32, 32, 16, 8)),
            ("image_sphere_light_bdpt32.npz", bdpt(scenes.cornell_sphere_light_pt(32, 32, 16, 8))),
            ("image_two_lights_bdpt32.npz", bdpt(scenes.cornell_two_lights_pt(32, 32, 16, 8)))]


C2_ROWS = (64, 192, 320, 448, 576, 704, 832, 960)


def _c2_worker(args):
    seeds, rows = args
    sc = scenes.bvh_bound_pt(1024, 1024, 64, 10, levels=9, seed=7)
    rs = refimpl.RefScene(sc, seed=1)
    out = []
    for s in seeds:
        strip = np.zeros((len(rows), 1024, 3), np.float64)
        for k, r in enumerate(rows):
            film, light, nans = rs.render_rows(50000 + 97 * s + k, r, r + 1)
            strip[k] = (film[r] + light[r]) / rs.spp
        out.append(strip)
    spp = rs.spp
    rs.close()
    return out, spp


def c2_strip_fixture(path, seeds=48, procs=8):
    """The headline BVH-bound workload itself (Cornell box + 1,048,576-triangle displaced
    sphere with per-triangle albedo, 1024x1024, 64 spp, depth 10, NEE) rendered by the
    reference on eight full image rows: per-pixel mean and standard error over `seeds`
    independent frames of those rows, and the per-frame strip means."""
    import multiprocessing as mp
    jobs = [(list(range(k, seeds, procs)), C2_ROWS) for k in range(procs)]
    frames = []
    with mp.get_context("spawn").Pool(procs) as pool:
        for out, spp in pool.map(_c2_worker, jobs):
            frames += out
    fr = np.stack(frames)
    mean = fr.mean(0).astype(F32)
    stderr = (fr.std(0, ddof=1) / np.sqrt(seeds)).astype(F32)
    np.savez_compressed(path, mean=mean, stderr=stderr, rows=np.array(C2_ROWS, np.int32), seeds=seeds, spp=spp,
                        depth=10, frame_means=fr.mean((1, 2, 3)))
    print(path, "strip mean", mean.reshape(-1, 3).mean(0), "frames", len(frames))


def obj_fixture(path):
    """The reference's Model(file, transform) on the OBJ texts of tests/obj_cases.py."""
    import tempfile
    from obj_cases import CASES, TRANSFORMS
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for case, text in CASES.items():
            p = os.path.join(d, case + ".obj")
            with open(p, "wb") as f:
                f.write(text.encode())
            for tname, m in TRANSFORMS.items():
                v, n = refimpl.load_obj(p, m)
                out[f"{case}__{tname}__v"] = v
                out[f"{case}__{tname}__n"] = n
    np.savez_compressed(path, **out)
    print(path, len(out) // 2, "loads")


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "textures":
        import tempfile
        import texture_cases as TC
        with tempfile.TemporaryDirectory() as d:
            img, hdr = TC.case_files(d)
            for name, sc in TEXTURE_CASES(img, hdr):
                image_fixture(os.path.join(HERE, name), scene=sc)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "combos2":
        # an image-based light around a medium (PT), the Cornell spheres in a medium under
        # BDPT, the spherical emitter under the Whitted ray tracer
        import tempfile
        import texture_cases as TC
        with tempfile.TemporaryDirectory() as d:
            img, hdr = TC.case_files(d)
            image_fixture(os.path.join(HERE, "image_ibl_medium_pt32.npz"),
                          scene=scenes.with_medium(TC.ibl_scene(32, 32, 16, 8, hdr)))
        image_fixture(os.path.join(HERE, "image_cornell_medium_bdpt32.npz"),
                      scene=scenes.with_medium(scenes.cornell_bdpt(32, 32, 16, 4, 5)))
        image_fixture(os.path.join(HERE, "image_sphere_light_whitted32.npz"),
                      scene=scenes.whitted(scenes.cornell_sphere_light_pt(32, 32, 16, 8)))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "tex_medium":
        # the textured Cornell scene inside a medium, path traced and under BDPT
        import tempfile
        import texture_cases as TC
        with tempfile.TemporaryDirectory() as d:
            img, hdr = TC.case_files(d)
            image_fixture(os.path.join(HERE, "image_tex_medium_pt32.npz"),
                          scene=scenes.with_medium(TC.textured_cornell(32, 32, 16, 8, img)))
            image_fixture(os.path.join(HERE, "image_tex_medium_bdpt32.npz"),
                          scene=scenes.with_medium(TC.textured_bdpt(32, 32, 16, img)))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "whitted":
        image_fixture(os.path.join(HERE, "image_whitted_cornell32.npz"),
                      scene=scenes.whitted(scenes.cornell_pt(32, 32, 16, 8)))
        image_fixture(os.path.join(HERE, "image_whitted_caustic32.npz"),
                      scene=scenes.whitted(scenes.volumetric_caustic(32, 32, 16, 4, 5, parity=True)))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "dof":
        camera_dof_fixture(os.path.join(HERE, "camera_dof.npz"), np.random.default_rng(88))
        image_fixture(os.path.join(HERE, "image_cornell_dof32.npz"), scene=scenes.cornell_dof_pt(32, 32, 16, 8))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "lights":
        for name, sc in LIGHT_CASES():
            image_fixture(os.path.join(HERE, name), scene=sc)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "c2":
        c2_strip_fixture(os.path.join(HERE, "image_bvh_bound_rows.npz"))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "obj":
        obj_fixture(os.path.join(HERE, "obj_loader.npz"))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "rmse":
        rmse_fixture(os.path.join(HERE, "rmse_cornell32.npz"))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "adjoint":
        adjoint_fixture(os.path.join(HERE, "adjoint_fd_ref32.npz"))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "media":
        sc = scenes.volumetric_caustic(32, 32, 16, 4, 5, parity=True)
        sc.tracer = scenes.PathTracer(8)
        image_fixture(os.path.join(HERE, "image_caustic_pt32.npz"), scene=sc)
        image_fixture(os.path.join(HERE, "image_sss_pt32.npz"), scene=scenes.subsurface_cornell(32, 32, 16, 12))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "more":
        # the thin-lens camera under BDPT (the reference's BDPT turns depth of field off),
        # and the Whitted ray tracer over the subsurface + glossy scene and two lights
        sc = scenes.cornell_dof_pt(32, 32, 16, 8)
        sc.tracer = scenes.BidirectionalPathTracer(4, 5)
        image_fixture(os.path.join(HERE, "image_dof_bdpt32.npz"), scene=sc)
        image_fixture(os.path.join(HERE, "image_sss_whitted32.npz"),
                      scene=scenes.whitted(scenes.subsurface_cornell(32, 32, 16, 12)))
        image_fixture(os.path.join(HERE, "image_two_lights_whitted32.npz"),
                      scene=scenes.whitted(scenes.cornell_two_lights_pt(32, 32, 16, 8)))
        # BDPT over a displaced-sphere mesh with per-triangle albedo (the workload's mesh
        # kind, 256 triangles)
        sc = scenes.bvh_bound_pt(32, 32, 16, 10, levels=3, seed=7)
        sc.tracer = scenes.BidirectionalPathTracer(4, 5)
        image_fixture(os.path.join(HERE, "image_mesh_bdpt32.npz"), scene=sc)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "sss_medium":
        # a subsurface sphere (its own random walk inside) within a scene medium, path
        # traced and under BDPT (4, 5)
        for name, bdpt in (("image_sss_medium_pt32.npz", False), ("image_sss_medium_bdpt32.npz", True)):
            sc = scenes.subsurface_cornell(32, 32, 16, 12)
            sc.volume = scenes.HomogeneousVolume((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.3, 0.3, 0.3),
                                                 (0.05, 0.05, 0.05), 0.0)
            if bdpt:
                sc.tracer = scenes.BidirectionalPathTracer(4, 5)
            image_fixture(os.path.join(HERE, name), scene=sc)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "lights_medium":
        # the spherical emitter inside the scene medium (path traced), and two area lights
        # in it under BDPT (4, 5)
        sc = scenes.cornell_sphere_light_pt(32, 32, 16, 8)
        sc.volume = scenes.HomogeneousVolume((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.3, 0.3, 0.3),
                                             (0.05, 0.05, 0.05), 0.0)
        image_fixture(os.path.join(HERE, "image_sphere_light_medium_pt32.npz"), scene=sc)
        sc = scenes.cornell_two_lights_pt(32, 32, 16, 8)
        sc.volume = scenes.HomogeneousVolume((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.3, 0.3, 0.3),
                                             (0.05, 0.05, 0.05), 0.0)
        sc.tracer = scenes.BidirectionalPathTracer(4, 5)
        image_fixture(os.path.join(HERE, "image_two_lights_medium_bdpt32.npz"), scene=sc)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "combos":
        # coloured (absorbing) glass under the three integrators; the sphere light and the two
        # lights inside a medium under the integrators not covered yet
        for name, sc in (("image_glass_pt32.npz", scenes.absorbing_glass_cornell()),
                         ("image_glass_bdpt32.npz", scenes.with_bdpt(scenes.absorbing_glass_cornell())),
                         ("image_glass_whitted32.npz", scenes.whitted(scenes.absorbing_glass_cornell())),
                         ("image_sphere_light_medium_bdpt32.npz",
                          scenes.with_bdpt(scenes.with_medium(scenes.cornell_sphere_light_pt(32, 32, 16, 8)))),
                         ("image_two_lights_medium_pt32.npz",
                          scenes.with_medium(scenes.cornell_two_lights_pt(32, 32, 16, 8)))):
            image_fixture(os.path.join(HERE, name), scene=sc)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "dof_whitted":
        image_fixture(os.path.join(HERE, "image_dof_whitted32.npz"),
                      scene=scenes.whitted(scenes.cornell_dof_pt(32, 32, 16, 8)))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "bdpt_sss":
        # BDPT over the subsurface sphere and the glossy sphere (materials the reference's
        # BDPT evaluates through BSDFSampling / Fr only)
        sc = scenes.subsurface_cornell(32, 32, 16, 12)
        sc.tracer = scenes.BidirectionalPathTracer(4, 5)
        image_fixture(os.path.join(HERE, "image_sss_bdpt32.npz"), scene=sc)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "bdpt67":
        # the volumetric-caustic workload's subpath lengths (6 light, 7 eye vertices) on its
        # area-light, isotropic-medium variant
        image_fixture(os.path.join(HERE, "image_caustic_bdpt67_32.npz"),
                      scene=scenes.volumetric_caustic(32, 32, 16, 6, 7, parity=True))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "bdpt":
        image_fixture(os.path.join(HERE, "image_cornell_bdpt32.npz"), scene=scenes.cornell_bdpt(32, 32, 16, 4, 5))
        image_fixture(os.path.join(HERE, "image_caustic_bdpt32.npz"),
                      scene=scenes.volumetric_caustic(32, 32, 16, 4, 5, parity=True))
        return
    rng = np.random.default_rng(20261203)
    c1 = scenes.cornell_pt(64, 64, 16, 8)
    rays = np.concatenate([rays_in_box(rng, 3072), camera_rays(rng, 1024)])
    hit_fixture(c1, rays, os.path.join(HERE, "hits_cornell.npz"))
    m5 = scenes.bvh_bound_pt(64, 64, 4, 10, levels=5, seed=7)
    tris = m5.flatten().tri_vertices
    rays = np.concatenate([camera_rays(rng, 2048, lo=(0.2, 0.1, 0.2), hi=(0.8, 0.6, 0.8)), rays_in_box(rng, 2048)])
    hit_fixture(m5, rays, os.path.join(HERE, "hits_mesh5.npz"),
                extra=dict(mesh_checksum=np.array(scenes.mesh_checksum(tris)), n_tris=np.int32(tris.shape[0])))
    material_fixture(os.path.join(HERE, "materials.npz"), rng)
    volume_fixture(os.path.join(HERE, "volume.npz"), rng)
    camera_fixture(os.path.join(HERE, "camera.npz"), rng)
    image_fixture(os.path.join(HERE, "image_cornell32.npz"))
    image_fixture(os.path.join(HERE, "image_cornell_bdpt32.npz"), scene=scenes.cornell_bdpt(32, 32, 16, 4, 5))
    image_fixture(os.path.join(HERE, "image_caustic_bdpt32.npz"),
                  scene=scenes.volumetric_caustic(32, 32, 16, 4, 5, parity=True))
    sc = scenes.volumetric_caustic(32, 32, 16, 4, 5, parity=True)
    sc.tracer = scenes.PathTracer(8)
    image_fixture(os.path.join(HERE, "image_caustic_pt32.npz"), scene=sc)
    image_fixture(os.path.join(HERE, "image_sss_pt32.npz"), scene=scenes.subsurface_cornell(32, 32, 16, 12))


if __name__ == "__main__":
    main()
